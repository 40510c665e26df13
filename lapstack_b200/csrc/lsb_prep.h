// Frame preparation on the device (lsb_prep.cu): the dust map, the quarter
// turns, the draft block mean and the resize of 16-bit interleaved frames.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "lapstack_b200.h"

namespace lsb {

struct DSpot;

// A dust map uploaded once (dust.rs:105 DustMap): the spots' rectangles and masks, each fill window's
// weight-0 map, the gains (flat mode), the pull-push scratch, and the layers of spots whose masks do
// not overlap (run in order).
struct DustDev {
    int W = 0, H = 0, mode = 0, nspots = 0;
    DSpot* spots = nullptr;
    uint8_t* masks = nullptr;
    uint8_t* wzero = nullptr;
    float* gains = nullptr;
    float* scratch = nullptr;
    int* list = nullptr;               // the spots, layer after layer
    std::vector<int> layer_off;        // layer k is list[layer_off[k] .. layer_off[k + 1])
    size_t scratch_bytes = 0;
    ~DustDev();
};

// Checks and uploads a map; on an error returns its text and leaves *out null.
std::string dust_create(const lsb_dust_map* m, DustDev** out);
// dust.rs:487 `apply_rgb16` in place on a W x H interleaved u16 frame on the device.
cudaError_t dust_apply_rgb16(const DustDev* d, uint16_t* rgb, cudaStream_t s);
// decode.rs:68 + :92: the turned (q quarter turns clockwise), 2^draft block-averaged frame; its size.
void turn_draft_dims(int w, int h, int q, int draft, int* ow, int* oh);
cudaError_t turn_draft_rgb16(const uint16_t* in, int w, int h, int q, int draft, uint16_t* out, cudaStream_t s);
// decode.rs:125 bilinear resize of an interleaved u16 frame.
cudaError_t resize_rgb16(const uint16_t* in, int sw, int sh, uint16_t* out, int w, int h, cudaStream_t s);

}  // namespace lsb
