// Internal interfaces between the engine's translation units (host side).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace lsb {

// Per-frame level-0 source transform: the inverse homography that maps an
// aligned pixel to its source point (align.rs:258 `inverse` of the frame's
// Sim::matrix) and the brightness gains (brightness.rs:124 `apply`).
struct FrameXform {
    double inv[9];
    float gain[3];
    int warp;      // 1: resample through `inv` (the pixel as shot where it leaves the frame)
    int affine;    // inv's last row is [0, 0, 1] (align.rs:485 `affine_row`)
    int gain_on;   // bit c: multiply channel c by gain[c] (|g - 1| > 1e-6)
    // the frame's 16-bit fixed-point level storage: 65535 / max(1, largest gain) and its inverse
    // (every Gaussian level of the frame is a convex combination of its gained inputs in [0, 1])
    float gscale, ginv;
};

enum SrcKind { SRC_U16 = 0, SRC_F32 = 1, SRC_G = 2 };

// One pyramid level's fold over all frames of a stack.
struct FoldArgs {
    int level, nframes;
    int W, H, W1, H1;
    int tiles_x, tiles_y, ntiles;
    // level-0 sources: interleaved u16 [n][H][W][3] or planar f32 [n][3][H][W]
    const uint16_t* src_u16;
    const float* src_f32;
    const FrameXform* xf;  // per frame, level 0 only
    int interp;            // align.rs Interp id for the warp
    // level >= 1 source and every level's output: planar [n][3][h][w] in the storage type
    const void* src_g;
    void* dst_g;
    // accumulator of this level: acc [3][H][W], best [H][W], winner [H][W] (depth level only)
    float* acc;
    float* best;
    uint16_t* winner;
    int use_chroma;
    // focus slices (level 0): [n][dh][dw], block k, measure
    void* slice;
    int dw, dh, bk;
    int focus_kind;  // 0 RDF, 1 SML
    int sml_step;
    int ntaps;
    int rdf13;  // the taps are the default ring difference filter (r_in 1, r_out 3)
    int* status;  // device error word
    // halo control (fuse.rs:112-136, 453-475): 1 at the guide level (select, and write each frame's
    // weight plane halo_w [n][H][W]); 2 at coarser levels (no selection: acc = sum w*L, best = sum w,
    // frames in order, with halo_w the weights REDUCEd to this level)
    int halo_mode;
    float halo_p;
    float* halo_w;
    cudaEvent_t between;  // host side: recorded between the REDUCE and the select launch (may be null)
    // what one fold_level call launches: the REDUCE of frames red_k0 .. red_k0 + red_n - 1
    // (none if red_n is 0) and, if select is set, the selection over frames sel_k0 .. sel_k1 - 1
    // (from sel_k0 > 0 it resumes from the acc / best / winner the frames before it left)
    int red_k0, red_n, select, sel_k0, sel_k1;
    // sel_groups > 1: the frames are split into that many groups selected side by side from a
    // fresh state, each into its slice of gacc [g][3][H][W] / gbest [g][H][W] / gwin [g][H][W],
    // then merged in group order (strict >, so the earliest frame with the largest energy wins)
    int sel_groups;
    float *gacc, *gbest;
    int* gwin;
    // level 0 only: fused0 set, the interior tiles (fold0_range(W, H, f0r)) are the fused kernel's, and
    // reduce_level_kernel / select_level_kernel walk the other ntiles tiles (fold0_border_tile)
    int fused0, f0r;
    int no_fused;  // 1: level 0 runs the two kernels on every tile (the fused kernel's cross-check)
    // 1: the level runs beside the registration chain: its persistent kernels take at most one CTA per
    // SM (they ask for BESIDE_SMEM of shared memory), so the chain's cooperative search keeps room
    int beside;
    cudaEvent_t after_fused;  // host side: recorded right after the fused level-0 kernel (may be null)
};
// shared memory a persistent fold kernel asks for beside the registration chain: more than half an SM's
constexpr size_t BESIDE_SMEM = 116 * 1024;

// Storage of the Gaussian levels >= 1 and the focus slices.
enum Storage { STORE_F32 = 0, STORE_UNORM16 = 1, STORE_F16 = 2 };

// Launchers (lsb_fold.cu).
cudaError_t fold_level(const FoldArgs& a, int src_kind, int storage, int radius, bool focus, cudaStream_t s, int grid_limit);
// The weighted average's accumulation (wav.rs:146-161): frames as level 0 of `a` reads them, weight planes
// wts [n][dh][dw] (grid scale k), out [3][H][W].
cudaError_t wav_accumulate(const FoldArgs& a, int src_kind, const float* wts, int n, int dw, int dh, int k, float* out, cudaStream_t s);
// Every frame through its warp (the pixel as shot where it leaves the frame):
// f32 planar [n][3][h][w], or u16 interleaved [n][h][w][3] rounded to the u16 step.
cudaError_t warp_frames(const uint16_t* frames, const FrameXform* xf, int interp, int w, int h, int n, bool u16_out, void* out,
                        cudaStream_t s);
cudaError_t set_focus_taps(const float* taps3, int ntaps, cudaStream_t s);
size_t fold_smem_bytes(int radius, bool focus);

// brightness.rs:93 `ratio` on the device for frame k: its gains from its
// brightness partials (part as bright_sums writes them, nparts per frame,
// summed in order), the gain flags and the frame's fixed-point storage scale,
// written into *xf (the frame's entry).
cudaError_t frame_gain(const double* part, int k, int nparts, FrameXform* xf, cudaStream_t s);

// Residual (top) level: fuse.rs:248 `fuse_residuals` over all frames' tops.
struct ResidualArgs {
    const void* tops;  // [n][3][h][w] storage type
    int n, w, h;
    int top_rule, radius, bins;
    float* dev;  // scratch [n][h][w]
    float* ent;  // scratch [n][h][w]
    float* out;  // [3][h][w]
    const FrameXform* xf;  // per frame: the fixed-point storage's scale
};
cudaError_t fuse_residuals(const ResidualArgs& a, int storage, const float* lnp, cudaStream_t s);

// Collapse: out_l = acc_l + EXPAND(coarse) (pyramid.rs:219); at level 0 also clamp and pack.
cudaError_t collapse_level(const float* acc, const float* coarse, float* out, int w, int h, int cw, int ch, bool last,
                           uint16_t* rgb_out, cudaStream_t s);

// Halo control's coarse part: each frame's weight plane REDUCEd one level
// (pyramid.rs:86, planes [n][h][w] -> [n][h1][w1]); the weighted sums of the
// top Gaussian level (acc [3][h][w] = sum w*G, best = sum w, frames in order);
// and the weighted means acc /= best.
cudaError_t reduce_weights(const float* src, int w, int h, int n, float* dst, int w1, int h1, cudaStream_t s);
cudaError_t halo_top(const void* tops, int storage, const FrameXform* xf, const float* wts, int n, int w, int h, float* acc, float* best,
                     cudaStream_t s);
cudaError_t halo_divide(float* acc, const float* best, int w, int h, cudaStream_t s);

// fuse.rs:336 upsample_index of the depth level's winner map to w x h (f32 frame indices).
cudaError_t upsample_index(const uint16_t* win, int dwl, int dhl, int scale, int w, int h, float* out, cudaStream_t s);

// winner_shares (fuse.rs:315) on the device: counts[frames] of detail cells.
cudaError_t winner_counts(const uint16_t* win, const float* best, int cells, int frames, unsigned int* counts,
                          float* scratch_max, cudaStream_t s);

// brightness.rs:107 `means` of every frame on the stride-4 grid (unwarped u16).
cudaError_t frame_means(const uint16_t* frames, int n, int w, int h, double* partial, int nparts, double* means,
                        cudaStream_t s);

}  // namespace lsb
