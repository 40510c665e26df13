// Internal interfaces of the registration kernels (host side).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>
#include <vector>

namespace lsb {

constexpr int MAX_CAND = 9;
constexpr int NM_MAX_BLOCKS = 148 * 4;

// The inverse homographies of a batch of candidate transforms (row-major 3x3).
struct CostBatch {
    double inv[MAX_CAND][9];
};
struct WarpXform {
    double inv[9];
    int affine, interp;
};
struct BrightXform {
    double inv[9];
    int ident, affine;
};

// Search state: the stream, scratch for the cost partials and counters.
struct AlignCtx {
    cudaStream_t s;
    double* part;      // device, MAX_CAND * 296 * 3
    double* sums_dev;  // device, MAX_CAND * 3
    double* sums_host; // pinned, MAX_CAND * 3
    // the search on the device (one cooperative launch per frame)
    double* nm_part;   // device, 2 * MAX_CAND * NM_MAX_BLOCKS * 3
    int* nm_ctl;       // device, 4: error, evaluations, barrier arrivals, spare
    double* nm_out;    // device, 8: the transform
    int device_search = 1;  // 0: the host drives the search, one launch per simplex step
    int max_blocks = 0;     // CTAs of the device search at most (0: two per SM); the engine's grid limit
    size_t evals = 0, launches = 0;
};

cudaError_t luma_u16(const uint16_t* f, int w, int h, float* y, cudaStream_t s);
void gauss_dims(int w, int h, std::vector<std::pair<int, int>>& dims);
cudaError_t gauss_levels(const float* y, int w, int h, const std::vector<float*>& lv, cudaStream_t s);
cudaError_t warp_plane(const float* src, int w, int h, const WarpXform& xf, float* out, cudaStream_t s);
// prep.rs:46 `resize` / :63 `resize_plane` of the window (x0, y0, sw x sh) of `planes` planes (rows `stride`
// floats, planes `pstride` floats apart) onto ow x oh planar out; a copy of the window when the sizes agree.
cudaError_t resize_planes(const float* src, size_t stride, size_t pstride, int planes, int x0, int y0, int sw, int sh, int ow, int oh,
                          int interp, float* out, cudaStream_t s);
cudaError_t bright_sums(const uint16_t* frames, int n, int w, int h, const BrightXform* xf_dev, int interp, int nparts, double* part,
                        cudaStream_t s);
// The same for frame k alone (k >= 1) on `blocks` blocks: its partials land where bright_sums puts them.
cudaError_t bright_sums_frame(const uint16_t* frames, int k, int w, int h, const BrightXform* xf_dev, int interp, int nparts, double* part,
                              int blocks, cudaStream_t s);
void sim_matrix(const double* v, int w, int h, double m[9]);
void mat_inverse(const double m[9], double inv[9]);
bool sim_is_id(const double* v);
cudaError_t multiscale_align(AlignCtx& C, const float* rf, const std::vector<float*>& pr, const float* tg,
                             const std::vector<float*>& pt, int w, int h, const double init[8], const bool freem[8], int coarsen,
                             double out[8]);
// Chained searches, one frame after another with no host round trip: the
// search of frame i starts from the device-resident result of frame i-1,
// leaves its transform and full-resolution warp in device memory and adds its
// evaluation count on the device; the error word is sticky until the end.
cudaError_t align_chain_begin(AlignCtx& C, unsigned long long* evals_dev);
cudaError_t multiscale_align_chain(AlignCtx& C, const float* rf, const std::vector<float*>& pr, const float* tg,
                                   const std::vector<float*>& pt, int w, int h, const double* init_dev, const bool freem[8], int coarsen,
                                   double* out_dev, double* warp_dev, unsigned long long* evals_dev);
cudaError_t align_chain_end(AlignCtx& C, const unsigned long long* evals_dev, size_t* evals);
// warp_plane with the warp a chained search left on the device (inverse [9], affine, identity)
cudaError_t warp_plane_dev(const float* src, int w, int h, const double* warp_dev, int interp, float* out, cudaStream_t s);
cudaError_t cost_single(AlignCtx& C, const float* rf, int aw, int ah, const float* tg, int tw, int th, const double sim[8],
                        double* cost);

}  // namespace lsb
