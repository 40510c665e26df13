// Internal interfaces of the depth pass and the WLS solve (host side).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace lsb {

struct AggArgs {
    const void* slices;  // [n][dh][dw], f32 or f16
    int n, dw, dh, r;
    float eps;
    const float* guide;
    const float* mean_i;
    const float* var_i;
    float* state;  // [9][dh][dw] peak tracker state
    int tiles_x, ntiles;
    int async16;  // set by aggregate_peaks: slice rows start on 16-byte boundaries
};

cudaError_t luma_and_guide(const float* img, int w, int h, int k, float* yfull, float* guide, int dw, int dh, cudaStream_t s);
void gf_stats(const float* guide, int w, int h, int r, float* tmp, float* mean_i, float* var_i, cudaStream_t s);
void gf_coeffs(const float* guide, const float* mean_i, const float* var_i, const float* p, int w, int h, int r, float eps,
               float* t0, float* t1, float* t2, float* tmp, float* abar, float* bbar, cudaStream_t s);
size_t aggregate_smem_bytes(int r);
// running: moving window sums (radius 3 and 8) rather than the direct window sums of the general kernel
cudaError_t aggregate_peaks(AggArgs a, bool slice_fp16, cudaStream_t s, int grid_limit, bool running = true);
cudaError_t select_kth(const float* v, size_t cnt, int stride, size_t rank, unsigned* hist, unsigned* sel, float* out,
                       cudaStream_t s);
cudaError_t peak_finish(const float* state, size_t m, int n, const float* floor_p, float gate, float* depth, float* conf,
                        float* mins, cudaStream_t s);
cudaError_t median3(const float* src, float* out, int w, int h, cudaStream_t s);
cudaError_t conf_scale(float* conf, size_t m, const float* p90, cudaStream_t s);
cudaError_t robust_weights(const float* conf, const float* d, const float* u, float tau, float* w2, size_t m, cudaStream_t s);
// the weighted average (wav.rs:92): scratch planes on the depth grid, one frame's weight plane
struct WavScratch {
    float *s0, *s1, *t0, *t1, *t2, *tmp, *abar, *bbar;
};
void box_mean_plane(const float* src, float* tmp, float* out, int w, int h, int r, cudaStream_t s);
cudaError_t wav_weights(const void* slice, bool half, const float* floor, int dw, int dh, float gate, float power, int smooth, bool edge,
                        const float* guide, const float* mean_i, const float* var_i, float eps, WavScratch& t, float* out, cudaStream_t s);
cudaError_t upsample(const float* abar, const float* bbar, const float* yfull, const float* guide, const float* conf, int w,
                     int h, int dw, int dh, int k, float max_d, bool guided, float* depth, float* conf_full, cudaStream_t s);

// ----------------------------------------------------------------- WLS
// depth.rs:958 `WlsSolver` on the device. Planes are owned by the solver.
struct WlsLevel {
    int w, h;
    float *wd, *ax, *ay, *dinv, *x, *b, *r;
    // BF16 copies the mixed-precision V-cycle (vcycle_mode 1) works on
    uint16_t *hwd, *hax, *hay, *hdinv, *hx, *hb, *hr;
};
struct WlsSolver;
WlsSolver* wls_create(const float* guide, int w, int h, float lambda, float sigma_c, int edge_mode, cudaStream_t s,
                      cudaError_t* err);
// The planes of a w x h solver (allocated once, reused by every solve of that size) ...
WlsSolver* wls_alloc(int w, int h, cudaError_t* err);
// ... and the edge weights of one guide (depth.rs:653), down the hierarchy.
cudaError_t wls_prepare(WlsSolver* s, const float* guide, float lambda, float sigma_c, int edge_mode, cudaStream_t st);
int wls_width(const WlsSolver* s);
int wls_height(const WlsSolver* s);
void wls_destroy(WlsSolver* s);
// wd = max(conf, 0) + 1e-4, aggregated down the hierarchy, diagonals taken
cudaError_t wls_set_weights(WlsSolver* s, const float* conf, cudaStream_t st);
// Solve for d into u; returns (rel, iters) through the pointers. mode 0: the
// reference FP32 V-cycle; 1: BF16 smoother/restriction inside FP32 CG.
// x0_given: u holds a start (the FGS guess is skipped). coarse_corr: optional
// additive coarse-grid correction plane (null for none).
cudaError_t wls_solve(WlsSolver* s, const float* d, int max_iters, float* u, float* rel, int* iters, cudaStream_t st,
                      int mode, bool x0_given, double* rel64);
int wls_levels(const WlsSolver* s);

}  // namespace lsb
