// The confidence-weighted, edge-aware WLS depth solve (crates/lapstack-core/
// src/depth.rs:958 `WlsSolver`) on the device: the separable fast-global-
// smoother guess (depth.rs:677/707 Thomas sweeps, depth.rs:1022-1034
// schedule), then CG on (W + lambda L) u = W d preconditioned by one V-cycle
// of the 2x2-aggregation multigrid hierarchy (depth.rs:753-947), stopping at
// a relative residual of 1e-5. The f32 stencil, smoother, restriction and
// prolongation follow the reference's operation order; the CG dot products
// are f64 sums in a fixed two-stage order.
#include <cuda_bf16.h>

#include <algorithm>
#include <functional>
#include <type_traits>
#include <vector>

#include "lsb_common.cuh"
#include "lsb_depth.h"

namespace lsb {

constexpr float MG_OMEGA = 0.8f;
constexpr int MG_COARSE = 32, MG_MIN = 16;
// the BF16 V-cycle: levels, and Jacobi sweeps before and after the coarse correction
constexpr int MG_H_LEVELS = 6, MG_H_SWEEPS = 2;
constexpr int DOT_BLOCKS = 592;

struct WlsSolver {
    int w, h;
    float lambda;
    float *ex, *ey;
    std::vector<WlsLevel> lv;
    float *cp, *dp, *f, *r, *z, *p, *ap;
    double *part, *scal;  // scal: [rz, pap, rr, bnorm2, rz_new]
    float* alpha_beta;    // [alpha, beta]
    float* host_rel;      // pinned: [rel, stop]
    std::vector<void*> allocs;
    // the CG iteration as two CUDA graphs (A: A p, alpha, the updates, |r|; B: the preconditioner,
    // beta, the new direction), captured on the first solve for this u and V-cycle mode
    cudaGraphExec_t gA = nullptr, gB = nullptr;
    const float* g_u = nullptr;
    int g_mode = -1;
    long long kA = 0, kB = 0;
    float* alloc(size_t n, cudaError_t* e) {
        void* p = nullptr;
        cudaError_t r = cudaMalloc(&p, n * sizeof(float));
        if (r != cudaSuccess) *e = r;
        else allocs.push_back(p);
        return (float*)p;
    }
};

static int g1(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }
static dim3 g2(int w, int h) { return dim3((w + 31) / 32, (h + 7) / 8); }
static const dim3 B2(32, 8);

// depth.rs:653 `edge_weights`: e = exp(-|dI| / sigma) right and below (mode 0);
// mode 1, the Gaussian-of-gradient weight exp(-dI^2 / (2 sigma^2)).
__global__ void edge_kernel(const float* __restrict__ g, int w, int h, float inv, float inv2s2, int mode, float lambda,
                            float* ex, float* ey, float* ax, float* ay) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t k = (size_t)y * w + x;
    float vx = 0.f, vy = 0.f;
    if (x + 1 < w) {
        const float d = fabsf(__fsub_rn(g[k], g[k + 1]));
        vx = mode == 0 ? expf(__fmul_rn(d, inv)) : expf(-__fmul_rn(__fmul_rn(d, d), inv2s2));
    }
    if (y + 1 < h) {
        const float d = fabsf(__fsub_rn(g[k], g[k + w]));
        vy = mode == 0 ? expf(__fmul_rn(d, inv)) : expf(-__fmul_rn(__fmul_rn(d, d), inv2s2));
    }
    ex[k] = vx;
    ey[k] = vy;
    ax[k] = __fmul_rn(lambda, vx);
    ay[k] = __fmul_rn(lambda, vy);
}

// depth.rs:852 `coarsen` (edges) and :886 `coarsen_wd_into` (data weights)
__global__ void coarsen_edges_kernel(const float* __restrict__ ax, const float* __restrict__ ay, int w, int h, float* cax,
                                     float* cay, int cw, int ch) {
    const int xx = blockIdx.x * blockDim.x + threadIdx.x, yy = blockIdx.y * blockDim.y + threadIdx.y;
    if (xx >= cw || yy >= ch) return;
    float a = 0.f;
    if (xx + 1 < cw)
        for (int y = 2 * yy; y < min(2 * yy + 2, h); y++) a = __fadd_rn(a, ax[(size_t)y * w + 2 * xx + 1]);
    cax[(size_t)yy * cw + xx] = a;
    float b = 0.f;
    if (yy + 1 < ch) {
        const int y = 2 * yy + 1;
        for (int x = 2 * xx; x < min(2 * xx + 2, w); x++) b = __fadd_rn(b, ay[(size_t)y * w + x]);
    }
    cay[(size_t)yy * cw + xx] = b;
}
// b_c = P^T r (depth.rs:911 `restrict`), the same block sum as the data weights
__device__ __forceinline__ float block_sum_at(const float* __restrict__ src, int w, int h, int xx, int yy) {
    float o = 0.f;
    for (int y = 2 * yy; y < min(2 * yy + 2, h); y++) {
        float rs = 0.f;
        for (int x = 2 * xx; x < min(2 * xx + 2, w); x++) rs = __fadd_rn(rs, src[(size_t)y * w + x]);
        o = __fadd_rn(o, rs);
    }
    return o;
}
// depth.rs:911 `restrict` (and the 2x2 aggregation of depth.rs:852 `coarsen`): 2x2 block sums.
__global__ void block_sum_kernel(const float* __restrict__ src, int w, int h, float* __restrict__ dst, int cw, int ch) {
    const int xx = blockIdx.x * blockDim.x + threadIdx.x, yy = blockIdx.y * blockDim.y + threadIdx.y;
    if (xx >= cw || yy >= ch) return;
    dst[(size_t)yy * cw + xx] = block_sum_at(src, w, h, xx, yy);
}
// depth.rs:812 `set_dinv`
__global__ void dinv_kernel(const float* __restrict__ wd, const float* __restrict__ ax, const float* __restrict__ ay, int w, int h,
                            float* __restrict__ dinv) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t k = (size_t)y * w + x;
    float v = wd[k];
    if (x > 0) v = __fadd_rn(v, ax[k - 1]);
    if (x + 1 < w) v = __fadd_rn(v, ax[k]);
    if (y > 0) v = __fadd_rn(v, ay[k - w]);
    if (y + 1 < h) v = __fadd_rn(v, ay[k]);
    dinv[k] = __fdiv_rn(1.f, fmaxf(v, 1e-12f));
}
// depth.rs:786 `apply`: mode 0 out = A x; 1 out = b - A x; 2 out = x + w D^-1 (b - A x)
__device__ __forceinline__ float stencil_at(const float* __restrict__ x, const float* __restrict__ b, const float* __restrict__ wd,
                                            const float* __restrict__ ax, const float* __restrict__ ay, const float* __restrict__ dinv,
                                            int w, int h, int i, int y, int mode) {
    const size_t k = (size_t)y * w + i;
    const float xk = x[k];
    float v = __fmul_rn(wd[k], xk);
    if (i > 0) v = __fadd_rn(v, __fmul_rn(ax[k - 1], __fsub_rn(xk, x[k - 1])));
    if (i + 1 < w) v = __fadd_rn(v, __fmul_rn(ax[k], __fsub_rn(xk, x[k + 1])));
    if (y > 0) v = __fadd_rn(v, __fmul_rn(ay[k - w], __fsub_rn(xk, x[k - w])));
    if (y + 1 < h) v = __fadd_rn(v, __fmul_rn(ay[k], __fsub_rn(xk, x[k + w])));
    if (mode == 0) return v;
    if (mode == 1) return __fsub_rn(b[k], v);
    return __fadd_rn(xk, __fmul_rn(__fmul_rn(MG_OMEGA, dinv[k]), __fsub_rn(b[k], v)));
}
// depth.rs:786 `MgLevel::apply` (mode 0: A x; 1: b - A x) and :837 `jacobi` (mode 2).
__global__ void stencil_kernel(const float* __restrict__ x, const float* __restrict__ b, const float* __restrict__ wd,
                               const float* __restrict__ ax, const float* __restrict__ ay, const float* __restrict__ dinv,
                               float* __restrict__ out, int w, int h, int mode) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || y >= h) return;
    const size_t k = (size_t)y * w + i;
    const float xk = x[k];
    float v = __fmul_rn(wd[k], xk);
    if (i > 0) v = __fadd_rn(v, __fmul_rn(ax[k - 1], __fsub_rn(xk, x[k - 1])));
    if (i + 1 < w) v = __fadd_rn(v, __fmul_rn(ax[k], __fsub_rn(xk, x[k + 1])));
    if (y > 0) v = __fadd_rn(v, __fmul_rn(ay[k - w], __fsub_rn(xk, x[k - w])));
    if (y + 1 < h) v = __fadd_rn(v, __fmul_rn(ay[k], __fsub_rn(xk, x[k + w])));
    if (mode == 0) out[k] = v;
    else if (mode == 1) out[k] = __fsub_rn(b[k], v);
    else out[k] = __fadd_rn(xk, __fmul_rn(__fmul_rn(MG_OMEGA, dinv[k]), __fsub_rn(b[k], v)));
}
// depth.rs:840 zero-start Jacobi: x = w * D^-1 * b
__global__ void jac0_kernel(const float* __restrict__ b, const float* __restrict__ dinv, float* __restrict__ x, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        x[k] = __fmul_rn(__fmul_rn(MG_OMEGA, dinv[k]), b[k]);
}
// depth.rs:901 `prolong_add`
__global__ void prolong_kernel(float* __restrict__ x, int w, int h, const float* __restrict__ xc, int cw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || y >= h) return;
    const size_t k = (size_t)y * w + i;
    x[k] = __fadd_rn(x[k], xc[(size_t)(y / 2) * cw + i / 2]);
}

// One fine level's way down the V-cycle in one pass (depth.rs:924-930): the zero-start Jacobi sweep
// x = w D^-1 b (depth.rs:840), the residual b - A x (depth.rs:786) and its restriction to the coarse
// right-hand side (depth.rs:911), one thread per coarse cell and its 2x2 fine cells; the neighbours'
// x are recomputed from b and D^-1 by the same product, so every value is the separate kernels' own.
__device__ __forceinline__ float jac0_at(const float* __restrict__ b, const float* __restrict__ dinv, size_t k) {
    return __fmul_rn(__fmul_rn(MG_OMEGA, dinv[k]), b[k]);
}
// A 32 x 8 block of coarse cells covers 64 x 16 fine cells: their x and a one-cell ring are
// computed once into shared memory, and every fine cell's residual reads its neighbours there.
constexpr int VC_FW = 2 * 32 + 2, VC_FH = 2 * 8 + 2;
__global__ void __launch_bounds__(256) vc_down_kernel(const float* __restrict__ b, const float* __restrict__ wd, const float* __restrict__ ax,
                                                      const float* __restrict__ ay, const float* __restrict__ dinv, float* __restrict__ x,
                                                      int w, int h, float* __restrict__ cb, int cw, int ch) {
    __shared__ float J[VC_FH][VC_FW];
    const int fx0 = 2 * blockIdx.x * blockDim.x - 1, fy0 = 2 * blockIdx.y * blockDim.y - 1;
    for (int e = threadIdx.y * blockDim.x + threadIdx.x; e < VC_FW * VC_FH; e += blockDim.x * blockDim.y) {
        const int r = e / VC_FW, c = e - r * VC_FW, gx = fx0 + c, gy = fy0 + r;
        J[r][c] = gx >= 0 && gx < w && gy >= 0 && gy < h ? jac0_at(b, dinv, (size_t)gy * w + gx) : 0.f;
    }
    __syncthreads();
    const int xx = blockIdx.x * blockDim.x + threadIdx.x, yy = blockIdx.y * blockDim.y + threadIdx.y;
    if (xx >= cw || yy >= ch) return;
    float o = 0.f;
    for (int y = 2 * yy; y < min(2 * yy + 2, h); y++) {
        float rs = 0.f;
        const int jr = y - fy0;
        for (int i = 2 * xx; i < min(2 * xx + 2, w); i++) {
            const size_t k = (size_t)y * w + i;
            const int jc = i - fx0;
            const float xk = J[jr][jc];
            x[k] = xk;
            float v = __fmul_rn(wd[k], xk);
            if (i > 0) v = __fadd_rn(v, __fmul_rn(ax[k - 1], __fsub_rn(xk, J[jr][jc - 1])));
            if (i + 1 < w) v = __fadd_rn(v, __fmul_rn(ax[k], __fsub_rn(xk, J[jr][jc + 1])));
            if (y > 0) v = __fadd_rn(v, __fmul_rn(ay[k - w], __fsub_rn(xk, J[jr - 1][jc])));
            if (y + 1 < h) v = __fadd_rn(v, __fmul_rn(ay[k], __fsub_rn(xk, J[jr + 1][jc])));
            rs = __fadd_rn(rs, __fsub_rn(b[k], v));
        }
        o = __fadd_rn(o, rs);
    }
    cb[(size_t)yy * cw + xx] = o;
}
// ... and its way up in one pass (depth.rs:932-946): the prolongation x += P x_c (depth.rs:901) and the
// damped Jacobi sweep (depth.rs:837) on the corrected x, the neighbours' corrected x recomputed by the
// same addition; into out (another buffer than x).
__device__ __forceinline__ float prolonged_at(const float* __restrict__ x, const float* __restrict__ xc, int w, int cw, int i, int y) {
    return __fadd_rn(x[(size_t)y * w + i], xc[(size_t)(y >> 1) * cw + (i >> 1)]);
}
// The block's 32 x 8 corrected x and a one-cell ring are computed once into shared memory.
__global__ void __launch_bounds__(256) vc_up_kernel(const float* __restrict__ x, const float* __restrict__ xc, int cw,
                                                    const float* __restrict__ b, const float* __restrict__ wd,
                                                    const float* __restrict__ ax, const float* __restrict__ ay,
                                                    const float* __restrict__ dinv, float* __restrict__ out, int w, int h) {
    __shared__ float X[8 + 2][32 + 2];
    const int x0 = blockIdx.x * blockDim.x - 1, y0 = blockIdx.y * blockDim.y - 1;
    for (int e = threadIdx.y * blockDim.x + threadIdx.x; e < 10 * 34; e += blockDim.x * blockDim.y) {
        const int r = e / 34, c = e - r * 34, gx = x0 + c, gy = y0 + r;
        X[r][c] = gx >= 0 && gx < w && gy >= 0 && gy < h ? prolonged_at(x, xc, w, cw, gx, gy) : 0.f;
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || y >= h) return;
    const size_t k = (size_t)y * w + i;
    const int r = threadIdx.y + 1, c = threadIdx.x + 1;
    const float xk = X[r][c];
    float v = __fmul_rn(wd[k], xk);
    if (i > 0) v = __fadd_rn(v, __fmul_rn(ax[k - 1], __fsub_rn(xk, X[r][c - 1])));
    if (i + 1 < w) v = __fadd_rn(v, __fmul_rn(ax[k], __fsub_rn(xk, X[r][c + 1])));
    if (y > 0) v = __fadd_rn(v, __fmul_rn(ay[k - w], __fsub_rn(xk, X[r - 1][c])));
    if (y + 1 < h) v = __fadd_rn(v, __fmul_rn(ay[k], __fsub_rn(xk, X[r + 1][c])));
    out[k] = __fadd_rn(xk, __fmul_rn(__fmul_rn(MG_OMEGA, dinv[k]), __fsub_rn(b[k], v)));
}

// The coarse end of the V-cycle (depth.rs:924 `vcycle` from level 0 of `T`
// down) in ONE CTA: each level's zero-start Jacobi, residual, restriction,
// the coarsest level's MG_COARSE sweeps, then prolongation and the smoothing
// sweep back up; __syncthreads between steps. The per-element arithmetic is
// the separate kernels'. Each level's solution ends in its lv[].x (a sweep
// writes r, then copies back), as the host-driven levels above expect.
constexpr int MG_TAIL_CELLS = 8192, MG_TAIL_MAX = 16;
struct MgTail {
    WlsLevel lv[MG_TAIL_MAX];
    int n;
};
__device__ __forceinline__ void tail_sweep(const WlsLevel& L, bool zero) {
    const int n = L.w * L.h;
    if (zero) {
        for (int k = threadIdx.x; k < n; k += blockDim.x) L.x[k] = __fmul_rn(__fmul_rn(MG_OMEGA, L.dinv[k]), L.b[k]);
        __syncthreads();
        return;
    }
    for (int k = threadIdx.x; k < n; k += blockDim.x) L.r[k] = stencil_at(L.x, L.b, L.wd, L.ax, L.ay, L.dinv, L.w, L.h, k % L.w, k / L.w, 2);
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) L.x[k] = L.r[k];
    __syncthreads();
}
// depth.rs:924 `vcycle` from the first level small enough for one CTA down to the coarsest.
__global__ void __launch_bounds__(1024) vcycle_tail_kernel(const MgTail T) {
    for (int l = 0; l + 1 < T.n; l++) {
        const WlsLevel &L = T.lv[l], &C = T.lv[l + 1];
        tail_sweep(L, true);
        for (int k = threadIdx.x; k < L.w * L.h; k += blockDim.x)
            L.r[k] = stencil_at(L.x, L.b, L.wd, L.ax, L.ay, L.dinv, L.w, L.h, k % L.w, k / L.w, 1);
        __syncthreads();
        for (int k = threadIdx.x; k < C.w * C.h; k += blockDim.x) C.b[k] = block_sum_at(L.r, L.w, L.h, k % C.w, k / C.w);
        __syncthreads();
    }
    const WlsLevel& Z = T.lv[T.n - 1];
    for (int it = 0; it < MG_COARSE; it++) tail_sweep(Z, it == 0);
    for (int l = T.n - 2; l >= 0; l--) {
        const WlsLevel &L = T.lv[l], &C = T.lv[l + 1];
        for (int k = threadIdx.x; k < L.w * L.h; k += blockDim.x) {
            const int i = k % L.w, y = k / L.w;
            L.x[k] = __fadd_rn(L.x[k], C.x[(size_t)(y / 2) * C.w + i / 2]);
        }
        __syncthreads();
        tail_sweep(L, false);
    }
}
// depth.rs:994 wd = max(conf, 0) + 1e-4
__global__ void wd_kernel(const float* __restrict__ conf, float* __restrict__ wd, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        wd[k] = __fadd_rn(fmaxf(conf[k], 0.f), 1e-4f);
}

// depth.rs:677 `solve_rows` / :707 `solve_cols`: the Thomas algorithm along
// every line, one thread per line, 32 lines per warp. The warp stages 32x32
// tiles of the coefficients through shared memory with coalesced row-segment
// loads (ROWS: a line is an image row, the tile is [line][element]; else a
// line is a column, the tile is [element][line]); each thread then walks its
// line's 32 elements of the tile in the reference's order and arithmetic.
constexpr int TT = 32;
template <bool ROWS>
__device__ __forceinline__ float& tl(float (*t)[TT + 1], int line, int e) {
    return ROWS ? t[line][e] : t[e][line];
}
__device__ __forceinline__ void cp_async4f(float* smem, const float* gmem) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// The 32 lines' elements e0 .. e0+31 of `src` into tile t (cp.async; `fill` where out of range).
template <bool ROWS>
__device__ __forceinline__ void tile_load(float (*t)[TT + 1], const float* __restrict__ src, int l0, int e0, int nlines, int len, int w,
                                          float fill) {
    const int lane = threadIdx.x;
    for (int q = 0; q < TT; q++) {
        const int ln = ROWS ? q : lane, e = ROWS ? e0 + lane : e0 + q;
        float* d = &tl<ROWS>(t, ln, e - e0);
        if (l0 + ln < nlines && e < len) cp_async4f(d, src + (ROWS ? (size_t)(l0 + ln) * w + e : (size_t)e * w + (l0 + ln)));
        else *d = fill;
    }
}
template <bool ROWS>
__device__ __forceinline__ void tile_store(float (*t)[TT + 1], float* __restrict__ dst, int l0, int e0, int nlines, int len, int w) {
    const int lane = threadIdx.x;
    for (int q = 0; q < TT; q++) {
        const int ln = ROWS ? q : lane, e = ROWS ? e0 + lane : e0 + q;
        if (l0 + ln < nlines && e < len) dst[ROWS ? (size_t)(l0 + ln) * w + e : (size_t)e * w + (l0 + ln)] = tl<ROWS>(t, ln, e - e0);
    }
}

// depth.rs:677 `solve_rows` / :707 `solve_cols`: the Thomas algorithm along
// every line, one thread per line, 32 lines per warp (ROWS: a line is an image
// row, the tile is [line][element]; else a line is a column, the tile is
// [element][line]). The coefficient tiles of the next 32 elements stream into
// shared memory (cp.async, two buffers) while the current 32 are eliminated,
// and the back substitution streams cp / dp the same way; each thread walks
// its line in the reference's order and arithmetic.
template <bool ROWS>
__global__ void __launch_bounds__(32) thomas_kernel(float* __restrict__ u, const float* __restrict__ f, const float* __restrict__ wd,
                                                    int unit_wd, const float* __restrict__ a, int w, int h, float lam,
                                                    float* __restrict__ cp, float* __restrict__ dp) {
    __shared__ float ta[2][TT][TT + 1], tw[2][TT][TT + 1], tf[2][TT][TT + 1], tc[2][TT][TT + 1], td[2][TT][TT + 1];
    const int lane = threadIdx.x;
    const int nlines = ROWS ? h : w, len = ROWS ? w : h;
    const int l0 = blockIdx.x * TT;
    const int li = l0 + lane;
    const int nch = (len + TT - 1) / TT;
    auto issue_fwd = [&](int c) {
        const int b = c & 1, e0 = c * TT;
        tile_load<ROWS>(ta[b], a, l0, e0, nlines, len, w, 0.f);
        tile_load<ROWS>(tf[b], f, l0, e0, nlines, len, w, 0.f);
        if (!unit_wd) tile_load<ROWS>(tw[b], wd, l0, e0, nlines, len, w, 1.f);
        cp_commit();
    };
    float prev_a = 0.f, cprev = 0.f, dprev = 0.f;
    const float nl = -lam;
    issue_fwd(0);
    for (int c = 0; c < nch; c++) {
        const int b = c & 1, e0 = c * TT, ne = min(TT, len - e0);
        if (c + 1 < nch) {
            issue_fwd(c + 1);
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        __syncwarp();
        if (li < nlines)
            for (int j = 0; j < ne; j++) {
                const int i = e0 + j;
                const float ai = i + 1 < len ? tl<ROWS>(ta[b], lane, j) : 0.f;
                const float wdi = unit_wd ? 1.f : tl<ROWS>(tw[b], lane, j);
                const float diag = __fadd_rn(wdi, __fmul_rn(lam, __fadd_rn(prev_a, ai)));
                const float lower = __fmul_rn(nl, prev_a), upper = __fmul_rn(nl, ai);
                float m = __fsub_rn(diag, __fmul_rn(lower, i > 0 ? cprev : 0.f));
                if (fabsf(m) < 1e-12f) m = 1e-12f;
                cprev = __fdiv_rn(upper, m);
                dprev = __fdiv_rn(__fsub_rn(__fmul_rn(wdi, tl<ROWS>(tf[b], lane, j)), __fmul_rn(lower, i > 0 ? dprev : 0.f)), m);
                tl<ROWS>(tc[b], lane, j) = cprev;
                tl<ROWS>(td[b], lane, j) = dprev;
                prev_a = ai;
            }
        __syncwarp();
        if (c + 1 < nch) {  // the last chunk stays in shared memory for the back substitution
            tile_store<ROWS>(tc[b], cp, l0, e0, nlines, len, w);
            tile_store<ROWS>(td[b], dp, l0, e0, nlines, len, w);
        }
        __syncwarp();
    }
    __threadfence_block();
    __syncwarp();
    // back substitution, chunks from the end; chunk c-1's cp / dp stream in while chunk c runs
    const int last = nch - 1;
    auto issue_bwd = [&](int c) {
        const int b = c & 1, e0 = c * TT;
        tile_load<ROWS>(tc[b], cp, l0, e0, nlines, len, w, 0.f);
        tile_load<ROWS>(td[b], dp, l0, e0, nlines, len, w, 0.f);
        cp_commit();
    };
    float nxt = 0.f;
    for (int c = last; c >= 0; c--) {
        const int b = c & 1, e0 = c * TT, ne = min(TT, len - e0);
        if (c - 1 >= 0) {
            issue_bwd(c - 1);
            if (c != last) cp_wait<1>();
        } else if (c != last) {
            cp_wait<0>();
        }
        __syncwarp();
        if (li < nlines)
            for (int j = ne - 1; j >= 0; j--) {
                const int i = e0 + j;
                nxt = i == len - 1 ? tl<ROWS>(td[b], lane, j) : __fsub_rn(tl<ROWS>(td[b], lane, j), __fmul_rn(tl<ROWS>(tc[b], lane, j), nxt));
                tl<ROWS>(tf[b], lane, j) = nxt;
            }
        __syncwarp();
        tile_store<ROWS>(tf[b], u, l0, e0, nlines, len, w);
        __syncwarp();
    }
    cp_wait<0>();
}
// The same systems (depth.rs:677 / :707), each line cut into P segments
// (the partition method); a warp per segment holds 32 lines (lane = line).
// (1) Each segment eliminates forward (pivots d', the spike g on the unknown
// before the segment, the right-hand side r') and backward, leaving each of
// its unknowns as rho + sigma * X_{s-1} + tau * X_s, X_s being the segment's
// last unknown. (2) One thread per line solves the P-unknown tridiagonal
// system that the segments' last equations make of the X_s. (3) Each segment
// recovers its unknowns. A line's sequential chain shrinks P-fold and P times
// as many threads run the lines; the result differs from the one-thread
// Thomas sweep by rounding only (the systems are diagonally dominant), and
// these sweeps only start the MG-PCG solve.
template <bool ROWS, int P>
__global__ void __launch_bounds__(32 * P) pthomas_kernel(float* __restrict__ u, const float* __restrict__ f, const float* __restrict__ wd,
                                                         int unit_wd, const float* __restrict__ a, int w, int h, float lam,
                                                         float* __restrict__ s0, float* __restrict__ s1, float* __restrict__ s2) {
    __shared__ float cf[P][7][32];  // per segment and line: the first unknown's (rho, sigma, tau); the last equation's d', g, r', u
    __shared__ float X[P][32];      // the segments' last unknowns
    __shared__ float rc[P][32], rr[P][32];
    const int lane = threadIdx.x & 31, seg = threadIdx.x >> 5;
    const int nlines = ROWS ? h : w, len = ROWS ? w : h;
    const int line = blockIdx.x * 32 + lane;
    const bool live = line < nlines;
    const int b = (int)((long long)seg * len / P), e = (int)((long long)(seg + 1) * len / P);  // len >= P: never empty
    auto at = [&](int i) -> size_t { return ROWS ? (size_t)line * w + i : (size_t)i * w + line; };
    const float nl = -lam;
    if (live) {
        float a_prev = b > 0 ? a[at(b - 1)] : 0.f;
        float dprev = 1.f, gprev = 0.f, rprev = 0.f, uprev = 0.f;
        for (int i = b; i < e; i++) {
            const size_t k = at(i);
            const float ai = i + 1 < len ? a[k] : 0.f;
            const float wdi = unit_wd ? 1.f : wd[k];
            const float diag = wdi + lam * (a_prev + ai);
            const float lower = nl * a_prev, upper = nl * ai;
            const float ri = wdi * f[k];
            float dd = diag, gg = lower, rv = ri;
            if (i > b) {
                const float mlt = lower / dprev;
                dd = diag - mlt * uprev;
                gg = -(mlt * gprev);
                rv = ri - mlt * rprev;
            }
            if (fabsf(dd) < 1e-12f) dd = 1e-12f;
            s0[k] = dd;
            s1[k] = gg;
            s2[k] = rv;
            dprev = dd;
            gprev = gg;
            rprev = rv;
            uprev = upper;
            a_prev = ai;
        }
        cf[seg][3][lane] = dprev;
        cf[seg][4][lane] = gprev;
        cf[seg][5][lane] = rprev;
        cf[seg][6][lane] = uprev;
        float rn = 0.f, sn = 0.f, tn = 1.f;  // the last unknown is X_s itself
        {
            const size_t k = at(e - 1);
            s0[k] = 0.f;
            s1[k] = 0.f;
            s2[k] = 1.f;
        }
        for (int i = e - 2; i >= b; i--) {
            const size_t k = at(i);
            const float upper = nl * a[k];  // i + 1 < len here
            const float inv = 1.f / s0[k];
            const float rho = (s2[k] - upper * rn) * inv, sig = (-s1[k] - upper * sn) * inv, tau = -(upper * tn) * inv;
            s0[k] = rho;
            s1[k] = sig;
            s2[k] = tau;
            rn = rho;
            sn = sig;
            tn = tau;
        }
        cf[seg][0][lane] = rn;
        cf[seg][1][lane] = sn;
        cf[seg][2][lane] = tn;
    }
    __syncthreads();
    if (seg == 0 && live) {
        // segment q's last equation: g X_{q-1} + d' X_q + u x_first(q+1) = r', x_first(q+1) = rho + sigma X_q + tau X_{q+1}
        float cprev = 0.f, rprev2 = 0.f;
        for (int q = 0; q < P; q++) {
            const bool nx = q + 1 < P;
            const float uq = cf[q][6][lane];
            const float A = q > 0 ? cf[q][4][lane] : 0.f;
            const float B = nx ? cf[q][3][lane] + uq * cf[q + 1][1][lane] : cf[q][3][lane];
            const float C = nx ? uq * cf[q + 1][2][lane] : 0.f;
            const float R = nx ? cf[q][5][lane] - uq * cf[q + 1][0][lane] : cf[q][5][lane];
            float den = B - A * cprev;
            if (fabsf(den) < 1e-12f) den = 1e-12f;
            cprev = C / den;
            rprev2 = (R - A * rprev2) / den;
            rc[q][lane] = cprev;
            rr[q][lane] = rprev2;
        }
        float xn = 0.f;
        for (int q = P - 1; q >= 0; q--) {
            xn = q == P - 1 ? rr[q][lane] : rr[q][lane] - rc[q][lane] * xn;
            X[q][lane] = xn;
        }
    }
    __syncthreads();
    if (live) {
        const float xl = seg > 0 ? X[seg - 1][lane] : 0.f, xs = X[seg][lane];
        for (int i = b; i < e; i++) {
            const size_t k = at(i);
            u[k] = s0[k] + s1[k] * xl + s2[k] * xs;
        }
    }
}
constexpr int PT_ROWS = 8, PT_COLS = 16;

// depth.rs:677 `solve_rows`: the row sweep with one row per warp held in shared memory (the partition
// method of pthomas_kernel with 32 segments, lane = segment): a row's
// coefficients are read once, coalesced, and every step of the segments'
// sweeps hits shared memory (segments start w/32 floats apart: no bank
// conflicts when that is odd, at most two-way otherwise). The reduced system
// is solved by lane 0 from the segments' end coefficients gathered with
// shuffles.
constexpr int PTR_SEGS = 32;
__global__ void __launch_bounds__(32) pthomas_rows_kernel(float* __restrict__ u, const float* __restrict__ f, const float* __restrict__ wd,
                                                          int unit_wd, const float* __restrict__ a, int w, int h, float lam) {
    extern __shared__ float sm[];
    __shared__ float X[PTR_SEGS];
    const int line = blockIdx.x, lane = threadIdx.x;
    if (line >= h) return;
    float* A = sm;
    float* WD = A + w;
    float* F = WD + w;
    float* S0 = F + w;
    float* S1 = S0 + w;
    float* S2 = S1 + w;
    const size_t row = (size_t)line * w;
    for (int i = lane; i < w; i += 32) {
        A[i] = a[row + i];
        F[i] = f[row + i];
        WD[i] = unit_wd ? 1.f : wd[row + i];
    }
    __syncwarp();
    const int len = w, b = (int)((long long)lane * len / PTR_SEGS), e = (int)((long long)(lane + 1) * len / PTR_SEGS);
    const float nl = -lam;
    float a_prev = b > 0 ? A[b - 1] : 0.f;
    float dprev = 1.f, gprev = 0.f, rprev = 0.f, uprev = 0.f;
    for (int i = b; i < e; i++) {
        const float ai = i + 1 < len ? A[i] : 0.f;
        const float wdi = WD[i];
        const float diag = wdi + lam * (a_prev + ai);
        const float lower = nl * a_prev, upper = nl * ai;
        const float ri = wdi * F[i];
        float dd = diag, gg = lower, rv = ri;
        if (i > b) {
            const float mlt = lower / dprev;
            dd = diag - mlt * uprev;
            gg = -(mlt * gprev);
            rv = ri - mlt * rprev;
        }
        if (fabsf(dd) < 1e-12f) dd = 1e-12f;
        S0[i] = dd;
        S1[i] = gg;
        S2[i] = rv;
        dprev = dd;
        gprev = gg;
        rprev = rv;
        uprev = upper;
        a_prev = ai;
    }
    const float dL = dprev, gL = gprev, rL = rprev, uL = uprev;  // the segment's last equation
    float rn = 0.f, sn = 0.f, tn = 1.f;
    S0[e - 1] = 0.f;
    S1[e - 1] = 0.f;
    S2[e - 1] = 1.f;
    for (int i = e - 2; i >= b; i--) {
        const float upper = nl * A[i];
        const float inv = 1.f / S0[i];
        const float rho = (S2[i] - upper * rn) * inv, sig = (-S1[i] - upper * sn) * inv, tau = -(upper * tn) * inv;
        S0[i] = rho;
        S1[i] = sig;
        S2[i] = tau;
        rn = rho;
        sn = sig;
        tn = tau;
    }
    // the reduced system on lane 0, the coefficients of segment q (and q + 1) by shuffle
    float cprev = 0.f, rprev2 = 0.f;
    float rc[PTR_SEGS], rr[PTR_SEGS];
#pragma unroll
    for (int q = 0; q < PTR_SEGS; q++) {
        const float dq = __shfl_sync(0xffffffffu, dL, q), gq = __shfl_sync(0xffffffffu, gL, q);
        const float rq = __shfl_sync(0xffffffffu, rL, q), uq = __shfl_sync(0xffffffffu, uL, q);
        const int nq = q + 1 < PTR_SEGS ? q + 1 : q;
        const float rF = __shfl_sync(0xffffffffu, rn, nq), sF = __shfl_sync(0xffffffffu, sn, nq), tF = __shfl_sync(0xffffffffu, tn, nq);
        const bool nx = q + 1 < PTR_SEGS;
        const float Aq = q > 0 ? gq : 0.f;
        const float Bq = nx ? dq + uq * sF : dq;
        const float Cq = nx ? uq * tF : 0.f;
        const float Rq = nx ? rq - uq * rF : rq;
        float den = Bq - Aq * cprev;
        if (fabsf(den) < 1e-12f) den = 1e-12f;
        cprev = Cq / den;
        rprev2 = (Rq - Aq * rprev2) / den;
        rc[q] = cprev;
        rr[q] = rprev2;
    }
    if (lane == 0) {
        float xn = 0.f;
#pragma unroll
        for (int q = PTR_SEGS - 1; q >= 0; q--) {
            xn = q == PTR_SEGS - 1 ? rr[q] : rr[q] - rc[q] * xn;
            X[q] = xn;
        }
    }
    __syncwarp();
    const float xl = lane > 0 ? X[lane - 1] : 0.f, xs = X[lane];
    for (int i = b; i < e; i++) S0[i] = S0[i] + S1[i] * xl + S2[i] * xs;
    __syncwarp();
    for (int i = lane; i < w; i += 32) u[row + i] = S0[i];
}

static void thomas(bool rows, float* u, const float* f, const float* wd, int unit_wd, const float* a, int w, int h, float lam,
                   float* cp, float* dp, float* sc, cudaStream_t s) {
    const int nlines = rows ? h : w, len = rows ? w : h;
    if (rows && len >= PTR_SEGS * 8 && (size_t)6 * len * sizeof(float) <= 200 * 1024) {
        const size_t smem = (size_t)6 * len * sizeof(float);
        cudaFuncSetAttribute(pthomas_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        lsb_launched(), pthomas_rows_kernel<<<nlines, 32, smem, s>>>(u, f, wd, unit_wd, a, w, h, lam);
        return;
    }
    if (sc && len >= (rows ? PT_ROWS : PT_COLS) * 8) {
        const int g = (nlines + 31) / 32;
        if (rows) lsb_launched(), pthomas_kernel<true, PT_ROWS><<<g, 32 * PT_ROWS, 0, s>>>(u, f, wd, unit_wd, a, w, h, lam, cp, dp, sc);
        else lsb_launched(), pthomas_kernel<false, PT_COLS><<<g, 32 * PT_COLS, 0, s>>>(u, f, wd, unit_wd, a, w, h, lam, cp, dp, sc);
        return;
    }
    if (rows) lsb_launched(), thomas_kernel<true><<<(nlines + TT - 1) / TT, TT, 0, s>>>(u, f, wd, unit_wd, a, w, h, lam, cp, dp);
    else lsb_launched(), thomas_kernel<false><<<(nlines + TT - 1) / TT, TT, 0, s>>>(u, f, wd, unit_wd, a, w, h, lam, cp, dp);
}

// ------------------------------------------------ the BF16 V-cycle (mode 1)
// The preconditioner's smoother, residual, restriction and prolongation on
// BF16 copies of the level operators and vectors, arithmetic in FP32; the
// outer CG stays FP32 with FP64 dot products. No reference counterpart: the
// reference's V-cycle is FP32 (vcycle_mode 0 here).
typedef __nv_bfloat16 bf;
__device__ __forceinline__ float ldh(const uint16_t* p, size_t k) { return __bfloat162float(((const bf*)p)[k]); }
__device__ __forceinline__ void sth(uint16_t* p, size_t k, float v) { ((bf*)p)[k] = __float2bfloat16_rn(v); }

__global__ void to_bf16_kernel(const float* __restrict__ a, uint16_t* __restrict__ o, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) sth(o, i, a[i]);
}
__global__ void from_bf16_kernel(const uint16_t* __restrict__ a, float* __restrict__ o, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) o[i] = ldh(a, i);
}
// A level's right-hand side and a sweep's output are BF16 (uint16_t) below level 0; at level 0 the
// right-hand side is the CG's FP32 residual and the last sweep writes the FP32 z.
__device__ __forceinline__ float ldv(const uint16_t* p, size_t k) { return ldh(p, k); }
__device__ __forceinline__ float ldv(const float* p, size_t k) { return p[k]; }
__device__ __forceinline__ void stv(uint16_t* p, size_t k, float v) { sth(p, k, v); }
__device__ __forceinline__ void stv(float* p, size_t k, float v) { p[k] = v; }
__device__ __forceinline__ float stencil_h_at(const uint16_t* __restrict__ x, float bk, const uint16_t* __restrict__ wd,
                                              const uint16_t* __restrict__ ax, const uint16_t* __restrict__ ay,
                                              const uint16_t* __restrict__ dinv, int w, int h, int i, int y, int mode) {
    const size_t k = (size_t)y * w + i;
    const float xk = ldh(x, k);
    float v = ldh(wd, k) * xk;
    if (i > 0) v += ldh(ax, k - 1) * (xk - ldh(x, k - 1));
    if (i + 1 < w) v += ldh(ax, k) * (xk - ldh(x, k + 1));
    if (y > 0) v += ldh(ay, k - w) * (xk - ldh(x, k - w));
    if (y + 1 < h) v += ldh(ay, k) * (xk - ldh(x, k + w));
    const float r = bk - v;
    return mode == 1 ? r : xk + MG_OMEGA * ldh(dinv, k) * r;
}
// mode 1: out = b - A x; mode 2: out = x + w D^-1 (b - A x)
template <class BT, class OT>
__global__ void stencil_h_kernel(const uint16_t* __restrict__ x, const BT* __restrict__ b, const uint16_t* __restrict__ wd,
                                 const uint16_t* __restrict__ ax, const uint16_t* __restrict__ ay, const uint16_t* __restrict__ dinv,
                                 OT* __restrict__ out, int w, int h, int mode) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || y >= h) return;
    const size_t k = (size_t)y * w + i;
    stv(out, k, stencil_h_at(x, ldv(b, k), wd, ax, ay, dinv, w, h, i, y, mode));
}
template <class BT>
__global__ void jac0_h_kernel(const BT* __restrict__ b, const uint16_t* __restrict__ dinv, uint16_t* __restrict__ x, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        sth(x, k, MG_OMEGA * ldh(dinv, k) * ldv(b, k));
}
// A fine level's way down and way up in one pass each, on tiles in shared memory: the same values
// as the separate kernels (every sweep's output rounded to BF16 where they store it), the
// neighbours' values computed once per block over a ring around the tile.
__device__ __forceinline__ float rbf(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }
// stencil_h_at with x read from a shared tile: (r, c) the cell's place in the tile
template <int PITCH>
__device__ __forceinline__ float sweep_tile(const float* X, int r, int c, float bk, const uint16_t* __restrict__ wd,
                                            const uint16_t* __restrict__ ax, const uint16_t* __restrict__ ay,
                                            const uint16_t* __restrict__ dinv, int w, int h, int i, int y, int mode) {
    const size_t k = (size_t)y * w + i;
    const float xk = X[r * PITCH + c];
    float v = ldh(wd, k) * xk;
    if (i > 0) v += ldh(ax, k - 1) * (xk - X[r * PITCH + c - 1]);
    if (i + 1 < w) v += ldh(ax, k) * (xk - X[r * PITCH + c + 1]);
    if (y > 0) v += ldh(ay, k - w) * (xk - X[(r - 1) * PITCH + c]);
    if (y + 1 < h) v += ldh(ay, k) * (xk - X[(r + 1) * PITCH + c]);
    const float rr = bk - v;
    return mode == 1 ? rr : xk + MG_OMEGA * ldh(dinv, k) * rr;
}
// Down: x0 = w D^-1 b, x1 = one sweep, r = b - A x1, its 2x2 block sums; x1 -> x, the sums -> cb.
// A 32 x 8 block of coarse cells: x0 over its 64 x 16 fine cells and a 2-cell ring, x1 with a 1-cell ring.
constexpr int VH_D0W = 64 + 4, VH_D0H = 16 + 4, VH_D1W = 64 + 2, VH_D1H = 16 + 2;
template <class BT>
__global__ void __launch_bounds__(256) vc_down_h_kernel(const BT* __restrict__ b, const uint16_t* __restrict__ wd,
                                                        const uint16_t* __restrict__ ax, const uint16_t* __restrict__ ay,
                                                        const uint16_t* __restrict__ dinv, uint16_t* __restrict__ x, int w, int h,
                                                        uint16_t* __restrict__ cb, int cw, int ch) {
    __shared__ float X0[VH_D0H * VH_D0W], X1[VH_D1H * VH_D1W];
    const int tid = threadIdx.y * 32 + threadIdx.x, fx = 64 * blockIdx.x, fy = 16 * blockIdx.y;
    for (int e = tid; e < VH_D0W * VH_D0H; e += 256) {
        const int r = e / VH_D0W, c = e - r * VH_D0W, gx = fx - 2 + c, gy = fy - 2 + r;
        X0[e] = gx >= 0 && gx < w && gy >= 0 && gy < h ? rbf(MG_OMEGA * ldh(dinv, (size_t)gy * w + gx) * ldv(b, (size_t)gy * w + gx)) : 0.f;
    }
    __syncthreads();
    for (int e = tid; e < VH_D1W * VH_D1H; e += 256) {
        const int r = e / VH_D1W, c = e - r * VH_D1W, gx = fx - 1 + c, gy = fy - 1 + r;
        X1[e] = gx >= 0 && gx < w && gy >= 0 && gy < h
                    ? rbf(sweep_tile<VH_D0W>(X0, r + 1, c + 1, ldv(b, (size_t)gy * w + gx), wd, ax, ay, dinv, w, h, gx, gy, 2))
                    : 0.f;
    }
    __syncthreads();
    const int xx = blockIdx.x * 32 + threadIdx.x, yy = blockIdx.y * 8 + threadIdx.y;
    if (xx >= cw || yy >= ch) return;
    float o = 0.f;
    for (int y = 2 * yy; y < min(2 * yy + 2, h); y++)
        for (int i = 2 * xx; i < min(2 * xx + 2, w); i++) {
            const size_t k = (size_t)y * w + i;
            const int r = y - fy + 1, c = i - fx + 1;
            sth(x, k, X1[r * VH_D1W + c]);
            o += rbf(sweep_tile<VH_D1W>(X1, r, c, ldv(b, k), wd, ax, ay, dinv, w, h, i, y, 1));
        }
    sth(cb, (size_t)yy * cw + xx, o);
}
// Up: x2 = x1 + P x_c, then two sweeps; the result -> out (BF16, or level 0's FP32 z).
// A 32 x 8 block of fine cells: x2 with a 2-cell ring, the first sweep with a 1-cell ring.
constexpr int VH_U2W = 32 + 4, VH_U2H = 8 + 4, VH_U3W = 32 + 2, VH_U3H = 8 + 2;
template <class BT, class OT>
__global__ void __launch_bounds__(256) vc_up_h_kernel(const uint16_t* __restrict__ x, const uint16_t* __restrict__ xc, int cw,
                                                      const BT* __restrict__ b, const uint16_t* __restrict__ wd,
                                                      const uint16_t* __restrict__ ax, const uint16_t* __restrict__ ay,
                                                      const uint16_t* __restrict__ dinv, OT* __restrict__ out, int w, int h) {
    __shared__ float X2[VH_U2H * VH_U2W], X3[VH_U3H * VH_U3W];
    const int tid = threadIdx.y * 32 + threadIdx.x, fx = 32 * blockIdx.x, fy = 8 * blockIdx.y;
    for (int e = tid; e < VH_U2W * VH_U2H; e += 256) {
        const int r = e / VH_U2W, c = e - r * VH_U2W, gx = fx - 2 + c, gy = fy - 2 + r;
        X2[e] = gx >= 0 && gx < w && gy >= 0 && gy < h ? rbf(ldh(x, (size_t)gy * w + gx) + ldh(xc, (size_t)(gy / 2) * cw + gx / 2)) : 0.f;
    }
    __syncthreads();
    for (int e = tid; e < VH_U3W * VH_U3H; e += 256) {
        const int r = e / VH_U3W, c = e - r * VH_U3W, gx = fx - 1 + c, gy = fy - 1 + r;
        X3[e] = gx >= 0 && gx < w && gy >= 0 && gy < h
                    ? rbf(sweep_tile<VH_U2W>(X2, r + 1, c + 1, ldv(b, (size_t)gy * w + gx), wd, ax, ay, dinv, w, h, gx, gy, 2))
                    : 0.f;
    }
    __syncthreads();
    const int i = fx + threadIdx.x, y = fy + threadIdx.y;
    if (i >= w || y >= h) return;
    const size_t k = (size_t)y * w + i;
    stv(out, k, sweep_tile<VH_U3W>(X3, threadIdx.y + 1, threadIdx.x + 1, ldv(b, k), wd, ax, ay, dinv, w, h, i, y, 2));
}

// The coarsest level's sweeps in one CTA of 32 x 32 threads with the level's planes in shared memory:
// the zero-start sweep, then sweeps - 1 damped Jacobi sweeps between two buffers, __syncthreads
// between them; the result is written to x.
constexpr int COARSE_H_PLANES = 7;
__global__ void __launch_bounds__(1024) coarse_h_kernel(uint16_t* __restrict__ x, const uint16_t* __restrict__ b,
                                                        const uint16_t* __restrict__ wd, const uint16_t* __restrict__ ax,
                                                        const uint16_t* __restrict__ ay, const uint16_t* __restrict__ dinv, int w,
                                                        int h, int sweeps) {
    extern __shared__ uint16_t csm[];
    const int n = w * h, tid = threadIdx.y * 32 + threadIdx.x;
    uint16_t *sb = csm, *swd = sb + n, *sax = swd + n, *say = sax + n, *sdi = say + n, *s0 = sdi + n, *s1 = s0 + n;
    for (int k = tid; k < n; k += 1024) {
        sb[k] = b[k];
        swd[k] = wd[k];
        sax[k] = ax[k];
        say[k] = ay[k];
        sdi[k] = dinv[k];
    }
    __syncthreads();
    for (int k = tid; k < n; k += 1024) sth(s0, k, MG_OMEGA * ldh(sdi, k) * ldh(sb, k));
    uint16_t *src = s0, *dst = s1;
    for (int sw = 1; sw < sweeps; sw++) {
        __syncthreads();
        for (int y = threadIdx.y; y < h; y += 32)
            for (int i = threadIdx.x; i < w; i += 32) {
                const size_t k = (size_t)y * w + i;
                sth(dst, k, stencil_h_at(src, ldh(sb, k), swd, sax, say, sdi, w, h, i, y, 2));
            }
        uint16_t* t = src;
        src = dst;
        dst = t;
    }
    __syncthreads();
    for (int k = tid; k < n; k += 1024) x[k] = src[k];
}
// depth.rs:1037 `dot`, f64 products: per-block partials, then the partials in order.
// Each thread's products (exact in f64) summed in a fixed order: 16-byte loads of four elements
// at a time when both planes allow them (more bytes in flight), the elements past the last four
// by the first threads.
__global__ void dot_partial_kernel(const float* __restrict__ a, const float* __restrict__ b, size_t n, double* part) {
    double s = 0.0;
    const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x, nt = (size_t)gridDim.x * blockDim.x;
    const bool vec = ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15) == 0;
    const size_t n4 = vec ? n / 4 : 0;
    const float4* a4 = reinterpret_cast<const float4*>(a);
    const float4* b4 = reinterpret_cast<const float4*>(b);
    for (size_t i = t0; i < n4; i += nt) {
        const float4 x = __ldg(a4 + i), y = __ldg(b4 + i);
        s += (double)x.x * (double)y.x;
        s += (double)x.y * (double)y.y;
        s += (double)x.z * (double)y.z;
        s += (double)x.w * (double)y.w;
    }
    for (size_t i = 4 * n4 + t0; i < n; i += nt) s += (double)a[i] * (double)b[i];
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}
// depth.rs:1039-1072, the CG scalars. mode: 0 rz; 1 pap -> alpha; 2 rz_new -> beta; 3 rr -> rel; 4 bb -> bnorm
__global__ void dot_final_kernel(const double* part, int nparts, double* scal, float* ab, float* host_rel, int mode) {
    // the partials summed by 256 threads (each a fixed stride of them), then a fixed tree
    __shared__ double red[256];
    double t = 0.0;
    for (int i = threadIdx.x; i < nparts; i += 256) t += part[i];
    red[threadIdx.x] = t;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    const double s = red[0];
    if (mode == 0) scal[0] = s;
    else if (mode == 1) {
        scal[1] = s;
        host_rel[1] = s <= 0.0 ? 1.f : 0.f;
        ab[0] = s <= 0.0 ? 0.f : (float)(scal[0] / s);
    } else if (mode == 2) {
        ab[1] = (float)(s / scal[0]);
        scal[0] = s;
    } else if (mode == 3) {
        scal[2] = s;
        host_rel[0] = (float)(sqrt(s) / scal[3]);
        host_rel[2] = 0.f;
        ((double*)(host_rel + 4))[0] = sqrt(s) / scal[3];
    } else {
        scal[3] = fmax(sqrt(s), 1e-30);
    }
}
// depth.rs:1064-1065: u += alpha p, r -= alpha Ap.
__global__ void axpy2_kernel(float* __restrict__ u, const float* __restrict__ p, float* __restrict__ r, const float* __restrict__ ap,
                             const float* ab, size_t n) {
    const float alpha = ab[0];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        u[i] = __fadd_rn(u[i], __fmul_rn(alpha, p[i]));
        r[i] = __fsub_rn(r[i], __fmul_rn(alpha, ap[i]));
    }
}
// depth.rs:1074: p = z + beta p.
__global__ void pupd_kernel(float* __restrict__ p, const float* __restrict__ z, const float* ab, size_t n) {
    const float beta = ab[1];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = __fadd_rn(z[i], __fmul_rn(beta, p[i]));
}
// depth.rs:1039: b = w d.
__global__ void mul_kernel(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ o, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        o[i] = __fmul_rn(a[i], b[i]);
}
__global__ void fill_kernel(float* o, float v, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) o[i] = v;
}

WlsSolver* wls_alloc(int w, int h, cudaError_t* err) {
    *err = cudaSuccess;
    // set here, outside the graph captures of the CG iteration that launch it
    static const cudaError_t coarse_attr = cudaFuncSetAttribute(coarse_h_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (coarse_attr != cudaSuccess) {
        *err = coarse_attr;
        return nullptr;
    }
    WlsSolver* S = new WlsSolver();
    S->w = w;
    S->h = h;
    size_t n = (size_t)w * h;
    S->ex = S->alloc(n, err);
    S->ey = S->alloc(n, err);
    int cw = w, ch = h;
    while (true) {
        WlsLevel L;
        L.w = cw;
        L.h = ch;
        size_t m = (size_t)cw * ch;
        L.wd = S->alloc(m, err);
        L.ax = S->alloc(m, err);
        L.ay = S->alloc(m, err);
        L.dinv = S->alloc(m, err);
        L.x = S->alloc(m, err);
        L.b = S->alloc(m, err);
        L.r = S->alloc(m, err);
        uint16_t** hs[7] = {&L.hwd, &L.hax, &L.hay, &L.hdinv, &L.hx, &L.hb, &L.hr};
        for (uint16_t** h : hs) *h = (uint16_t*)S->alloc((m + 1) / 2, err);
        S->lv.push_back(L);
        if (std::max(cw, ch) <= MG_MIN) break;
        cw = (cw + 1) / 2;
        ch = (ch + 1) / 2;
    }
    S->cp = S->alloc(n, err);
    S->dp = S->alloc(n, err);
    S->f = S->alloc(n, err);
    S->r = S->alloc(n, err);
    S->z = S->alloc(n, err);
    S->p = S->alloc(n, err);
    S->ap = S->alloc(n, err);
    S->part = (double*)S->alloc(2 * DOT_BLOCKS, err);
    S->scal = (double*)S->alloc(16, err);
    S->alpha_beta = S->alloc(4, err);
    if (cudaHostAlloc((void**)&S->host_rel, 64, cudaHostAllocDefault) != cudaSuccess) *err = cudaErrorMemoryAllocation;
    return S;
}

cudaError_t wls_prepare(WlsSolver* S, const float* guide, float lambda, float sigma_c, int edge_mode, cudaStream_t s) {
    const int w = S->w, h = S->h;
    S->lambda = lambda;
    const float inv = -1.0f / std::max(sigma_c, 1e-6f);
    const float inv2s2 = 1.0f / (2.0f * sigma_c * sigma_c);
    lsb_launched(), edge_kernel<<<g2(w, h), B2, 0, s>>>(guide, w, h, inv, inv2s2, edge_mode, lambda, S->ex, S->ey, S->lv[0].ax, S->lv[0].ay);
    for (size_t l = 1; l < S->lv.size(); l++) {
        const WlsLevel &F = S->lv[l - 1], &C = S->lv[l];
        lsb_launched(), coarsen_edges_kernel<<<g2(C.w, C.h), B2, 0, s>>>(F.ax, F.ay, F.w, F.h, C.ax, C.ay, C.w, C.h);
    }
    return cudaGetLastError();
}

WlsSolver* wls_create(const float* guide, int w, int h, float lambda, float sigma_c, int edge_mode, cudaStream_t s,
                      cudaError_t* err) {
    WlsSolver* S = wls_alloc(w, h, err);
    if (*err != cudaSuccess) return S;
    *err = wls_prepare(S, guide, lambda, sigma_c, edge_mode, s);
    return S;
}

int wls_width(const WlsSolver* s) { return s->w; }
int wls_height(const WlsSolver* s) { return s->h; }

void wls_destroy(WlsSolver* s) {
    if (!s) return;
    if (s->gA) cudaGraphExecDestroy(s->gA);
    if (s->gB) cudaGraphExecDestroy(s->gB);
    for (void* p : s->allocs) cudaFree(p);
    if (s->host_rel) cudaFreeHost(s->host_rel);
    delete s;
}

int wls_levels(const WlsSolver* s) { return (int)s->lv.size(); }

cudaError_t wls_set_weights(WlsSolver* S, const float* conf, cudaStream_t s) {
    lsb_launched(), wd_kernel<<<g1((size_t)S->w * S->h), 256, 0, s>>>(conf, S->lv[0].wd, (size_t)S->w * S->h);
    for (size_t l = 0; l < S->lv.size(); l++) {
        const WlsLevel& C = S->lv[l];
        if (l > 0) {
            const WlsLevel& F = S->lv[l - 1];
            lsb_launched(), block_sum_kernel<<<g2(C.w, C.h), B2, 0, s>>>(F.wd, F.w, F.h, C.wd, C.w, C.h);
        }
        lsb_launched(), dinv_kernel<<<g2(C.w, C.h), B2, 0, s>>>(C.wd, C.ax, C.ay, C.w, C.h, C.dinv);
    }
    // the BF16 V-cycle's operators (levels 0 .. MG_H_LEVELS-1)
    for (size_t l = 0; l < S->lv.size() && l < (size_t)MG_H_LEVELS; l++) {
        const WlsLevel& C = S->lv[l];
        const size_t m = (size_t)C.w * C.h;
        const float* src[4] = {C.wd, C.ax, C.ay, C.dinv};
        uint16_t* dst[4] = {C.hwd, C.hax, C.hay, C.hdinv};
        for (int q = 0; q < 4; q++) lsb_launched(), to_bf16_kernel<<<g1(m), 256, 0, s>>>(src[q], dst[q], m);
    }
    return cudaGetLastError();
}

static void jacobi(WlsLevel& L, bool zero, cudaStream_t s) {
    if (zero) {
        lsb_launched(), jac0_kernel<<<g1((size_t)L.w * L.h), 256, 0, s>>>(L.b, L.dinv, L.x, (size_t)L.w * L.h);
        return;
    }
    lsb_launched(), stencil_kernel<<<g2(L.w, L.h), B2, 0, s>>>(L.x, L.b, L.wd, L.ax, L.ay, L.dinv, L.r, L.w, L.h, 2);
    std::swap(L.x, L.r);
}

static bool tail_level(const WlsSolver* S, size_t l) {
    return (size_t)S->lv[l].w * S->lv[l].h <= (size_t)MG_TAIL_CELLS && S->lv.size() - l <= (size_t)MG_TAIL_MAX;
}
// depth.rs:924 `vcycle` on a level with a coarser one (MG_PRE = MG_POST = 1): down and up in one pass
// each. The right-hand side is bin (null: the level's b); the result lands in xout (null: the level's
// x, through its r buffer).
static void vcycle(WlsSolver* S, size_t l, cudaStream_t s);
static void vcycle_fused(WlsSolver* S, size_t l, const float* bin, float* xout, cudaStream_t s) {
    WlsLevel& T = S->lv[l];
    WlsLevel& C = S->lv[l + 1];
    const float* b = bin ? bin : T.b;
    lsb_launched(), vc_down_kernel<<<g2(C.w, C.h), B2, 0, s>>>(b, T.wd, T.ax, T.ay, T.dinv, T.x, T.w, T.h, C.b, C.w, C.h);
    vcycle(S, l + 1, s);
    float* out = xout ? xout : T.r;
    lsb_launched(), vc_up_kernel<<<g2(T.w, T.h), B2, 0, s>>>(T.x, C.x, C.w, b, T.wd, T.ax, T.ay, T.dinv, out, T.w, T.h);
    if (!xout) std::swap(T.x, T.r);
}
static void vcycle(WlsSolver* S, size_t l, cudaStream_t s) {
    WlsLevel& T = S->lv[l];
    if (l + 1 < S->lv.size() && !tail_level(S, l)) {
        vcycle_fused(S, l, nullptr, nullptr, s);
        return;
    }
    if (tail_level(S, l)) {
        MgTail tl;
        tl.n = (int)(S->lv.size() - l);
        for (int q = 0; q < tl.n; q++) tl.lv[q] = S->lv[l + q];
        lsb_launched(), vcycle_tail_kernel<<<1, 1024, 0, s>>>(tl);
        return;
    }
    if (l + 1 == S->lv.size()) {
        for (int k = 0; k < MG_COARSE; k++) jacobi(T, k == 0, s);
        return;
    }
    jacobi(T, true, s);
    lsb_launched(), stencil_kernel<<<g2(T.w, T.h), B2, 0, s>>>(T.x, T.b, T.wd, T.ax, T.ay, T.dinv, T.r, T.w, T.h, 1);
    WlsLevel& C = S->lv[l + 1];
    lsb_launched(), block_sum_kernel<<<g2(C.w, C.h), B2, 0, s>>>(T.r, T.w, T.h, C.b, C.w, C.h);
    vcycle(S, l + 1, s);
    lsb_launched(), prolong_kernel<<<g2(T.w, T.h), B2, 0, s>>>(T.x, T.w, T.h, C.x, C.w);
    jacobi(T, false, s);
}

// A damped Jacobi sweep on level L (zero: the zero-start one) against its BF16 right-hand side:
// the coarsest level's sweeps when it does not fit one CTA's shared memory.
static void jacobi_h(WlsLevel& L, bool zero, cudaStream_t s) {
    if (zero) {
        lsb_launched(), jac0_h_kernel<uint16_t><<<g1((size_t)L.w * L.h), 256, 0, s>>>(L.hb, L.hdinv, L.hx, (size_t)L.w * L.h);
        return;
    }
    lsb_launched(), stencil_h_kernel<uint16_t, uint16_t><<<g2(L.w, L.h), B2, 0, s>>>(L.hx, L.hb, L.hwd, L.hax, L.hay, L.hdinv, L.hr, L.w,
                                                                                   L.h, 2);
    std::swap(L.hx, L.hr);
}
static size_t coarse_h_smem(const WlsLevel& L) { return sizeof(uint16_t) * COARSE_H_PLANES * (size_t)L.w * L.h; }
static bool coarse_h_fits(const WlsLevel& L) { return coarse_h_smem(L) <= 227 * 1024; }
// the mixed-precision V-cycle: MG_H_SWEEPS pre/post sweeps, MG_H_LEVELS levels, MG_COARSE sweeps on
// the coarsest (one CTA). b32 / z32: level 0 takes the CG's FP32 residual as its right-hand side and
// its last sweep writes the FP32 z (no conversion passes).
static void vcycle_h(WlsSolver* S, size_t l, cudaStream_t s, const float* b32 = nullptr, float* z32 = nullptr) {
    WlsLevel& T = S->lv[l];
    const size_t last = std::min(S->lv.size(), (size_t)MG_H_LEVELS) - 1;
    if (l == last) {
        if (coarse_h_fits(T)) {
            const size_t smem = coarse_h_smem(T);  // at most 227 KB (wls_alloc raised the kernel's limit)
            lsb_launched(), coarse_h_kernel<<<1, dim3(32, 32), smem, s>>>(T.hx, T.hb, T.hwd, T.hax, T.hay, T.hdinv, T.w, T.h, MG_COARSE);
        } else {
            for (int k = 0; k < MG_COARSE; k++) jacobi_h(T, k == 0, s);
        }
        return;
    }
    static_assert(MG_H_SWEEPS == 2, "the fused BF16 passes run the zero-start sweep and one more down, two up");
    auto down_up = [&](auto* b) {  // the way down and the way up in one pass each
        using BT = std::remove_cv_t<std::remove_pointer_t<decltype(b)>>;
        WlsLevel& C = S->lv[l + 1];
        lsb_launched(), vc_down_h_kernel<BT><<<g2(C.w, C.h), B2, 0, s>>>(b, T.hwd, T.hax, T.hay, T.hdinv, T.hx, T.w, T.h, C.hb, C.w, C.h);
        vcycle_h(S, l + 1, s);
        if (z32) {
            lsb_launched(), vc_up_h_kernel<BT, float><<<g2(T.w, T.h), B2, 0, s>>>(T.hx, C.hx, C.w, b, T.hwd, T.hax, T.hay, T.hdinv, z32, T.w, T.h);
        } else {
            lsb_launched(), vc_up_h_kernel<BT, uint16_t><<<g2(T.w, T.h), B2, 0, s>>>(T.hx, C.hx, C.w, b, T.hwd, T.hax, T.hay, T.hdinv, T.hr, T.w,
                                                                                    T.h);
            std::swap(T.hx, T.hr);
        }
    };
    if (b32) down_up(b32);
    else down_up((const uint16_t*)T.hb);
}

static void dot(WlsSolver* S, const float* a, const float* b, size_t n, int mode, cudaStream_t s) {
    int nb = (int)std::min<size_t>(DOT_BLOCKS, (n + 255) / 256);
    lsb_launched(), dot_partial_kernel<<<nb, 256, 0, s>>>(a, b, n, S->part);
    lsb_launched(), dot_final_kernel<<<1, 256, 0, s>>>(S->part, nb, S->scal, S->alpha_beta, S->host_rel, mode);
}

cudaError_t wls_solve(WlsSolver* S, const float* d, int max_iters, float* u, float* rel_out, int* iters_out, cudaStream_t s,
                      int mode, bool x0_given, double* rel64) {
    const int w = S->w, h = S->h;
    const size_t n = (size_t)w * h;
    WlsLevel& L0 = S->lv[0];
    if (w == 1 || h == 1) {
        if (h == 1) thomas(true, u, d, L0.wd, 0, S->ex, w, h, S->lambda, S->cp, S->dp, nullptr, s);
        else thomas(false, u, d, L0.wd, 0, S->ey, w, h, S->lambda, S->cp, S->dp, nullptr, s);
        *rel_out = 0.f;
        *iters_out = 0;
        if (rel64) *rel64 = 0.0;
        return cudaGetLastError();
    }
    if (!x0_given) {
        // depth.rs:1022-1034: three separable sweeps, the first confidence-weighted
        cudaMemcpyAsync(S->f, d, n * sizeof(float), cudaMemcpyDeviceToDevice, s);
        for (int t = 1; t <= 3; t++) {
            float p4 = 1.f;
            for (int q = 0; q < 3 - t; q++) p4 *= 4.f;
            const float lam_t = (1.5f * S->lambda * p4) / (64.f - 1.f);
            thomas(true, u, S->f, L0.wd, t == 1 ? 0 : 1, S->ex, w, h, lam_t, S->cp, S->dp, S->z, s);
            cudaMemcpyAsync(S->f, u, n * sizeof(float), cudaMemcpyDeviceToDevice, s);
            thomas(false, u, S->f, L0.wd, 1, S->ey, w, h, lam_t, S->cp, S->dp, S->z, s);
            cudaMemcpyAsync(S->f, u, n * sizeof(float), cudaMemcpyDeviceToDevice, s);
        }
    }
    // b = W d, |b|, r = b - A u, z = M r, p = z
    lsb_launched(), mul_kernel<<<g1(n), 256, 0, s>>>(L0.wd, d, S->f, n);
    dot(S, S->f, S->f, n, 4, s);
    lsb_launched(), stencil_kernel<<<g2(w, h), B2, 0, s>>>(u, S->f, L0.wd, L0.ax, L0.ay, L0.dinv, S->r, w, h, 1);
    auto precond = [&]() {
        if (mode == 1) {
            if (std::min(S->lv.size(), (size_t)MG_H_LEVELS) > 1) {  // r in, z out, no conversion passes
                vcycle_h(S, 0, s, S->r, S->z);
                return;
            }
            lsb_launched(), to_bf16_kernel<<<g1(n), 256, 0, s>>>(S->r, L0.hb, n);
            vcycle_h(S, 0, s);
            lsb_launched(), from_bf16_kernel<<<g1(n), 256, 0, s>>>(S->lv[0].hx, S->z, n);
            return;
        }
        if (S->lv.size() > 1 && !tail_level(S, 0)) {  // r in, z out: no copies
            vcycle_fused(S, 0, S->r, S->z, s);
            return;
        }
        cudaMemcpyAsync(L0.b, S->r, n * sizeof(float), cudaMemcpyDeviceToDevice, s);
        vcycle(S, 0, s);
        cudaMemcpyAsync(S->z, S->lv[0].x, n * sizeof(float), cudaMemcpyDeviceToDevice, s);
    };
    precond();
    cudaMemcpyAsync(S->p, S->z, n * sizeof(float), cudaMemcpyDeviceToDevice, s);
    dot(S, S->r, S->z, n, 0, s);
    dot(S, S->r, S->r, n, 3, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    float rel = S->host_rel[0];
    int iters = 0;
    auto partA = [&]() {
        lsb_launched(), stencil_kernel<<<g2(w, h), B2, 0, s>>>(S->p, S->f, L0.wd, L0.ax, L0.ay, L0.dinv, S->ap, w, h, 0);
        dot(S, S->p, S->ap, n, 1, s);
        lsb_launched(), axpy2_kernel<<<g1(n), 256, 0, s>>>(u, S->p, S->r, S->ap, S->alpha_beta, n);
        dot(S, S->r, S->r, n, 3, s);
    };
    auto partB = [&]() {
        precond();
        dot(S, S->r, S->z, n, 2, s);
        lsb_launched(), pupd_kernel<<<g1(n), 256, 0, s>>>(S->p, S->z, S->alpha_beta, n);
    };
    // Every V-cycle restarts each level from zero, so which of a level's two buffers holds x
    // carries nothing from one cycle to the next: one captured cycle serves every iteration.
    auto capture = [&](const std::function<void()>& part, cudaGraphExec_t* ex, long long* kcount) -> bool {
        cudaGraph_t g = nullptr;
        const uint64_t c0 = lsb_launched_now();
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return false;
        part();
        const cudaError_t ec = cudaStreamEndCapture(s, &g);
        *kcount = (long long)(lsb_launched_now() - c0);
        lsb_launched_add(-*kcount);  // captured, not launched
        bool ok = ec == cudaSuccess && g && cudaGraphInstantiate(ex, g, 0) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
        return ok;
    };
    bool graphs = max_iters > 0;
    if (graphs && (!S->gA || S->g_u != u || S->g_mode != mode)) {
        if (S->gA) cudaGraphExecDestroy(S->gA);
        if (S->gB) cudaGraphExecDestroy(S->gB);
        S->gA = S->gB = nullptr;
        graphs = capture(partA, &S->gA, &S->kA) && capture(partB, &S->gB, &S->kB);
        if (!graphs) {  // launch directly instead
            if (S->gA) cudaGraphExecDestroy(S->gA);
            if (S->gB) cudaGraphExecDestroy(S->gB);
            S->gA = S->gB = nullptr;
            cudaGetLastError();
        } else {
            S->g_u = u;
            S->g_mode = mode;
        }
    }
    for (int it = 0; it < max_iters; it++) {
        if (rel < 1e-5f) break;
        iters++;
        if (graphs) {
            e = cudaGraphLaunch(S->gA, s);
            if (e != cudaSuccess) return e;
            lsb_launched_add(S->kA);
        } else {
            partA();
        }
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return e;
        if (S->host_rel[1] != 0.f) break;  // p.Ap <= 0: alpha was 0, u and r are unchanged (depth.rs:1060)
        rel = S->host_rel[0];
        if (rel < 1e-5f) break;
        if (graphs) {
            e = cudaGraphLaunch(S->gB, s);
            if (e != cudaSuccess) return e;
            lsb_launched_add(S->kB);
        } else {
            partB();
        }
    }
    *rel_out = rel;
    *iters_out = iters;
    if (rel64) *rel64 = ((double*)(S->host_rel + 4))[0];
    return cudaGetLastError();
}

}  // namespace lsb
