// Registration on the device (crates/lapstack-core/src/align.rs): the luma
// registration pyramid (align.rs:674 `reduce_burt`, a = 0.33, border-
// renormalised), the DC-removed RMS cost of a warped target (align.rs:581
// `warp_cost`: f64 source points and sums, f32 Spline4x4 taps) evaluated for
// a BATCH of candidate transforms per launch, the full-frame luma warp that
// becomes the next frame's reference (align.rs:542 `warp_plane`), and the
// brightness sums of every aligned frame against frame 0 (brightness.rs:67).
//
// The bounded Nelder-Mead search (align.rs:796) evaluates the reflection,
// expansion and contraction points of an iteration together (the search then
// takes the branch the reference takes), and a shrink's n points together.
// By default the whole multi-level search of a frame runs in one cooperative
// launch (`multiscale_align_dev`); the host-driven form, one launch and one
// small read-back per simplex step, stays for a device without cooperative
// launch and as the cross-check of the device search.
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <functional>
#include <vector>

#include "lsb_align.h"
#include "lsb_common.cuh"
#include "lsb_interp.cuh"

namespace lsb {
namespace cg = cooperative_groups;

// align.rs:220 `Sim::SPAN`: the search box around the initial transform, per parameter.
static const double SPAN[8] = {0.10, 0.10, 0.10, 0.087266462599716474, 0.05, 0.05, 0.05, 0.05};
__constant__ double c_span[8] = {0.10, 0.10, 0.10, 0.087266462599716474, 0.05, 0.05, 0.05, 0.05};

// ------------------------------------------------------------------ kernels
__global__ void luma_u16_kernel(const uint16_t* __restrict__ f, size_t n, float* __restrict__ y) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint16_t* p = f + 3 * i;
        y[i] = lsb_luma(__fmul_rn((float)p[0], LSB_INV16), __fmul_rn((float)p[1], LSB_INV16), __fmul_rn((float)p[2], LSB_INV16));
    }
}

// align.rs:650 Burt's kernel, a = 0.33: [c, b, a, b, c] with c = 0.25 - a/2 in f32
// (set from the host, whose f32 division and subtraction round the same way).
__constant__ float c_burt[5];
// align.rs:658 `norm_full`: the in-bounds taps summed in order
__device__ __forceinline__ float burt_norm(int i, int n) {
    float s = 0.f;
#pragma unroll
    for (int t = 0; t < 5; t++) {
        int x = i + t - 2;
        if (x >= 0 && x < n) s = __fadd_rn(s, c_burt[t]);
    }
    return s;
}
// align.rs:674 `reduce_burt`, one output sample: the horizontal in-bounds sums
// of the five rows, the vertical in-bounds sum, then / (row norm * column norm).
__global__ void reduce_burt_kernel(const float* __restrict__ src, int w, int h, float* __restrict__ out, int ow, int oh) {
    const int oj = blockIdx.x * blockDim.x + threadIdx.x, oi = blockIdx.y * blockDim.y + threadIdx.y;
    if (oj >= ow || oi >= oh) return;
    const int cx = 2 * oj, cy = 2 * oi;
    float v = 0.f;
    if (cx >= 2 && cx + 2 < w && cy >= 2 && cy + 2 < h) {
        const float* row = src + (size_t)(cy - 2) * w + cx - 2;
#pragma unroll
        for (int t = 0; t < 5; t++, row += w) {
            float a = 0.f;
#pragma unroll
            for (int u = 0; u < 5; u++) a = __fadd_rn(a, __fmul_rn(c_burt[u], row[u]));
            v = __fadd_rn(v, __fmul_rn(c_burt[t], a));
        }
    } else {
        for (int t = 0; t < 5; t++) {
            const int y = cy + t - 2;
            if (y < 0 || y >= h) continue;
            const float* row = src + (size_t)y * w;
            float a = 0.f;
            for (int u = 0; u < 5; u++) {
                const int x = cx + u - 2;
                if (x >= 0 && x < w) a = __fadd_rn(a, __fmul_rn(c_burt[u], row[x]));
            }
            v = __fadd_rn(v, __fmul_rn(c_burt[t], a));
        }
    }
    out[(size_t)oi * ow + oj] = __fdiv_rn(v, __fmul_rn(burt_norm(cy, h), burt_norm(cx, w)));
}

// align.rs:639 `spline4f`
__device__ __forceinline__ void spline4f(float t, float w[4]) {
    w[0] = __fmul_rn(__fsub_rn(__fmul_rn(__fadd_rn(__fmul_rn(-1.0f / 3.0f, t), 0.8f), t), 0.46666667f), t);
    w[1] = __fadd_rn(__fmul_rn(__fsub_rn(__fmul_rn(__fsub_rn(t, 1.8f), t), 0.2f), t), 1.0f);
    w[2] = __fmul_rn(__fadd_rn(__fmul_rn(__fsub_rn(1.2f, t), t), 0.8f), t);
    w[3] = __fmul_rn(__fsub_rn(__fmul_rn(__fsub_rn(__fmul_rn(1.0f / 3.0f, t), 0.2f), t), 0.13333334f), t);
}

// align.rs:485 `affine_row` + align.rs:291 `map`
__device__ __forceinline__ void src_point(const double* m, bool aff, double x, double y, double& sx, double& sy) {
    if (aff) {
        sx = __dadd_rn(__dadd_rn(__dmul_rn(m[1], y), m[2]), __dmul_rn(m[0], x));
        sy = __dadd_rn(__dadd_rn(__dmul_rn(m[4], y), m[5]), __dmul_rn(m[3], x));
    } else {
        const double d = __dadd_rn(__dadd_rn(__dmul_rn(m[6], x), __dmul_rn(m[7], y)), m[8]);
        sx = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[0], x), __dmul_rn(m[1], y)), m[2]), d);
        sy = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[3], x), __dmul_rn(m[4], y)), m[5]), d);
    }
}

// align.rs:581 `warp_cost` for up to MAX_CAND candidates (blockIdx.y): per
// block f64 partial sums of d, d^2 and the count, tree-reduced in a fixed order.
__global__ void cost_kernel(const float* __restrict__ rf, int aw, int ah, const float* __restrict__ tgt, int tw, int th,
                            const CostBatch cb, double* __restrict__ part) {
    const int k = blockIdx.y;
    const double* m = cb.inv[k];
    const bool aff = m[6] == 0.0 && m[7] == 0.0 && m[8] == 1.0;
    const double xmax = (double)(tw - 1), ymax = (double)(th - 1);
    double sd = 0.0, sd2 = 0.0, cnt = 0.0;
    const size_t n = (size_t)aw * ah;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % aw), y = (int)(i / aw);
        double sx, sy;
        src_point(m, aff, (double)x, (double)y, sx, sy);
        if (!(sx >= 0.0 && sx <= xmax && sy >= 0.0 && sy <= ymax)) continue;
        const double fx = floor(sx), fy = floor(sy);
        const int x0 = (int)fx, y0 = (int)fy;
        float wx[4], wy[4];
        spline4f((float)__dsub_rn(sx, fx), wx);
        spline4f((float)__dsub_rn(sy, fy), wy);
        float acc = 0.f;
        for (int j = 0; j < 4; j++) {
            const float* row = tgt + (size_t)min(max(y0 + j - 1, 0), th - 1) * tw;
            float r = 0.f;
            for (int u = 0; u < 4; u++) r = __fadd_rn(r, __fmul_rn(wx[u], row[min(max(x0 + u - 1, 0), tw - 1)]));
            acc = __fadd_rn(acc, __fmul_rn(wy[j], r));
        }
        const double d = (double)__fsub_rn(rf[i], acc);
        sd += d;
        sd2 += d * d;
        cnt += 1.0;
    }
    __shared__ double red[3][256];
    red[0][threadIdx.x] = sd;
    red[1][threadIdx.x] = sd2;
    red[2][threadIdx.x] = cnt;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st)
            for (int q = 0; q < 3; q++) red[q][threadIdx.x] += red[q][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; q++) part[((size_t)k * gridDim.x + blockIdx.x) * 3 + q] = red[q][0];
}
// align.rs:581 `warp_cost`, its f64 sums (align.rs:629): the per-block partials of every candidate summed in a fixed order: one
// block per candidate, each thread a fixed stride of blocks, then a tree.
__global__ void cost_final_kernel(const double* __restrict__ part, int nblocks, int ncand, double* __restrict__ out) {
    const int k = blockIdx.x;
    if (k >= ncand) return;
    double s[3] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
        for (int q = 0; q < 3; q++) s[q] += part[((size_t)k * nblocks + b) * 3 + q];
    __shared__ double red[3][128];
    for (int q = 0; q < 3; q++) red[q][threadIdx.x] = s[q];
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st)
            for (int q = 0; q < 3; q++) red[q][threadIdx.x] += red[q][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; q++) out[3 * k + q] = red[q][0];
}

// align.rs:489 `warp_with` on an f32 plane (edge-clamped; no fallback), the
// interpolation weights as in the fold's level-0 warp. The plane is w x h
// with rows `stride` floats apart.
__device__ __forceinline__ float warp_window_px(const float* __restrict__ src, size_t stride, int w, int h, const double* inv, bool affine,
                                                int interp, int x, int y) {
    double sx, sy;
    src_point(inv, affine, (double)x, (double)y, sx, sy);
    const double fx = floor(sx), fy = floor(sy);
    const int x0 = (int)fx, y0 = (int)fy;
    float wx[6], wy[6];
    const int n = interp_w(interp, __dsub_rn(sx, fx), wx);
    interp_w(interp, __dsub_rn(sy, fy), wy);
    const int start = 1 - n / 2;
    float acc = 0.f;
    for (int j = 0; j < n; j++) {
        const float* row = src + (size_t)min(max(y0 + start + j, 0), h - 1) * stride;
        float r = 0.f;
        for (int i = 0; i < n; i++) r = __fadd_rn(r, __fmul_rn(wx[i], row[min(max(x0 + start + i, 0), w - 1)]));
        acc = __fadd_rn(acc, __fmul_rn(wy[j], r));
    }
    return acc;
}
__device__ __forceinline__ float warp_plane_px(const float* __restrict__ src, int w, int h, const double* inv, bool affine, int interp,
                                               int x, int y) {
    return warp_window_px(src, (size_t)w, w, h, inv, affine, interp, x, y);
}
// prep.rs:46 `resize` / :63 `resize_plane` of a window (x0, y0, sw x sh) of planes `stride` floats
// wide, `pstride` floats apart: align.rs:542 `warp_plane` of the window through the scaling Sim the
// host turned into `inv`, onto ow x oh (blockIdx.z the plane). Without `inv` (the sizes agree) the
// window is copied, as the reference returns the plane unchanged.
__global__ void resize_kernel(const float* __restrict__ src, size_t stride, size_t pstride, int x0, int y0, int sw, int sh,
                              const WarpXform xf, int scaled, int ow, int oh, float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= ow || y >= oh) return;
    const float* p = src + (size_t)blockIdx.z * pstride + (size_t)y0 * stride + x0;
    out[(size_t)blockIdx.z * ow * oh + (size_t)y * ow + x] =
        scaled ? warp_window_px(p, stride, sw, sh, xf.inv, xf.affine, xf.interp, x, y) : p[(size_t)y * stride + x];
}
// align.rs:542 `warp_plane`, one thread per output pixel.
__global__ void warp_plane_kernel(const float* __restrict__ src, int w, int h, const WarpXform xf, float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    out[(size_t)y * w + x] = warp_plane_px(src, w, h, xf.inv, xf.affine, xf.interp, x, y);
}
// align.rs:542 `warp_plane` with the warp a search left in device memory: inverse [9],
// affine flag, identity flag (an identity result copies the plane, as the
// host path does).
__global__ void warp_plane_dev_kernel(const float* __restrict__ src, int w, int h, const double* __restrict__ wd, int interp,
                                      float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t k = (size_t)y * w + x;
    if (wd[10] != 0.0) {
        out[k] = src[k];
        return;
    }
    double inv[9];
    for (int q = 0; q < 9; q++) inv[q] = wd[q];
    out[k] = warp_plane_px(src, w, h, inv, wd[9] != 0.0, interp, x, y);
}

// brightness.rs:67 `sums` of every aligned frame against frame 0: over the
// stride-4 grid points that the frame's map (align.rs:291) keeps inside,
// the warped frame's channels (the pixel as shot where the warp leaves the
// frame) and frame 0's; f64 partials per part of the grid points, then in
// order. A block takes parts blockIdx.x, + gridDim.x, ...: the partials do
// not depend on how many blocks run.
__global__ void bright_kernel(const uint16_t* __restrict__ frames, int w, int h, const BrightXform* __restrict__ xf, int interp,
                              int nparts, double* __restrict__ part, int k0) {
    const int k = k0 + (int)blockIdx.y;
    const int gw = (w + 3) / 4, gh = (h + 3) / 4, ng = gw * gh;
    const uint16_t* f = frames + (size_t)k * w * h * 3;
    const BrightXform X = xf[k];
    __shared__ double red[7][128];
    for (int pi = blockIdx.x; pi < nparts; pi += gridDim.x) {
        const int per = (ng + nparts - 1) / nparts, lo = pi * per, hi = min(ng, lo + per);
        double s[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int g = lo + threadIdx.x; g < hi; g += blockDim.x) {
            const int x = (g % gw) * 4, y = (g / gw) * 4;
            if (!X.ident) {
                const double* m = X.inv;
                const double d = __dadd_rn(__dadd_rn(__dmul_rn(m[6], (double)x), __dmul_rn(m[7], (double)y)), m[8]);
                const double sx = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[0], (double)x), __dmul_rn(m[1], (double)y)), m[2]), d);
                const double sy = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[3], (double)x), __dmul_rn(m[4], (double)y)), m[5]), d);
                if (!(sx >= 0.0 && sx <= (double)(w - 1) && sy >= 0.0 && sy <= (double)(h - 1))) continue;
            }
            float v[3];
            load_px_core(f, X.inv, !X.ident, X.affine, interp, w, h, x, y, v);
            const uint16_t* r = frames + ((size_t)y * w + x) * 3;
            for (int c = 0; c < 3; c++) {
                s[c] += (double)v[c];
                s[3 + c] += (double)__fmul_rn((float)r[c], LSB_INV16);
            }
            s[6] += 1.0;
        }
        for (int q = 0; q < 7; q++) red[q][threadIdx.x] = s[q];
        __syncthreads();
        for (int st = blockDim.x / 2; st > 0; st >>= 1) {
            if (threadIdx.x < st)
                for (int q = 0; q < 7; q++) red[q][threadIdx.x] += red[q][threadIdx.x + st];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            for (int q = 0; q < 7; q++) part[((size_t)k * nparts + pi) * 7 + q] = red[q][0];
        __syncthreads();  // red is reused by the next part
    }
}

// brightness.rs:93 `ratio` of frame k from its partials (the host's bratio,
// operation for operation), with the gain flags and the storage scale.
__global__ void frame_gain_kernel(const double* __restrict__ part, int k, int nparts, FrameXform* __restrict__ xf) {
    __shared__ double ssum[7];
    if (threadIdx.x < 7) {  // one sum per thread, over the blocks in order
        const int q = threadIdx.x;
        double v = 0.0;
        for (int p = 0; p < nparts; p++) v += part[((size_t)k * nparts + p) * 7 + q];
        ssum[q] = v;
    }
    __syncthreads();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double sm[7];
    for (int q = 0; q < 7; q++) sm[q] = ssum[q];
    const size_t cnt = (size_t)sm[6];
    float maxg = 1.f;
    int on = 0;
    for (int c = 0; c < 3; c++) {
        float g = 1.0f;
        if (cnt >= 64) {
            const float v = sm[c] > 1e-9 ? (float)(sm[3 + c] / sm[c]) : 1.0f;
            g = fminf(fmaxf(v, 0.25f), 4.0f);
        }
        xf->gain[c] = g;
        if (fabsf(g - 1.0f) > 1e-6f) on |= 1 << c;
        maxg = fmaxf(maxg, g);
    }
    xf->gain_on = on;
    xf->gscale = (float)(65535.0 / maxg);
    xf->ginv = (float)(maxg / 65535.0);
}

// ------------------------------------------------------------------- host
cudaError_t frame_gain(const double* part, int k, int nparts, FrameXform* xf, cudaStream_t s) {
    lsb_launched(), frame_gain_kernel<<<1, 32, 0, s>>>(part, k, nparts, xf);
    return cudaGetLastError();
}

static int gsz(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

cudaError_t luma_u16(const uint16_t* f, int w, int h, float* y, cudaStream_t s) {
    size_t n = (size_t)w * h;
    lsb_launched(), luma_u16_kernel<<<gsz(n), 256, 0, s>>>(f, n, y);
    return cudaGetLastError();
}

void gauss_dims(int w, int h, std::vector<std::pair<int, int>>& dims) {
    dims.clear();
    int cw = w, ch = h;
    while (ch > 64 && cw > 8) {
        cw = (cw + 1) / 2;
        ch = (ch + 1) / 2;
        dims.push_back({cw, ch});
    }
}

static cudaError_t set_burt(cudaStream_t s) {
    static std::atomic<int> done[128];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
    if (done[dev].load()) return cudaSuccess;
    volatile float a = 0.33f, two = 2.0f, q = 0.25f;  // f32 arithmetic, as the reference's const fn
    const float c = q - a / two;
    const float k[5] = {c, 0.25f, 0.33f, 0.25f, c};
    cudaError_t e = cudaMemcpyToSymbol(c_burt, k, sizeof k);
    if (e == cudaSuccess) done[dev].store(1);
    (void)s;
    return e;
}

cudaError_t gauss_levels(const float* y, int w, int h, const std::vector<float*>& lv, cudaStream_t s) {
    cudaError_t e0 = set_burt(s);
    if (e0 != cudaSuccess) return e0;
    std::vector<std::pair<int, int>> dims;
    gauss_dims(w, h, dims);
    const float* src = y;
    int cw = w, ch = h;
    for (size_t l = 0; l < dims.size() && l < lv.size(); l++) {
        dim3 b(32, 8), g((dims[l].first + 31) / 32, (dims[l].second + 7) / 8);
        lsb_launched(), reduce_burt_kernel<<<g, b, 0, s>>>(src, cw, ch, lv[l], dims[l].first, dims[l].second);
        src = lv[l];
        cw = dims[l].first;
        ch = dims[l].second;
    }
    return cudaGetLastError();
}

cudaError_t warp_plane(const float* src, int w, int h, const WarpXform& xf, float* out, cudaStream_t s) {
    dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    lsb_launched(), warp_plane_kernel<<<g, b, 0, s>>>(src, w, h, xf, out);
    return cudaGetLastError();
}

// prep.rs:63 `resize_plane`: the Sim that maps the sw x sh source onto ow x oh with pixel centres
// corresponding (output pixel o reads source (o + 1/2) / k - 1/2, k = ow / sw on each axis).
cudaError_t resize_planes(const float* src, size_t stride, size_t pstride, int planes, int x0, int y0, int sw, int sh, int ow, int oh,
                          int interp, float* out, cudaStream_t s) {
    if (planes <= 0 || ow <= 0 || oh <= 0) return cudaSuccess;
    WarpXform xf{};
    xf.interp = interp;
    const bool scaled = sw != ow || sh != oh;
    if (scaled) {
        const double fw = (double)sw, fh = (double)sh, kx = (double)ow / fw, ky = (double)oh / fh;
        const double v[8] = {(kx - 1.0) * (fw + 1.0) / (2.0 * fw), (ky - 1.0) * (fh + 1.0) / (2.0 * fh), kx, 0.0, ky / kx, 0.0, 0.0, 0.0};
        double m[9];
        sim_matrix(v, sw, sh, m);
        mat_inverse(m, xf.inv);
        xf.affine = xf.inv[6] == 0.0 && xf.inv[7] == 0.0 && xf.inv[8] == 1.0;
    }
    dim3 b(32, 8), g((ow + 31) / 32, (oh + 7) / 8, planes);
    lsb_launched(), resize_kernel<<<g, b, 0, s>>>(src, stride, pstride, x0, y0, sw, sh, xf, scaled ? 1 : 0, ow, oh, out);
    return cudaGetLastError();
}

// align.rs:542 `warp_plane` in its Spline4x4 form over 64x16 tiles: the tile's source footprint (its
// corners' images, the taps' reach and a pixel of margin, clamped like the
// taps) is staged in shared memory once; the taps, weights and sums are
// warp_plane_px's. Identity warps copy; tiles whose footprint does not fit,
// and projective warps, take the per-pixel path. The CTAs are persistent: the
// next tile's footprint arrives by cp.async into the other buffer while this
// one is warped.
constexpr int PT_W = 64, PT_H = 16, PB_W = PT_W + 16, PB_H = PT_H + 16;
__device__ __forceinline__ void wp_cp4(float* sdst, const float* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(sdst)), "l"(gsrc));
}
// The footprint of tile t (affine warps): its origin and extent, and whether it fits the buffer.
__device__ __forceinline__ bool wp_footprint(const double* m, int w, int h, int tiles_x, int t, int& bx0, int& by0, int& bw, int& bh) {
    const int x0 = (t % tiles_x) * PT_W, y0 = (t / tiles_x) * PT_H;
    double mnx = 1e300, mxx = -1e300, mny = 1e300, mxy = -1e300;
    const int cx[2] = {x0, min(x0 + PT_W - 1, w - 1)}, cy[2] = {y0, min(y0 + PT_H - 1, h - 1)};
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++) {
            double sx, sy;
            src_point(m, true, (double)cx[a], (double)cy[b], sx, sy);
            mnx = fmin(mnx, sx);
            mxx = fmax(mxx, sx);
            mny = fmin(mny, sy);
            mxy = fmax(mxy, sy);
        }
    if (!(mnx > -1e9 && mxx < 1e9 && mny > -1e9 && mxy < 1e9)) return false;
    bx0 = (int)floor(mnx) - 2;
    by0 = (int)floor(mny) - 2;
    bw = (int)floor(mxx) + 3 - bx0 + 1;
    bh = (int)floor(mxy) + 3 - by0 + 1;
    return bw <= PB_W && bh <= PB_H;
}
__global__ void __launch_bounds__(256) warp_plane_tile_kernel(const float* __restrict__ src, int w, int h, const double* __restrict__ wd,
                                                              float* __restrict__ out) {
    __shared__ float box[2][PB_H][PB_W];
    __shared__ int fp[2][5];  // per buffer: fits, bx0, by0, bw, bh
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int tiles_x = (w + PT_W - 1) / PT_W, ntiles = tiles_x * ((h + PT_H - 1) / PT_H);
    const bool ident = wd[10] != 0.0, affine = wd[9] != 0.0;
    double m[9];
    for (int q = 0; q < 9; q++) m[q] = wd[q];
    // tile t's footprint into buffer b (thread 0 decides, every thread copies its share)
    auto stage = [&](int t, int b) {
        if (threadIdx.x == 0) {
            int bx0 = 0, by0 = 0, bw = 0, bh = 0;
            const bool f = t < ntiles && !ident && affine && wp_footprint(m, w, h, tiles_x, t, bx0, by0, bw, bh);
            fp[b][0] = f;
            fp[b][1] = bx0;
            fp[b][2] = by0;
            fp[b][3] = bw;
            fp[b][4] = bh;
        }
        __syncthreads();
        if (fp[b][0]) {
            const int bx0 = fp[b][1], by0 = fp[b][2], bw = fp[b][3], bh = fp[b][4];
            // m / bw by a multiply (exact for m < 2^16, bw <= 80)
            const unsigned magic = (unsigned)((0xffffffffull + bw) / bw);
            for (int e = threadIdx.x; e < bw * bh; e += 256) {
                const int r = (int)__umulhi((unsigned)e, magic), c = e - r * bw;
                wp_cp4(&box[b][r][c], src + (size_t)min(max(by0 + r, 0), h - 1) * w + min(max(bx0 + c, 0), w - 1));
            }
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    int b = 0;
    stage(blockIdx.x, 0);
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, b ^= 1) {
        stage(t + gridDim.x, b ^ 1);  // the other buffer's last reader finished before the loop's last barrier
        asm volatile("cp.async.wait_group 1;\n" ::);
        __syncthreads();  // tile t's footprint is in
        const int x0 = (t % tiles_x) * PT_W, y0 = (t / tiles_x) * PT_H;
        const bool fits = fp[b][0] != 0;
        const int bx0 = fp[b][1], by0 = fp[b][2];
#pragma unroll 1
        for (int q = 0; q < 4; q++) {
            const int x = x0 + tx + 32 * (q & 1), y = y0 + ty + 8 * (q >> 1);
            if (x >= w || y >= h) continue;
            const size_t k = (size_t)y * w + x;
            if (ident) {
                out[k] = src[k];
                continue;
            }
            if (!fits) {
                out[k] = warp_plane_px(src, w, h, m, affine, 3, x, y);
                continue;
            }
            double sx, sy;
            src_point(m, true, (double)x, (double)y, sx, sy);
            const double fx = floor(sx), fy = floor(sy);
            const int ix = (int)fx - 1 - bx0, iy = (int)fy - 1 - by0;
            float wx[4], wy[4];
            spline4_d(__dsub_rn(sx, fx), wx);
            spline4_d(__dsub_rn(sy, fy), wy);
            float acc = 0.f;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float r = 0.f;
#pragma unroll
                for (int i = 0; i < 4; i++) r = __fadd_rn(r, __fmul_rn(wx[i], box[b][iy + j][ix + i]));
                acc = __fadd_rn(acc, __fmul_rn(wy[j], r));
            }
            out[k] = acc;
        }
        __syncthreads();  // buffer b and its footprint record are free for tile t + 2 grid
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
}

static int warp_plane_grid(int ntiles) {
    static const int resident = [] {  // once per process, whichever thread comes first
        int dev = 0, sms = 1, per_sm = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, warp_plane_tile_kernel, 256, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
        return per_sm * std::max(sms, 1);
    }();
    return std::max(1, std::min(ntiles, resident));
}

cudaError_t warp_plane_dev(const float* src, int w, int h, const double* warp_dev, int interp, float* out, cudaStream_t s) {
    if (interp == 3) {
        const int ntiles = ((w + PT_W - 1) / PT_W) * ((h + PT_H - 1) / PT_H);
        lsb_launched(), warp_plane_tile_kernel<<<warp_plane_grid(ntiles), 256, 0, s>>>(src, w, h, warp_dev, out);
        return cudaGetLastError();
    }
    dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    lsb_launched(), warp_plane_dev_kernel<<<g, b, 0, s>>>(src, w, h, warp_dev, interp, out);
    return cudaGetLastError();
}

cudaError_t bright_sums(const uint16_t* frames, int n, int w, int h, const BrightXform* xf_dev, int interp, int nparts, double* part,
                        cudaStream_t s) {
    if (n < 2) return cudaSuccess;
    dim3 g(nparts, n - 1);
    lsb_launched(), bright_kernel<<<g, 128, 0, s>>>(frames, w, h, xf_dev, interp, nparts, part, 1);
    return cudaGetLastError();
}
cudaError_t bright_sums_frame(const uint16_t* frames, int k, int w, int h, const BrightXform* xf_dev, int interp, int nparts, double* part,
                              int blocks, cudaStream_t s) {
    if (k < 1) return cudaSuccess;
    lsb_launched(), bright_kernel<<<dim3(std::min(std::max(blocks, 1), nparts), 1), 128, 0, s>>>(frames, w, h, xf_dev, interp, nparts, part, k);
    return cudaGetLastError();
}

// --------------------------------------------------- the search (host side)
// align.rs:200-294 Sim::matrix and inverse, exactly as the reference.
void sim_matrix(const double* v, int w, int h, double m[9]) {
    const double cx = (double)w / 2.0, cy = (double)h / 2.0;
    const double c = std::cos(v[3]), sn = std::sin(v[3]);
    const double sc = v[2], shear = v[5], aspect = v[4];
    const double a = sc * c, b = sc * (c * shear - sn * aspect), d = sc * sn, e = sc * (sn * shear + c * aspect);
    const double gx = v[6] / (double)w, gy = v[7] / (double)h;
    const double a2 = a + cx * gx, b2 = b + cx * gy, d2 = d + cy * gx, e2 = e + cy * gy;
    m[0] = a2;
    m[1] = b2;
    m[2] = cx + v[0] * (double)w - (a2 * cx + b2 * cy);
    m[3] = d2;
    m[4] = e2;
    m[5] = cy + v[1] * (double)h - (d2 * cx + e2 * cy);
    m[6] = gx;
    m[7] = gy;
    m[8] = 1.0 - gx * cx - gy * cy;
}
void mat_inverse(const double m[9], double inv[9]) {
    if (m[6] == 0.0 && m[7] == 0.0 && m[8] == 1.0) {
        const double a = m[0], b = m[1], tx = m[2], d = m[3], e = m[4], ty = m[5];
        const double det = a * e - b * d;
        const double ia = e / det, ib = -b / det, id = -d / det, ie = a / det;
        inv[0] = ia;
        inv[1] = ib;
        inv[2] = -(ia * tx + ib * ty);
        inv[3] = id;
        inv[4] = ie;
        inv[5] = -(id * tx + ie * ty);
        inv[6] = 0.0;
        inv[7] = 0.0;
        inv[8] = 1.0;
        return;
    }
    auto M = [&](int i, int j) { return m[3 * i + j]; };
    auto cof = [&](int i, int j) {
        const int r0 = (i + 1) % 3, r1 = (i + 2) % 3, c0 = (j + 1) % 3, c1 = (j + 2) % 3;
        return M(r0, c0) * M(r1, c1) - M(r0, c1) * M(r1, c0);
    };
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) inv[3 * i + j] = cof(j, i);
    const double k = inv[8];
    for (int i = 0; i < 9; i++) inv[i] /= k;
}
bool sim_is_id(const double* v) {
    static const double id[8] = {0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < 8; k++)
        if (v[k] != id[k]) return false;
    return true;
}

// align.rs:581's cost for a batch of full Sim vectors on one level pair.
static cudaError_t eval_batch(AlignCtx& C, const float* rf, int aw, int ah, const float* tg, int tw, int th,
                              const std::vector<std::vector<double>>& sims, std::vector<double>& costs) {
    costs.assign(sims.size(), 0.0);
    for (size_t b0 = 0; b0 < sims.size(); b0 += MAX_CAND) {
        const int nc = (int)std::min<size_t>(MAX_CAND, sims.size() - b0);
        CostBatch cb;
        for (int k = 0; k < nc; k++) {
            double m[9];
            sim_matrix(sims[b0 + k].data(), tw, th, m);
            mat_inverse(m, cb.inv[k]);
        }
        const size_t npx = (size_t)aw * ah;
        const int nblocks = (int)std::min<size_t>(std::max<size_t>((npx + 255) / 256, 1), 296);
        dim3 g(nblocks, nc);
        lsb_launched(), cost_kernel<<<g, 256, 0, C.s>>>(rf, aw, ah, tg, tw, th, cb, C.part);
        lsb_launched(), cost_final_kernel<<<nc, 128, 0, C.s>>>(C.part, nblocks, nc, C.sums_dev);
        cudaMemcpyAsync(C.sums_host, C.sums_dev, sizeof(double) * 3 * nc, cudaMemcpyDeviceToHost, C.s);
        cudaError_t e = cudaStreamSynchronize(C.s);
        if (e != cudaSuccess) return e;
        C.launches++;
        for (int k = 0; k < nc; k++) {
            const double sd = C.sums_host[3 * k], sd2 = C.sums_host[3 * k + 1], cnt = C.sums_host[3 * k + 2];
            costs[b0 + k] = cnt < 16.0 ? 1e9 : std::sqrt(std::max((sd2 - sd * sd / cnt) / cnt, 0.0));
        }
    }
    return cudaSuccess;
}

// align.rs:796 `nelder_mead`, evaluations batched per iteration.
static cudaError_t nelder_mead_dev(AlignCtx& C, const std::function<cudaError_t(const std::vector<std::vector<double>>&, std::vector<double>&)>& F,
                                   const std::vector<double>& x0, const std::vector<double>& lo, const std::vector<double>& hi,
                                   const std::vector<double>& step, const std::vector<double>& tol, std::vector<double>& out) {
    const size_t n = x0.size();
    out = x0;
    if (n == 0) return cudaSuccess;
    auto clampv = [&](std::vector<double>& v) {
        for (size_t k = 0; k < n; k++) v[k] = std::min(std::max(v[k], lo[k]), hi[k]);
    };
    std::vector<std::vector<double>> simplex{x0};
    for (size_t k = 0; k < n; k++) {
        std::vector<double> v = x0;
        v[k] += step[k];
        clampv(v);
        simplex.push_back(v);
    }
    std::vector<double> fv;
    cudaError_t e = F(simplex, fv);
    if (e != cudaSuccess) return e;
    C.evals += n + 1;
    const double alpha = 1.0, gamma = 2.0, rho = 0.5, sigma = 0.5;
    for (int it = 0; it < 200; it++) {
        std::vector<size_t> idx(n + 1);
        for (size_t i = 0; i <= n; i++) idx[i] = i;
        std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return fv[a] < fv[b]; });
        std::vector<std::vector<double>> s2;
        std::vector<double> f2;
        for (size_t i : idx) {
            s2.push_back(simplex[i]);
            f2.push_back(fv[i]);
        }
        simplex.swap(s2);
        fv.swap(f2);
        // align.rs:888 `converged`
        bool conv = std::fabs(fv[n] - fv[0]) <= 1e-4 * (1.0 + std::fabs(fv[0]));
        for (size_t i = 1; conv && i <= n; i++)
            for (size_t k = 0; k < n; k++)
                if (!(std::fabs(simplex[i][k] - simplex[0][k]) <= tol[k])) {
                    conv = false;
                    break;
                }
        if (conv) break;
        std::vector<double> c(n, 0.0);
        for (size_t i = 0; i < n; i++)
            for (size_t k = 0; k < n; k++) c[k] += simplex[i][k];
        for (size_t k = 0; k < n; k++) c[k] /= (double)n;
        std::vector<double> xr(n), xe(n), xc(n);
        for (size_t k = 0; k < n; k++) xr[k] = c[k] + alpha * (c[k] - simplex[n][k]);
        clampv(xr);
        for (size_t k = 0; k < n; k++) xe[k] = c[k] + gamma * (xr[k] - c[k]);
        clampv(xe);
        for (size_t k = 0; k < n; k++) xc[k] = c[k] + rho * (simplex[n][k] - c[k]);
        clampv(xc);
        std::vector<double> f3;
        e = F({xr, xe, xc}, f3);
        if (e != cudaSuccess) return e;
        const double fr = f3[0], fe = f3[1], fc = f3[2];
        C.evals += 1;
        if (fr < fv[0]) {
            C.evals += 1;
            if (fe < fr) {
                simplex[n] = xe;
                fv[n] = fe;
            } else {
                simplex[n] = xr;
                fv[n] = fr;
            }
        } else if (fr < fv[n - 1]) {
            simplex[n] = xr;
            fv[n] = fr;
        } else {
            C.evals += 1;
            if (fc < fv[n]) {
                simplex[n] = xc;
                fv[n] = fc;
            } else {
                std::vector<std::vector<double>> pts;
                for (size_t i = 1; i <= n; i++) {
                    for (size_t k = 0; k < n; k++) simplex[i][k] = simplex[0][k] + sigma * (simplex[i][k] - simplex[0][k]);
                    clampv(simplex[i]);
                    pts.push_back(simplex[i]);
                }
                std::vector<double> fs;
                e = F(pts, fs);
                if (e != cudaSuccess) return e;
                C.evals += n;
                for (size_t i = 1; i <= n; i++) fv[i] = fs[i - 1];
            }
        }
    }
    size_t best = 0;
    for (size_t i = 1; i <= n; i++)
        if (fv[i] < fv[best]) best = i;
    out = simplex[best];
    return cudaSuccess;
}

// align.rs:896 `multiscale_align`: rf/tg full-res planes with their levels,
// the search driven from the host.
static cudaError_t multiscale_align_host(AlignCtx& C, const float* rf, const std::vector<float*>& pr, const float* tg,
                             const std::vector<float*>& pt, int w, int h, const double init[8], const bool freem[8], int coarsen,
                             double out[8]) {
    std::vector<std::pair<int, int>> dims;
    gauss_dims(w, h, dims);
    const size_t n = dims.size() + 1;
    std::vector<size_t> free_idx;
    for (size_t k = 0; k < 8; k++)
        if (freem[k]) free_idx.push_back(k);
    std::vector<double> lo_f, hi_f;
    for (size_t k : free_idx) {
        lo_f.push_back(init[k] - SPAN[k]);
        hi_f.push_back(init[k] + SPAN[k]);
    }
    std::vector<double> cur(init, init + 8);
    const size_t finest = std::min((size_t)coarsen, n - 1);
    for (size_t lvl = n; lvl-- > finest;) {
        const float* a_d = lvl == 0 ? rf : pr[lvl - 1];
        const float* t_d = lvl == 0 ? tg : pt[lvl - 1];
        const int lw = lvl == 0 ? w : dims[lvl - 1].first, lh = lvl == 0 ? h : dims[lvl - 1].second;
        const std::vector<double> snap = cur;
        auto F = [&](const std::vector<std::vector<double>>& xs, std::vector<double>& fs) {
            std::vector<std::vector<double>> sims;
            for (auto& xf : xs) {
                std::vector<double> v = snap;
                for (size_t k = 0; k < free_idx.size(); k++) v[free_idx[k]] = xf[k];
                sims.push_back(v);
            }
            return eval_batch(C, a_d, lw, lh, t_d, lw, lh, sims, fs);
        };
        std::vector<double> x0, step, tol;
        for (size_t k : free_idx) x0.push_back(cur[k]);
        // align.rs:784 `level_steps`
        const double wf = w, hf = h, r = std::max(wf, hf) / 2.0;
        const double gain[8] = {wf, hf, r, r, hf / 2.0, hf / 2.0, wf / 4.0, hf / 4.0};
        const double px = (double)((uint64_t)1 << lvl);
        for (size_t k : free_idx) {
            step.push_back(1.0 * px / gain[k]);
            tol.push_back(0.1 * px / gain[k]);
        }
        std::vector<double> best;
        cudaError_t e = nelder_mead_dev(C, F, x0, lo_f, hi_f, step, tol, best);
        if (e != cudaSuccess) return e;
        for (size_t k = 0; k < free_idx.size(); k++) cur[free_idx[k]] = best[k];
    }
    for (int k = 0; k < 8; k++) out[k] = cur[k];
    return cudaSuccess;
}

cudaError_t cost_single(AlignCtx& C, const float* rf, int aw, int ah, const float* tg, int tw, int th, const double sim[8],
                        double* cost) {
    std::vector<double> fs;
    cudaError_t e = eval_batch(C, rf, aw, ah, tg, tw, th, {std::vector<double>(sim, sim + 8)}, fs);
    *cost = fs.empty() ? 0.0 : fs[0];
    return e;
}

// ------------------------------------------- the search on the device
// align.rs:896 `multiscale_align` for one frame in ONE cooperative launch.
// Every block keeps its own copy of the Nelder-Mead state (align.rs:796).
// Per batch it evaluates the pending candidates over its share of the
// level's pixels (the cost of align.rs:581: f64 sums of d, d^2 and the
// count), publishes its partial sums, meets the other blocks at a grid
// barrier (only the blocks with pixels arrive; every block waits), sums
// those blocks' partials in one fixed order and advances its copy of the
// search. Every copy sees the same sums and takes the same
// branches, so one barrier per batch suffices; the partials alternate
// between two buffers, so a batch's writes never meet a slower block's reads
// of the batch before. The barrier's wait is bounded: on a timeout the
// kernel records an error and every block returns.
struct NmLevel {
    const float* rf;
    const float* tg;
    int w, h, lvl;
};
struct NmJob {
    NmLevel lv[24];
    int nlv;   // levels searched, coarsest first
    int W, H;  // full resolution
    double init[8];
    int free_idx[8], nfree;
    double* part;   // [2][MAX_CAND][3][gridDim.x]
    unsigned* bar;  // [0] arrivals of every batch so far (zero at launch)
    int* ctl;       // [0] error (sticky): 1 barrier timeout, 2 batch limit; [1] evaluations (the reference's count)
    double* out;    // the transform found [8]
    // chained searches (no host round trip between frames):
    const double* init_dev;        // if set, the initial transform (the previous frame's result) instead of init
    double* warp_dev;              // if set, the full-resolution warp of the result: inverse [9], affine, identity
    unsigned long long* evals_dev; // if set, evaluations are added here
    long long spin_limit;          // polls of the hand-off's wait before it gives up
};

__device__ void dev_sim_matrix(const double* v, int w, int h, double m[9]) {
    const double cx = (double)w / 2.0, cy = (double)h / 2.0;
    const double c = cos(v[3]), sn = sin(v[3]);
    const double sc = v[2], shear = v[5], aspect = v[4];
    const double a = __dmul_rn(sc, c), b = __dmul_rn(sc, __dsub_rn(__dmul_rn(c, shear), __dmul_rn(sn, aspect)));
    const double d = __dmul_rn(sc, sn), e = __dmul_rn(sc, __dadd_rn(__dmul_rn(sn, shear), __dmul_rn(c, aspect)));
    const double gx = __ddiv_rn(v[6], (double)w), gy = __ddiv_rn(v[7], (double)h);
    const double a2 = __dadd_rn(a, __dmul_rn(cx, gx)), b2 = __dadd_rn(b, __dmul_rn(cx, gy));
    const double d2 = __dadd_rn(d, __dmul_rn(cy, gx)), e2 = __dadd_rn(e, __dmul_rn(cy, gy));
    m[0] = a2;
    m[1] = b2;
    m[2] = __dsub_rn(__dadd_rn(cx, __dmul_rn(v[0], (double)w)), __dadd_rn(__dmul_rn(a2, cx), __dmul_rn(b2, cy)));
    m[3] = d2;
    m[4] = e2;
    m[5] = __dsub_rn(__dadd_rn(cy, __dmul_rn(v[1], (double)h)), __dadd_rn(__dmul_rn(d2, cx), __dmul_rn(e2, cy)));
    m[6] = gx;
    m[7] = gy;
    m[8] = __dsub_rn(__dsub_rn(1.0, __dmul_rn(gx, cx)), __dmul_rn(gy, cy));
}
__device__ void dev_mat_inverse(const double m[9], double inv[9]) {
    if (m[6] == 0.0 && m[7] == 0.0 && m[8] == 1.0) {
        const double a = m[0], b = m[1], tx = m[2], d = m[3], e = m[4], ty = m[5];
        const double det = __dsub_rn(__dmul_rn(a, e), __dmul_rn(b, d));
        const double ia = __ddiv_rn(e, det), ib = __ddiv_rn(-b, det), id = __ddiv_rn(-d, det), ie = __ddiv_rn(a, det);
        inv[0] = ia;
        inv[1] = ib;
        inv[2] = -__dadd_rn(__dmul_rn(ia, tx), __dmul_rn(ib, ty));
        inv[3] = id;
        inv[4] = ie;
        inv[5] = -__dadd_rn(__dmul_rn(id, tx), __dmul_rn(ie, ty));
        inv[6] = 0.0;
        inv[7] = 0.0;
        inv[8] = 1.0;
        return;
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            const int r0 = (j + 1) % 3, r1 = (j + 2) % 3, c0 = (i + 1) % 3, c1 = (i + 2) % 3;
            inv[3 * i + j] = __dsub_rn(__dmul_rn(m[3 * r0 + c0], m[3 * r1 + c1]), __dmul_rn(m[3 * r0 + c1], m[3 * r1 + c0]));
        }
    const double k = inv[8];
    for (int i = 0; i < 9; i++) inv[i] = __ddiv_rn(inv[i], k);
}

// A block's copy of the search: the simplex, its costs, the box and steps of
// the level, and the points of the batch in flight.
struct NmState {
    double cur[8], snap[8], simplex[9][8], fv[9], lo[8], hi[8], step[8], tol[8], xr[8], xe[8], xc[8];
    double pts[MAX_CAND][8];  // the pending candidates (free coordinates)
    int it, phase, evals;
};
enum { NM_INIT = 0, NM_RXC = 1, NM_SHRINK = 2 };

__device__ __forceinline__ void nm_put(NmState& S, int n, int k, const double* x) {
    for (int q = 0; q < n; q++) S.pts[k][q] = x[q];
}
__device__ void nm_clamp(const NmState& S, int n, double* v) {
    for (int q = 0; q < n; q++) v[q] = fmin(fmax(v[q], S.lo[q]), S.hi[q]);
}
// Start level L: the first simplex (align.rs:806-813). Returns the candidates pending.
__device__ int nm_level_start(const NmJob& J, NmState& S, int L) {
    const int n = J.nfree;
    for (int q = 0; q < 8; q++) S.snap[q] = S.cur[q];
    // align.rs:784 `level_steps`
    const double wf = J.W, hf = J.H, r = fmax(wf, hf) / 2.0;
    const double gain[8] = {wf, hf, r, r, hf / 2.0, hf / 2.0, wf / 4.0, hf / 4.0};
    const double px = (double)(1ull << J.lv[L].lvl);
    for (int q = 0; q < n; q++) {
        S.step[q] = __ddiv_rn(__dmul_rn(1.0, px), gain[J.free_idx[q]]);
        S.tol[q] = __ddiv_rn(__dmul_rn(0.1, px), gain[J.free_idx[q]]);
    }
    for (int q = 0; q < n; q++) S.simplex[0][q] = S.cur[J.free_idx[q]];
    for (int k = 0; k < n; k++) {
        for (int q = 0; q < n; q++) S.simplex[k + 1][q] = S.simplex[0][q];
        S.simplex[k + 1][k] = __dadd_rn(S.simplex[k + 1][k], S.step[k]);
        nm_clamp(S, n, S.simplex[k + 1]);
    }
    for (int k = 0; k <= n; k++) nm_put(S, n, k, S.simplex[k]);
    S.phase = NM_INIT;
    S.it = 0;
    return n + 1;
}
// One step of align.rs:796's loop (the top of align.rs:815's loop and the branch on the
// batch's costs), run by one warp: lane q owns free
// parameter q of every vertex, so the per-parameter arithmetic (centroid,
// reflection, expansion, contraction, shrink, clamps, the convergence test)
// runs in parallel in the reference's per-parameter operation order; the
// scalar decisions are taken identically by every lane. The stable sort by
// cost places vertex i at #{j: f_j < f_i} + #{j < i: f_j == f_i}, the
// position the insertion sort gives it.
__device__ int nm_iterate_warp(const NmJob& J, NmState& S, int lane) {
    const int n = J.nfree;
    const bool lq = lane < n;
    bool done = S.it >= 200;
    if (!done) {
        __syncwarp();
        if (lane == 0) S.it++;
        // stable sort: each lane i <= n moves its own vertex
        double row[8], fi = 0.0;
        int rank = 0;
        if (lane <= n) {
            fi = S.fv[lane];
            for (int q = 0; q < n; q++) row[q] = S.simplex[lane][q];
            for (int j = 0; j <= n; j++) {
                const double fj = S.fv[j];
                rank += (fj < fi) || (fj == fi && j < lane);
            }
        }
        __syncwarp();
        if (lane <= n) {
            S.fv[rank] = fi;
            for (int q = 0; q < n; q++) S.simplex[rank][q] = row[q];
        }
        __syncwarp();
        // align.rs:888 `converged`
        bool conv = fabs(__dsub_rn(S.fv[n], S.fv[0])) <= __dmul_rn(1e-4, __dadd_rn(1.0, fabs(S.fv[0])));
        bool mine = true;
        if (lq)
            for (int i = 1; i <= n; i++) mine = mine && fabs(__dsub_rn(S.simplex[i][lane], S.simplex[0][lane])) <= S.tol[lane];
        done = conv && __all_sync(0xffffffffu, mine);
    }
    if (done) {
        int best = 0;
        for (int i = 1; i <= n; i++)
            if (S.fv[i] < S.fv[best]) best = i;
        __syncwarp();
        if (lq) S.cur[J.free_idx[lane]] = S.simplex[best][lane];
        __syncwarp();
        return 0;
    }
    if (lq) {
        const int q = lane;
        double c = 0.0;
        for (int i = 0; i < n; i++) c = __dadd_rn(c, S.simplex[i][q]);
        c = __ddiv_rn(c, (double)n);
        const double xn = S.simplex[n][q];
        double xr = __dadd_rn(c, __dmul_rn(1.0, __dsub_rn(c, xn)));
        xr = fmin(fmax(xr, S.lo[q]), S.hi[q]);
        double xe = __dadd_rn(c, __dmul_rn(2.0, __dsub_rn(xr, c)));
        xe = fmin(fmax(xe, S.lo[q]), S.hi[q]);
        double xc = __dadd_rn(c, __dmul_rn(0.5, __dsub_rn(xn, c)));
        xc = fmin(fmax(xc, S.lo[q]), S.hi[q]);
        S.xr[q] = xr;
        S.xe[q] = xe;
        S.xc[q] = xc;
        S.pts[0][q] = xr;
        S.pts[1][q] = xe;
        S.pts[2][q] = xc;
    }
    if (lane == 0) S.phase = NM_RXC;
    __syncwarp();
    return 3;
}
__device__ int nm_advance_warp(const NmJob& J, NmState& S, const double* cost, int lane) {
    const int n = J.nfree;
    const bool lq = lane < n;
    const int phase = S.phase;
    __syncwarp();
    if (phase == NM_INIT) {
        if (lane <= n) S.fv[lane] = cost[lane];
        if (lane == 0) S.evals += n + 1;
        __syncwarp();
        return nm_iterate_warp(J, S, lane);
    }
    if (phase == NM_SHRINK) {
        if (lane >= 1 && lane <= n) S.fv[lane] = cost[lane - 1];
        if (lane == 0) S.evals += n;
        __syncwarp();
        return nm_iterate_warp(J, S, lane);
    }
    const double fr = cost[0], fe = cost[1], fc = cost[2];
    int evals = 1;
    int take = -1;  // 0 xr, 1 xe, 2 xc, 3 shrink
    if (fr < S.fv[0]) {
        evals += 1;
        take = fe < fr ? 1 : 0;
    } else if (fr < S.fv[n - 1]) {
        take = 0;
    } else {
        evals += 1;
        take = fc < S.fv[n] ? 2 : 3;
    }
    __syncwarp();
    if (lane == 0) S.evals += evals;
    if (take < 3) {
        if (lq) S.simplex[n][lane] = take == 0 ? S.xr[lane] : (take == 1 ? S.xe[lane] : S.xc[lane]);
        if (lane == 0) S.fv[n] = take == 0 ? fr : (take == 1 ? fe : fc);
        __syncwarp();
        return nm_iterate_warp(J, S, lane);
    }
    if (lq) {
        const int q = lane;
        const double s0 = S.simplex[0][q];
        for (int i = 1; i <= n; i++) {
            double v = __dadd_rn(s0, __dmul_rn(0.5, __dsub_rn(S.simplex[i][q], s0)));
            v = fmin(fmax(v, S.lo[q]), S.hi[q]);
            S.simplex[i][q] = v;
            S.pts[i - 1][q] = v;
        }
    }
    if (lane == 0) S.phase = NM_SHRINK;
    __syncwarp();
    return n;
}

// The bounded wait of the search's grid-wide hand-off (at least ~0.1 s of polling);
// LSB_NM_SPIN_LIMIT overrides it (tests shorten it to make the wait run out).
constexpr long long NM_SPIN_LIMIT = 1ll << 22;
static long long spin_limit() {
    if (const char* v = getenv("LSB_NM_SPIN_LIMIT")) return std::max(1ll, atoll(v));
    return NM_SPIN_LIMIT;
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

constexpr int NM_THREADS = 256, NM_WARPS = NM_THREADS / 32;
// align.rs:896 `multiscale_align` of one frame: the NmJob's whole coarse-to-fine search.
__global__ void __launch_bounds__(NM_THREADS) nm_search_kernel(const NmJob J) {
    __shared__ NmState S;
    __shared__ double cand[MAX_CAND][9];
    __shared__ double wred[MAX_CAND][3][NM_WARPS];
    __shared__ double gred[NM_THREADS];
    __shared__ double cost[MAX_CAND];
    __shared__ int pending;
    __shared__ int s_ok;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) {
        for (int q = 0; q < 8; q++) S.cur[q] = J.init_dev ? J.init_dev[q] : J.init[q];
        for (int q = 0; q < J.nfree; q++) {
            S.lo[q] = __dsub_rn(S.cur[J.free_idx[q]], c_span[J.free_idx[q]]);
            S.hi[q] = __dadd_rn(S.cur[J.free_idx[q]], c_span[J.free_idx[q]]);
        }
        S.evals = 0;
    }
    int batch = 0;
    unsigned arrived = 0;  // the counter's value once this batch's arrivals are in
    const unsigned stride = gridDim.x * NM_THREADS;
    for (int L = 0; L < J.nlv; L++) {
        const NmLevel lv = J.lv[L];
        __syncthreads();
        if (tid == 0) pending = J.nfree > 0 ? nm_level_start(J, S, L) : 0;
        __syncthreads();
        const double xmax = (double)(lv.w - 1), ymax = (double)(lv.h - 1);
        const unsigned npx = (unsigned)lv.w * lv.h;  // < 2^32 (the host checks)
        const int nown = (int)min((unsigned)gridDim.x, (npx + NM_THREADS - 1) / NM_THREADS);  // CTAs with pixels
        const bool own = (int)blockIdx.x < nown;
        const unsigned sdy = stride / (unsigned)lv.w, sdx = stride - sdy * (unsigned)lv.w;
        const unsigned i0 = blockIdx.x * NM_THREADS + tid;
        const int y0s = (int)(i0 / (unsigned)lv.w), x0s = (int)(i0 - (unsigned)y0s * lv.w);
        int passes = 0;
        while (pending > 0) {
            const int nc = pending;
            if (tid < nc) {
                double v[8], m[9];
                for (int q = 0; q < 8; q++) v[q] = S.snap[q];
                for (int q = 0; q < J.nfree; q++) v[J.free_idx[q]] = S.pts[tid][q];
                dev_sim_matrix(v, lv.w, lv.h, m);
                dev_mat_inverse(m, cand[tid]);
            }
            __syncthreads();
            // the batch's candidates three at a time in one pass over this block's pixels: the
            // reference value and the pixel's coordinates are shared, the three chains interleave
            for (int k0 = 0; k0 < nc; k0 += 3) {
                const int kn = min(3, nc - k0);
                double sd[3] = {0.0, 0.0, 0.0}, sd2[3] = {0.0, 0.0, 0.0};
                int cnt[3] = {0, 0, 0};
                bool aff[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const double* m = cand[k0 + min(c, kn - 1)];
                    aff[c] = m[6] == 0.0 && m[7] == 0.0 && m[8] == 1.0;
                }
                int x = x0s, y = y0s;
                for (unsigned i = i0; i < npx; i += stride) {
                    const float rv = lv.rf[i];
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        if (c < kn) {
                            double sx, sy;
                            src_point(cand[k0 + c], aff[c], (double)x, (double)y, sx, sy);
                            if (sx >= 0.0 && sx <= xmax && sy >= 0.0 && sy <= ymax) {
                                const double fx = floor(sx), fy = floor(sy);
                                const int xa = (int)fx, ya = (int)fy;
                                float wx[4], wy[4];
                                spline4f((float)__dsub_rn(sx, fx), wx);
                                spline4f((float)__dsub_rn(sy, fy), wy);
                                float acc = 0.f;
                                if (xa >= 1 && xa + 2 < lv.w && ya >= 1 && ya + 2 < lv.h) {
                                    // the 4x4 footprint inside the plane: no clamps
                                    const float* row = lv.tg + (size_t)(ya - 1) * lv.w + (xa - 1);
#pragma unroll
                                    for (int j = 0; j < 4; j++, row += lv.w) {
                                        float r = 0.f;
#pragma unroll
                                        for (int u = 0; u < 4; u++) r = __fadd_rn(r, __fmul_rn(wx[u], __ldg(row + u)));
                                        acc = __fadd_rn(acc, __fmul_rn(wy[j], r));
                                    }
                                } else {
#pragma unroll
                                    for (int j = 0; j < 4; j++) {
                                        const float* row = lv.tg + (size_t)min(max(ya + j - 1, 0), lv.h - 1) * lv.w;
                                        float r = 0.f;
#pragma unroll
                                        for (int u = 0; u < 4; u++) r = __fadd_rn(r, __fmul_rn(wx[u], __ldg(row + min(max(xa + u - 1, 0), lv.w - 1))));
                                        acc = __fadd_rn(acc, __fmul_rn(wy[j], r));
                                    }
                                }
                                const double d = (double)__fsub_rn(rv, acc);
                                sd[c] += d;
                                sd2[c] += d * d;
                                cnt[c]++;
                            }
                        }
                    }
                    x += (int)sdx;
                    y += (int)sdy;
                    if (x >= lv.w) {
                        x -= lv.w;
                        y++;
                    }
                }
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    if (c >= kn) break;
                    const double a = warp_sum(sd[c]), b = warp_sum(sd2[c]), n1 = warp_sum((double)cnt[c]);
                    if (lane == 0) {
                        wred[k0 + c][0][wid] = a;
                        wred[k0 + c][1][wid] = b;
                        wred[k0 + c][2][wid] = n1;
                    }
                }
            }
            __syncthreads();
            double* P = J.part + (size_t)(batch & 1) * MAX_CAND * gridDim.x * 3;
            if (own && tid < 3 * nc) {
                const int k = tid / 3, q = tid % 3;
                double s = 0.0;
                for (int w8 = 0; w8 < NM_WARPS; w8++) s += wred[k][q][w8];
                P[((size_t)k * 3 + q) * gridDim.x + blockIdx.x] = s;
            }
            // The hand-off: the CTAs with pixels arrive on a counter that only grows; every CTA
            // waits until this batch's arrivals are in, then sums the partials itself.
            arrived += (unsigned)nown;
            __syncthreads();
            if (tid == 0) {
                // the arrival releases this CTA's partials (written before the barrier above); the
                // wait acquires everyone's once the count is in: no fence, no returning atomic
                if (own) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(J.bar) : "memory");
                volatile int* verr = J.ctl;
                long long t = 0;
                int good = 1;
                for (;;) {
                    unsigned c;
                    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(c) : "l"(J.bar) : "memory");
                    if ((int)(c - arrived) >= 0) break;
                    if (*verr != 0 || ++t > J.spin_limit) {
                        good = 0;
                        break;
                    }
                    __nanosleep(32);
                }
                if (!good) atomicCAS(J.ctl, 0, 1);
                s_ok = good;
            }
            __syncthreads();
            if (!s_ok) return;
            // every CTA: each of the 3*nc sums over the CTAs with pixels, by gsz threads (thread r
            // takes CTAs r, r + gsz, ...), then the threads' sums in order: the same order in every copy
            {
                const int np = 3 * nc, gsz = NM_THREADS / np;
                const int pi = tid / gsz, r = tid - pi * gsz;
                double sv = 0.0;
                if (pi < np) {
                    // the first 12 partials loaded at once (one round of L2 latency), then added in
                    // the order of b, as the rest
                    const double* row = P + (size_t)pi * gridDim.x;
                    constexpr int PRE = 12;
                    double pv[PRE];
#pragma unroll
                    for (int u = 0; u < PRE; u++) pv[u] = r + u * gsz < nown ? __ldcg(row + r + u * gsz) : 0.0;
#pragma unroll
                    for (int u = 0; u < PRE; u++)
                        if (r + u * gsz < nown) sv += pv[u];
                    for (int b = r + PRE * gsz; b < nown; b += gsz) sv += __ldcg(row + b);
                }
                gred[tid] = sv;
                __syncthreads();
                if (tid < nc) {
                    double v3[3];
                    for (int q = 0; q < 3; q++) {
                        const double* g = gred + (size_t)(tid * 3 + q) * gsz;
                        double a = 0.0;
                        for (int i = 0; i < gsz; i++) a += g[i];
                        v3[q] = a;
                    }
                    const double sdv = v3[0], sd2v = v3[1], cn = v3[2];
                    cost[tid] = cn < 16.0 ? 1e9 : sqrt(fmax(__ddiv_rn(__dsub_rn(sd2v, __ddiv_rn(__dmul_rn(sdv, sdv), cn)), cn), 0.0));
                }
            }
            __syncthreads();
            if (wid == 0) {
                int nx = nm_advance_warp(J, S, cost, lane);
                // <= 200 iterations of at most two batches each, plus the first simplex
                if (lane == 0) {
                    if (++passes > 402 && nx > 0) {
                        nx = 0;
                        if (blockIdx.x == 0) atomicCAS(J.ctl, 0, 2);
                    }
                    pending = nx;
                }
            }
            batch++;
            __syncthreads();
        }
    }
    if (blockIdx.x == 0 && tid == 0) {
        for (int q = 0; q < 8; q++) J.out[q] = S.cur[q];
        J.ctl[1] = S.evals;
        if (J.evals_dev) atomicAdd(J.evals_dev, (unsigned long long)S.evals);
        if (J.warp_dev) {
            // align.rs:258: the inverse of the frame's matrix, as the warp of the next reference reads it
            const double id[8] = {0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 0.0};
            bool ident = true;
            for (int q = 0; q < 8; q++) ident = ident && S.cur[q] == id[q];
            double m[9], inv[9];
            dev_sim_matrix(S.cur, J.W, J.H, m);
            dev_mat_inverse(m, inv);
            for (int q = 0; q < 9; q++) J.warp_dev[q] = inv[q];
            J.warp_dev[9] = inv[6] == 0.0 && inv[7] == 0.0 && inv[8] == 1.0 ? 1.0 : 0.0;
            J.warp_dev[10] = ident ? 1.0 : 0.0;
        }
    }
}

static std::atomic<int> g_nm_blocks{0};  // the search's grid on this device (set once, by any thread)

// One frame's search job: the levels searched (coarsest first) and the free parameters.
static cudaError_t nm_job(AlignCtx& C, const float* rf, const std::vector<float*>& pr, const float* tg, const std::vector<float*>& pt,
                          int w, int h, const bool freem[8], int coarsen, NmJob& J) {
    std::vector<std::pair<int, int>> dims;
    gauss_dims(w, h, dims);
    const int n = (int)dims.size() + 1;
    const int finest = std::min(coarsen, n - 1);
    memset(&J, 0, sizeof J);
    for (int lvl = n - 1; lvl >= finest && J.nlv < 24; lvl--) {
        NmLevel& L = J.lv[J.nlv++];
        L.rf = lvl == 0 ? rf : pr[lvl - 1];
        L.tg = lvl == 0 ? tg : pt[lvl - 1];
        L.w = lvl == 0 ? w : dims[lvl - 1].first;
        L.h = lvl == 0 ? h : dims[lvl - 1].second;
        L.lvl = lvl;
    }
    if ((uint64_t)w * h >= (1ull << 31)) return cudaErrorInvalidValue;
    J.W = w;
    J.H = h;
    for (int q = 0; q < 8; q++)
        if (freem[q]) J.free_idx[J.nfree++] = q;
    if (g_nm_blocks.load() == 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, nm_search_kernel, NM_THREADS, 0);
        if (e != cudaSuccess) return e;
        if (per < 1) return cudaErrorCooperativeLaunchTooLarge;
        int want = 2;  // CTAs per SM: more warps hide the gathers, more CTAs make every barrier dearer
        if (const char* v = getenv("LSB_NM_CTAS_PER_SM")) want = std::max(1, atoi(v));
        g_nm_blocks.store(std::min(std::min(per, want) * sms, NM_MAX_BLOCKS));
    }
    J.spin_limit = spin_limit();
    J.part = C.nm_part;
    J.bar = (unsigned*)C.nm_ctl + 2;
    J.ctl = C.nm_ctl;
    J.out = C.nm_out;
    return cudaSuccess;
}
static cudaError_t nm_launch(AlignCtx& C, NmJob& J) {
    cudaError_t e = cudaMemsetAsync(C.nm_ctl + 2, 0, sizeof(int) * 2, C.s);  // the barrier; the error word stays sticky
    if (e != cudaSuccess) return e;
    void* args[] = {(void*)&J};
    lsb_launched();
    const int blocks = C.max_blocks > 0 ? std::min(g_nm_blocks.load(), C.max_blocks) : g_nm_blocks.load();
    return cudaLaunchCooperativeKernel((void*)nm_search_kernel, dim3(blocks), dim3(NM_THREADS), args, 0, C.s);
}

static cudaError_t multiscale_align_dev(AlignCtx& C, const float* rf, const std::vector<float*>& pr, const float* tg,
                                        const std::vector<float*>& pt, int w, int h, const double init[8], const bool freem[8],
                                        int coarsen, double out[8]) {
    NmJob J;
    cudaError_t e = nm_job(C, rf, pr, tg, pt, w, h, freem, coarsen, J);
    if (e != cudaSuccess) return e;
    for (int q = 0; q < 8; q++) J.init[q] = init[q];
    e = cudaMemsetAsync(C.nm_ctl, 0, sizeof(int) * 2, C.s);
    if (e == cudaSuccess) e = nm_launch(C, J);
    if (e != cudaSuccess) return e;
    cudaMemcpyAsync(C.sums_host, C.nm_out, sizeof(double) * 8, cudaMemcpyDeviceToHost, C.s);
    cudaMemcpyAsync(C.sums_host + 8, C.nm_ctl, sizeof(int) * 2, cudaMemcpyDeviceToHost, C.s);
    e = cudaStreamSynchronize(C.s);
    if (e != cudaSuccess) return e;
    int ctl[2];
    memcpy(ctl, C.sums_host + 8, sizeof ctl);
    if (ctl[0] != 0) return cudaErrorLaunchTimeout;  // a barrier wait or the batch limit ran out
    for (int q = 0; q < 8; q++) out[q] = C.sums_host[q];
    C.evals += ctl[1];
    C.launches++;
    return cudaSuccess;
}

cudaError_t align_chain_begin(AlignCtx& C, unsigned long long* evals_dev) {
    cudaError_t e = cudaMemsetAsync(C.nm_ctl, 0, sizeof(int) * 4, C.s);
    if (e == cudaSuccess) e = cudaMemsetAsync(evals_dev, 0, sizeof(unsigned long long), C.s);
    return e;
}
cudaError_t multiscale_align_chain(AlignCtx& C, const float* rf, const std::vector<float*>& pr, const float* tg,
                                   const std::vector<float*>& pt, int w, int h, const double* init_dev, const bool freem[8], int coarsen,
                                   double* out_dev, double* warp_dev, unsigned long long* evals_dev) {
    NmJob J;
    cudaError_t e = nm_job(C, rf, pr, tg, pt, w, h, freem, coarsen, J);
    if (e != cudaSuccess) return e;
    J.init_dev = init_dev;
    J.out = out_dev;
    J.warp_dev = warp_dev;
    J.evals_dev = evals_dev;
    C.launches++;
    return nm_launch(C, J);
}
cudaError_t align_chain_end(AlignCtx& C, const unsigned long long* evals_dev, size_t* evals) {
    int err = 0;
    unsigned long long ev = 0;
    cudaError_t e = cudaMemcpyAsync(&err, C.nm_ctl, sizeof err, cudaMemcpyDeviceToHost, C.s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ev, evals_dev, sizeof ev, cudaMemcpyDeviceToHost, C.s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(C.s);
    if (e != cudaSuccess) return e;
    if (err != 0) return cudaErrorLaunchTimeout;
    *evals = (size_t)ev;
    return cudaSuccess;
}

cudaError_t multiscale_align(AlignCtx& C, const float* rf, const std::vector<float*>& pr, const float* tg,
                             const std::vector<float*>& pt, int w, int h, const double init[8], const bool freem[8], int coarsen,
                             double out[8]) {
    if (C.device_search) return multiscale_align_dev(C, rf, pr, tg, pt, w, h, init, freem, coarsen, out);
    return multiscale_align_host(C, rf, pr, tg, pt, w, h, init, freem, coarsen, out);
}

// ------------------------------------------ the cost without any allocation
// Scratch of lsb_warp_cost_noalloc: the per-block partial sums (MAX_CAND
// candidates x NOALLOC_BLOCKS blocks x 3 doubles) and the reduced sums
// (MAX_CAND x 3): 64,152 bytes (62.6 KiB), held by every GPU that loads the library until
// the process exits. Each call writes every partial it later reads, so
// nothing has to start at zero; calls that overlap on the GPU race on it.
constexpr int NOALLOC_BLOCKS = 296;
constexpr size_t NOALLOC_PARTS = (size_t)MAX_CAND * NOALLOC_BLOCKS * 3;
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_PARTS + MAX_CAND * 3];

// The array's device address, looked up once per device with that device
// current (in host code its name is only a host-side stand-in).
static double* g_noalloc_dev[128];
static std::atomic<int> g_noalloc_ready[128];

static const char* noalloc_scratch(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return "lsb_warp_cost_noalloc: no current CUDA device";
    if (dev < 0 || dev >= 128) return "lsb_warp_cost_noalloc: device ordinal out of range";
    if (g_noalloc_ready[dev].load(std::memory_order_acquire) == 0) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr)
            return "lsb_warp_cost_noalloc: cudaGetSymbolAddress of the scratch failed";
        g_noalloc_dev[dev] = (double*)p;
        g_noalloc_ready[dev].store(1, std::memory_order_release);
    }
    *out = g_noalloc_dev[dev];
    return nullptr;
}

}  // namespace lsb

using namespace lsb;

// align.rs:581 warp_cost of device planes for up to MAX_CAND transforms, using
// only the static scratch above. The error string, when one is returned, is
// static: do not free it.
extern "C" const char* lsb_warp_cost_noalloc(const float* rf_dev, uint32_t aw, uint32_t ah, const float* tgt_dev, uint32_t tw,
                                             uint32_t th, const double* sims8, uint32_t n_sims, double* costs, void* stream) {
    if (!rf_dev || !tgt_dev || !sims8 || !costs) return "lsb_warp_cost_noalloc: null argument";
    if (aw == 0 || ah == 0 || tw == 0 || th == 0) return "lsb_warp_cost_noalloc: empty plane";
    // the limits of the other entry points: the kernels index planes with 32-bit ints
    for (const uint32_t* d : {&aw, &ah, &tw, &th})
        if (*d > 65535u) return "lsb_warp_cost_noalloc: width and height must be at most 65535";
    if ((uint64_t)aw * ah * 3 > 0x7fffffffull || (uint64_t)tw * th * 3 > 0x7fffffffull)
        return "lsb_warp_cost_noalloc: at most 715 Mpx per plane (3 w h must fit 31 bits)";
    if (n_sims == 0 || n_sims > (uint32_t)MAX_CAND) return "lsb_warp_cost_noalloc: 1 to 9 transforms per call";
    double* scratch = nullptr;
    if (const char* e = noalloc_scratch(&scratch)) return e;
    cudaStream_t s = (cudaStream_t)stream;
    CostBatch cb;
    for (uint32_t k = 0; k < n_sims; k++) {
        double m[9];
        sim_matrix(sims8 + 8 * k, (int)tw, (int)th, m);
        mat_inverse(m, cb.inv[k]);
    }
    const size_t npx = (size_t)aw * ah;
    const int nblocks = (int)std::min<size_t>(std::max<size_t>((npx + 255) / 256, 1), NOALLOC_BLOCKS);
    dim3 g(nblocks, n_sims);
    lsb_launched(), cost_kernel<<<g, 256, 0, s>>>(rf_dev, (int)aw, (int)ah, tgt_dev, (int)tw, (int)th, cb, scratch);
    lsb_launched(), cost_final_kernel<<<n_sims, 128, 0, s>>>(scratch, nblocks, (int)n_sims, scratch + NOALLOC_PARTS);
    double sums[MAX_CAND * 3];
    if (cudaMemcpyAsync(sums, scratch + NOALLOC_PARTS, sizeof(double) * 3 * n_sims, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return "lsb_warp_cost_noalloc: the cost kernels failed";
    for (uint32_t k = 0; k < n_sims; k++) {
        const double sd = sums[3 * k], sd2 = sums[3 * k + 1], cnt = sums[3 * k + 2];
        costs[k] = cnt < 16.0 ? 1e9 : std::sqrt(std::max((sd2 - sd * sd / cnt) / cnt, 0.0));
    }
    return nullptr;
}
