// The depth-from-focus pass (crates/lapstack-core/src/depth.rs:1119
// `depth_from_slices`) on the device.
//
// * The guided-filter aggregation of every slice (depth.rs:352 GuidedFilter,
//   r = agg_radius) and the streamed peak tracker (depth.rs:533 PeakTracker)
//   run as ONE persistent kernel: a CTA owns a tile of the working grid, keeps
//   the guide's statistics for it in shared memory, walks the N slices in
//   order and keeps every cell's profile state in registers, so a slice is read
//   from HBM once (plus its halo) and the tracker state never round-trips.
// * Box sums follow depth.rs:285 `BoxFilter::sum_into`: border-clipped, f64
//   sums rounded to f32 after the horizontal and after the vertical pass; at
//   radii 3 and 8 the window sums are moving f64 sums along short runs, at
//   other radii direct sums of 2R+1 taps (both equal to the reference's f64
//   running sums whenever those are exact, which they are unless a window's
//   values span more than about 2^24 in magnitude).
// * The two medians of a subsample (noise floor depth.rs:578, p90
//   depth.rs:616) are exact k-th-value selections on the device (two 16-bit
//   radix passes over the total-order key of each float).
#include <algorithm>

#include "lsb_common.cuh"
#include "lsb_depth.h"

namespace lsb {

// ------------------------------------------------------------------ helpers
__global__ void luma_kernel(const float* __restrict__ img, float* __restrict__ y, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = lsb_luma(img[i], img[n + i], img[2 * n + i]);
}

// depth.rs:174 `block_mean`: per row of the block the row sum, added in order, then / count.
__global__ void block_mean_kernel(const float* __restrict__ src, int w, int h, int k, float* __restrict__ out, int dw, int dh) {
    const int ox = blockIdx.x * blockDim.x + threadIdx.x, oy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ox >= dw || oy >= dh) return;
    const int x0 = ox * k, x1 = min(x0 + k, w), y0 = oy * k, y1 = min(y0 + k, h);
    float o = 0.f;
    for (int y = y0; y < y1; y++) {
        float rs = 0.f;
        for (int x = x0; x < x1; x++) rs = __fadd_rn(rs, src[(size_t)y * w + x]);
        o = __fadd_rn(o, rs);
    }
    out[(size_t)oy * dw + ox] = __fdiv_rn(o, (float)((y1 - y0) * (x1 - x0)));
}

__device__ __forceinline__ float box_inv_count(int x, int y, int w, int h, int r) {
    const float cy = (float)(min(y + r + 1, h) - max(y - r, 0));
    const float cx = (float)(min(x + r + 1, w) - max(x - r, 0));
    return __fdiv_rn(1.f, __fmul_rn(cy, cx));
}

// depth.rs:285 `BoxFilter::sum_into`, horizontal pass: box sums (optionally of a*b), f64 window sum rounded to f32.
__global__ void box_h_kernel(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ out, int w, int h, int r) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    const float* ra = a + (size_t)y * w;
    const float* rb = b ? b + (size_t)y * w : nullptr;
    double s = 0.0;
    for (int t = max(x - r, 0); t <= min(x + r, w - 1); t++) s += rb ? (double)__fmul_rn(ra[t], rb[t]) : (double)ra[t];
    out[(size_t)y * w + x] = (float)s;
}
// depth.rs:285/337 `BoxFilter::sum_into` / `mean_into`, vertical pass: box sums of the horizontal sums, rounded to f32, times the inverse count.
__global__ void box_v_kernel(const float* __restrict__ hs, float* __restrict__ out, int w, int h, int r) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    double s = 0.0;
    for (int t = max(y - r, 0); t <= min(y + r, h - 1); t++) s += (double)hs[(size_t)t * w + x];
    out[(size_t)y * w + x] = __fmul_rn((float)s, box_inv_count(x, y, w, h, r));
}

static void box_mean(const float* a, const float* b, float* tmp, float* out, int w, int h, int r, cudaStream_t s) {
    dim3 blk(128), g((w + 127) / 128, h);
    lsb_launched(), box_h_kernel<<<g, blk, 0, s>>>(a, b, tmp, w, h, r);
    lsb_launched(), box_v_kernel<<<g, blk, 0, s>>>(tmp, out, w, h, r);
}

// depth.rs:363 GuidedFilter::new: var_i = max(mean(I*I) - mean_i^2, 0)
__global__ void gf_var_kernel(const float* __restrict__ mean_i, float* __restrict__ var_i, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        var_i[i] = fmaxf(__fsub_rn(var_i[i], __fmul_rn(mean_i[i], mean_i[i])), 0.f);
}
// depth.rs:385: a = (corr - mean_i * mean_p) / (var_i + eps), b = mean_p - a * mean_i
// b may be the corr buffer itself (gf_coeffs writes b over corr_Ip in place), so neither is __restrict__.
__global__ void gf_ab_kernel(const float* __restrict__ mp, const float* corr, const float* __restrict__ mi,
                             const float* __restrict__ vi, float eps, float* __restrict__ a, float* b, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float av = __fdiv_rn(__fsub_rn(corr[i], __fmul_rn(mi[i], mp[i])), __fadd_rn(vi[i], eps));
        a[i] = av;
        b[i] = __fsub_rn(mp[i], __fmul_rn(av, mi[i]));
    }
}

static int grid1(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

void box_mean_plane(const float* src, float* tmp, float* out, int w, int h, int r, cudaStream_t s) { box_mean(src, nullptr, tmp, out, w, h, r, s); }

void gf_stats(const float* guide, int w, int h, int r, float* tmp, float* mean_i, float* var_i, cudaStream_t s) {
    box_mean(guide, nullptr, tmp, mean_i, w, h, r, s);
    box_mean(guide, guide, tmp, var_i, w, h, r, s);
    lsb_launched(), gf_var_kernel<<<grid1((size_t)w * h), 256, 0, s>>>(mean_i, var_i, (size_t)w * h);
}

// depth.rs:379 `coeffs_into` for one plane p: a-bar into abar, b-bar into bbar.
void gf_coeffs(const float* guide, const float* mean_i, const float* var_i, const float* p, int w, int h, int r, float eps,
               float* t0, float* t1, float* t2, float* tmp, float* abar, float* bbar, cudaStream_t s) {
    size_t n = (size_t)w * h;
    box_mean(p, nullptr, tmp, t0, w, h, r, s);    // mean_p
    box_mean(guide, p, tmp, t1, w, h, r, s);      // corr_Ip (I*p formed inside)
    lsb_launched(), gf_ab_kernel<<<grid1(n), 256, 0, s>>>(t0, t1, mean_i, var_i, eps, t2, t1, n);  // a -> t2, b -> t1
    box_mean(t2, nullptr, tmp, abar, w, h, r, s);
    box_mean(t1, nullptr, tmp, bbar, w, h, r, s);
}

// --------------------------------------------- fused aggregation + peaks
struct PeakState {
    float c1, l1, r1, c2, prev, prev2, sum, cmin;
    int i1;
};
__device__ __forceinline__ void peak_reg(PeakState& p, float val, int idx, float l, float r) {
    if (val > p.c1) {
        if (p.c1 >= 0.f) p.c2 = p.c1;
        p.c1 = val;
        p.i1 = idx;
        p.l1 = l;
        p.r1 = r;
    } else if (val > p.c2) {
        p.c2 = val;
    }
}
// depth.rs:547 `push` of slice m
__device__ __forceinline__ void peak_push(PeakState& p, float v, int m) {
    if (m >= 1) {
        const bool is_peak = (m == 1 || p.prev >= p.prev2) && p.prev > v;
        if (is_peak) peak_reg(p, p.prev, m - 1, m >= 2 ? p.prev2 : -1.f, v);
    }
    p.sum = __fadd_rn(p.sum, v);
    p.cmin = fminf(p.cmin, v);
    p.prev2 = p.prev;
    p.prev = v;
}

// depth.rs:1119 `depth_from_slices`: each focus slice's guided-filter aggregation (depth.rs:401
// `GuidedFilter::filter_into`) fed straight to the peak tracker (depth.rs:547 `PeakTracker::push`).
// RT: the aggregation radius as a compile-time constant (0: a.r at run time).
// Tiles whose windows stay inside the grid take fixed, unrolled 2R+1-tap
// windows; border tiles clip them as BoxFilter does.
template <int TWD, int THD, class SS, int RT>
__global__ void __launch_bounds__(256, 2) aggregate_kernel(const AggArgs a) {
    constexpr int CPT = TWD * THD / 256;
    extern __shared__ float sm[];
    const int R = RT > 0 ? RT : a.r, w = a.dw, h = a.dh, tid = threadIdx.x;
    const int PW = TWD + 4 * R, PH = THD + 4 * R, QW = TWD + 2 * R, QH = THD + 2 * R;
    constexpr int NW = 2 * RT + 1;  // window taps when RT > 0
    constexpr int KS = RT <= 4 ? 8 : 4;  // interior tiles: outputs per thread in a window pass
    float* P = sm;                 // [PH][PW] slice over tile +- 2R
    float* I = P + PW * PH;        // [PH][PW] guide
    float* MI = I + PW * PH;       // [QH][QW] mean_i
    float* VI = MI + QW * QH;      // [QH][QW] var_i
    float* HP = VI + QW * QH;      // [PH][QW] horizontal sums of p, then of a
    float* HQ = HP + PH * QW;      // [PH][QW] horizontal sums of I*p, then of b
    float* A = HQ + PH * QW;       // [QH][QW]
    float* B = A + QW * QH;        // [QH][QW]
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const int x0 = (tile % a.tiles_x) * TWD, y0 = (tile / a.tiles_x) * THD;
        const int px0 = x0 - 2 * R, py0 = y0 - 2 * R, qx0 = x0 - R, qy0 = y0 - R;
        const bool inner = RT > 0 && px0 >= 0 && py0 >= 0 && px0 + PW <= w && py0 + PH <= h;
        const float ic_in = box_inv_count(R, R, 4 * R + 1, 4 * R + 1, R);  // the interior's 1 / (2R+1)^2
        for (int i = tid; i < PW * PH; i += 256) {
            const int x = px0 + i % PW, y = py0 + i / PW;
            I[i] = (x >= 0 && x < w && y >= 0 && y < h) ? a.guide[(size_t)y * w + x] : 0.f;
        }
        for (int i = tid; i < QW * QH; i += 256) {
            const int x = qx0 + i % QW, y = qy0 + i / QW;
            const bool in = x >= 0 && x < w && y >= 0 && y < h;
            MI[i] = in ? a.mean_i[(size_t)y * w + x] : 0.f;
            VI[i] = in ? a.var_i[(size_t)y * w + x] : 0.f;
        }
        PeakState st[CPT];
#pragma unroll
        for (int j = 0; j < CPT; j++) st[j] = PeakState{-1.f, -1.f, -1.f, -1.f, 0.f, 0.f, 0.f, __int_as_float(0x7f800000), 0};
        for (int m = 0; m < a.n; m++) {
            const SS* sl = (const SS*)a.slices + (size_t)m * w * h;
            __syncthreads();
            if (inner) {
                for (int i = tid; i < PW * PH; i += 256) P[i] = lsb_ld<SS>(sl + (size_t)(py0 + i / PW) * w + px0 + i % PW);
            } else {
                for (int i = tid; i < PW * PH; i += 256) {
                    const int x = px0 + i % PW, y = py0 + i / PW;
                    P[i] = (x >= 0 && x < w && y >= 0 && y < h) ? lsb_ld<SS>(sl + (size_t)y * w + x) : 0.f;
                }
            }
            __syncthreads();
            // horizontal sums of p and I*p over rows of tile +- 2R, columns of tile +- R
            if (inner) {
                // a strip of KS outputs per thread: each input converted to f64 once, each
                // output's window summed from zero in tap order
                constexpr int NV = KS + 2 * RT;
                const int nst = (QW + KS - 1) / KS;
                for (int it = tid; it < PH * nst; it += 256) {
                    const int r = it / nst, c0 = (it - r * nst) * KS;
                    const float* pr = P + r * PW + c0;
                    const float* ir = I + r * PW + c0;
                    double v[NV];
#pragma unroll
                    for (int t = 0; t < NV; t++) v[t] = c0 + t < PW ? (double)pr[t] : 0.0;
#pragma unroll
                    for (int k = 0; k < KS; k++)
                        if (c0 + k < QW) {
                            double sp = 0.0;
#pragma unroll
                            for (int t = 0; t < NW; t++) sp += v[k + t];
                            HP[r * QW + c0 + k] = (float)sp;
                        }
#pragma unroll
                    for (int t = 0; t < NV; t++) v[t] = c0 + t < PW ? (double)__fmul_rn(ir[t], pr[t]) : 0.0;
#pragma unroll
                    for (int k = 0; k < KS; k++)
                        if (c0 + k < QW) {
                            double sq = 0.0;
#pragma unroll
                            for (int t = 0; t < NW; t++) sq += v[k + t];
                            HQ[r * QW + c0 + k] = (float)sq;
                        }
                }
            } else
            for (int i = tid; i < PH * QW; i += 256) {
                const int r = i / QW, c = i % QW, x = qx0 + c;
                double sp = 0.0, sq = 0.0;
                {
                    const int lo = max(x - R, 0) - px0, hi = min(x + R, w - 1) - px0;
                    for (int t = lo; t <= hi; t++) {
                        const float pv = P[r * PW + t];
                        sp += (double)pv;
                        sq += (double)__fmul_rn(I[r * PW + t], pv);
                    }
                }
                HP[i] = (float)sp;
                HQ[i] = (float)sq;
            }
            __syncthreads();
            // vertical: mean_p, corr_Ip -> a, b over tile +- R
            if (inner) {
                constexpr int NV = KS + 2 * RT;
                const int nst = (QH + KS - 1) / KS;
                for (int it = tid; it < QW * nst; it += 256) {
                    const int c = it % QW, r0 = (it / QW) * KS;
                    double v[NV];
                    float sps[KS];  // the sums as f32, as the reference rounds them
#pragma unroll
                    for (int t = 0; t < NV; t++) v[t] = r0 + t < PH ? (double)HP[(r0 + t) * QW + c] : 0.0;
#pragma unroll
                    for (int k = 0; k < KS; k++) {
                        double sp = 0.0;
#pragma unroll
                        for (int t = 0; t < NW; t++) sp += v[k + t];
                        sps[k] = (float)sp;
                    }
#pragma unroll
                    for (int t = 0; t < NV; t++) v[t] = r0 + t < PH ? (double)HQ[(r0 + t) * QW + c] : 0.0;
#pragma unroll
                    for (int k = 0; k < KS; k++) {
                        const int r = r0 + k;
                        if (r >= QH) break;
                        double sq = 0.0;
#pragma unroll
                        for (int t = 0; t < NW; t++) sq += v[k + t];
                        const int i = r * QW + c;
                        const float mp = __fmul_rn(sps[k], ic_in), corr = __fmul_rn((float)sq, ic_in);
                        const float av = __fdiv_rn(__fsub_rn(corr, __fmul_rn(MI[i], mp)), __fadd_rn(VI[i], a.eps));
                        A[i] = av;
                        B[i] = __fsub_rn(mp, __fmul_rn(av, MI[i]));
                    }
                }
            } else
            for (int i = tid; i < QW * QH; i += 256) {
                const int r = i / QW, c = i % QW, x = qx0 + c, y = qy0 + r;
                if (!inner && (x < 0 || x >= w || y < 0 || y >= h)) {
                    A[i] = 0.f;
                    B[i] = 0.f;
                    continue;
                }
                double sp = 0.0, sq = 0.0;
                float ic;
                if (inner) {
#pragma unroll
                    for (int t = 0; t < NW; t++) {
                        sp += (double)HP[(r + t) * QW + c];
                        sq += (double)HQ[(r + t) * QW + c];
                    }
                    ic = ic_in;
                } else {
                    const int lo = max(y - R, 0) - py0, hi = min(y + R, h - 1) - py0;
                    for (int t = lo; t <= hi; t++) {
                        sp += (double)HP[t * QW + c];
                        sq += (double)HQ[t * QW + c];
                    }
                    ic = box_inv_count(x, y, w, h, R);
                }
                const float mp = __fmul_rn((float)sp, ic), corr = __fmul_rn((float)sq, ic);
                const float av = __fdiv_rn(__fsub_rn(corr, __fmul_rn(MI[i], mp)), __fadd_rn(VI[i], a.eps));
                A[i] = av;
                B[i] = __fsub_rn(mp, __fmul_rn(av, MI[i]));
            }
            __syncthreads();
            // horizontal sums of a and b over rows of tile +- R, the tile's columns
            if (inner) {
                constexpr int NV = KS + 2 * RT;
                constexpr int nst = TWD / KS;
                for (int it = tid; it < QH * nst; it += 256) {
                    const int r = it / nst, c0 = (it - r * nst) * KS;
                    const float* ar = A + r * QW + c0;
                    const float* br = B + r * QW + c0;
                    double v[NV];
#pragma unroll
                    for (int t = 0; t < NV; t++) v[t] = (double)ar[t];
#pragma unroll
                    for (int k = 0; k < KS; k++) {
                        double sa = 0.0;
#pragma unroll
                        for (int t = 0; t < NW; t++) sa += v[k + t];
                        HP[r * TWD + c0 + k] = (float)sa;
                    }
#pragma unroll
                    for (int t = 0; t < NV; t++) v[t] = (double)br[t];
#pragma unroll
                    for (int k = 0; k < KS; k++) {
                        double sb = 0.0;
#pragma unroll
                        for (int t = 0; t < NW; t++) sb += v[k + t];
                        HQ[r * TWD + c0 + k] = (float)sb;
                    }
                }
            } else
            for (int i = tid; i < QH * TWD; i += 256) {
                const int r = i / TWD, c = i % TWD, x = x0 + c;
                if (!inner && x >= w) continue;
                double sa = 0.0, sb = 0.0;
                if (inner) {
#pragma unroll
                    for (int t = 0; t < NW; t++) {
                        sa += (double)A[r * QW + c + t];
                        sb += (double)B[r * QW + c + t];
                    }
                } else {
                    const int lo = max(x - R, 0) - qx0, hi = min(x + R, w - 1) - qx0;
                    for (int t = lo; t <= hi; t++) {
                        sa += (double)A[r * QW + t];
                        sb += (double)B[r * QW + t];
                    }
                }
                HP[i] = (float)sa;
                HQ[i] = (float)sb;
            }
            __syncthreads();
            if (inner) {
                // the thread's CPT cells: column tid % TWD, rows (tid / TWD) * CPT + 0 .. CPT-1
                constexpr int NV = CPT + 2 * RT;
                const int c = tid % TWD, r0 = (tid / TWD) * CPT;
                double v[NV];
                float sas[CPT];
#pragma unroll
                for (int t = 0; t < NV; t++) v[t] = (double)HP[(r0 + t) * TWD + c];
#pragma unroll
                for (int k = 0; k < CPT; k++) {
                    double sa = 0.0;
#pragma unroll
                    for (int t = 0; t < NW; t++) sa += v[k + t];
                    sas[k] = (float)sa;
                }
#pragma unroll
                for (int t = 0; t < NV; t++) v[t] = (double)HQ[(r0 + t) * TWD + c];
#pragma unroll
                for (int k = 0; k < CPT; k++) {
                    double sb = 0.0;
#pragma unroll
                    for (int t = 0; t < NW; t++) sb += v[k + t];
                    const float abar = __fmul_rn(sas[k], ic_in), bbar = __fmul_rn((float)sb, ic_in);
                    const float q = fmaxf(__fadd_rn(__fmul_rn(abar, I[(r0 + k + 2 * R) * PW + c + 2 * R]), bbar), 0.f);
                    peak_push(st[k], q, m);
                }
                continue;
            }
#pragma unroll
            for (int j = 0; j < CPT; j++) {
                const int p = tid + 256 * j, c = p % TWD, r = p / TWD, x = x0 + c, y = y0 + r;
                if (!inner && (x >= w || y >= h)) continue;
                double sa = 0.0, sb = 0.0;
                float ic;
                if (inner) {
#pragma unroll
                    for (int t = 0; t < NW; t++) {
                        sa += (double)HP[(r + t) * TWD + c];
                        sb += (double)HQ[(r + t) * TWD + c];
                    }
                    ic = ic_in;
                } else {
                    const int lo = max(y - R, 0) - qy0, hi = min(y + R, h - 1) - qy0;
                    for (int t = lo; t <= hi; t++) {
                        sa += (double)HP[t * TWD + c];
                        sb += (double)HQ[t * TWD + c];
                    }
                    ic = box_inv_count(x, y, w, h, R);
                }
                const float abar = __fmul_rn((float)sa, ic), bbar = __fmul_rn((float)sb, ic);
                // depth.rs:404 q = a-bar * I + b-bar, then depth.rs:1146 max(q, 0)
                const float q = fmaxf(__fadd_rn(__fmul_rn(abar, I[(r + 2 * R) * PW + c + 2 * R]), bbar), 0.f);
                peak_push(st[j], q, m);
            }
        }
#pragma unroll
        for (int j = 0; j < CPT; j++) {
            const int p = tid + 256 * j;
            const int c = inner ? tid % TWD : p % TWD, r = inner ? (tid / TWD) * CPT + j : p / TWD, x = x0 + c, y = y0 + r;
            if (x >= w || y >= h) continue;
            const size_t o = (size_t)y * w + x, m = (size_t)w * h;
            float* S = a.state;
            S[o] = st[j].c1;
            S[m + o] = st[j].l1;
            S[2 * m + o] = st[j].r1;
            S[3 * m + o] = st[j].c2;
            S[4 * m + o] = st[j].prev;
            S[5 * m + o] = st[j].prev2;
            S[6 * m + o] = st[j].sum;
            S[7 * m + o] = st[j].cmin;
            S[8 * m + o] = __int_as_float(st[j].i1);
        }
        __syncthreads();
    }
}

// --------------------------- aggregation by moving sums, one slice ahead
// 16-byte global -> shared copies (cp.async.cg), zero-filled where the source lies outside the grid
__device__ __forceinline__ void agg_cp16(void* sdst, const void* gsrc, bool in) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gsrc), "r"(in ? 16 : 0));
}
__device__ __forceinline__ void agg_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void agg_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }
template <class S>
__device__ __forceinline__ float agg_f(S v);
template <>
__device__ __forceinline__ float agg_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ float agg_f<__half>(__half v) { return __half2float(v); }
template <class S>
__device__ __forceinline__ S agg_zero();
template <>
__device__ __forceinline__ float agg_zero<float>() { return 0.f; }
template <>
__device__ __forceinline__ __half agg_zero<__half>() { return __ushort_as_half((unsigned short)0); }

// Run length of a pass over `lines` lines of `len` outputs, so that the lines' runs fit 256 threads once.
__host__ __device__ constexpr int agg_run(int lines, int len) {
    return (len + (256 / lines > 0 ? 256 / lines : 1) - 1) / (256 / lines > 0 ? 256 / lines : 1);
}

// One step of a moving window sum of NW = 2R+1 values along a run (t: the entering value's
// index): the first window is summed as two interleaved partial sums, then each step adds the
// entering value less the leaving one. Every partial sum of up to 18 f32 values is exact in f64
// unless their magnitudes span more than about 2^24, so the window sum is then the exact sum,
// whatever the order of the adds, as the reference's moving sums give it while they are exact.
template <int R, int NV>
__device__ __forceinline__ void agg_step_t(double& s, double& s2, const double (&v)[NV], int t) {
    if (t < 2 * R) {
        if (t & 1) s2 += v[t];
        else s += v[t];
    } else if (t == 2 * R) {
        s = (s + s2) + v[t];
    } else {
        s += v[t] - v[t - 2 * R - 1];
    }
}
#define agg_step(s, s2, v, t) agg_step_t<R>(s, s2, v, t)

// depth.rs:1119 `depth_from_slices` over tiles of TW x TH cells, with the window sums of the
// guided filter (depth.rs:379-406) formed as depth.rs:285 `BoxFilter::sum_into` forms them:
// moving f64 sums along runs of a line (the entering value added, then the leaving one subtracted),
// rounded to f32 after the horizontal and after the vertical pass. A run converts each input to
// f64 once and keeps it in a register until it leaves the window. The sums are the reference's
// whenever its f64 sums are exact (true unless a window's values span more than about 2^24).
// A CTA stages slice m+1's window (tile +- 2R) by cp.async while it filters slice m; the
// window is zero outside the grid, so the sums there equal BoxFilter's border-clipped ones,
// and a (a, b) outside the grid is zero. Each thread keeps the peak tracker (depth.rs:547) of
// CPT cells of one column in registers.
template <int R, int TW, int TH, class SS, int MINB>
__global__ void __launch_bounds__(256, MINB) guided_peaks_kernel(const AggArgs a) {
    constexpr int NT = 256, CPT = TW * TH / NT;
    constexpr int PW = TW + 4 * R, PH = TH + 4 * R, QW = TW + 2 * R, QH = TH + 2 * R;
    constexpr int CE = 16 / (int)sizeof(SS);            // elements of one 16-byte copy
    constexpr int LEAD = (2 * R + CE - 1) / CE * CE;    // staged columns left of the tile
    constexpr int T0 = LEAD - 2 * R;                    // the window's first column in a staged row
    constexpr int PS = (T0 + PW + CE - 1) / CE * CE;    // staged row length
    constexpr int NCH = PS / CE;
    constexpr int PWI = PW | 1;                         // guide row pitch
    constexpr int L1 = agg_run(PH, QW), NS1 = (QW + L1 - 1) / L1;  // horizontal runs of p and I*p
    constexpr int L2 = agg_run(QW, QH), NS2 = (QH + L2 - 1) / L2;  // vertical runs -> a, b
    constexpr int L3 = agg_run(QH, TW), NS3 = (TW + L3 - 1) / L3;  // horizontal runs of a and b
    static_assert(TW % CE == 0 && CPT * NT == TW * TH, "tile");
    extern __shared__ __align__(16) unsigned char agg_sm[];
    SS* P0 = (SS*)agg_sm;                                           // [2][PH][PS] slice windows
    float* I = (float*)(agg_sm + sizeof(SS) * 2 * PH * PS);         // [PH][PWI] guide
    float* MI = I + PH * PWI;                                       // [QH][QW] mean_i
    float* VE = MI + QH * QW;                                       // [QH][QW] var_i + eps
    float* HP = VE + QH * QW;                                       // [PH][QW] sums of p; then [QH][TW] of a
    float* HQ = HP + PH * QW;                                       // [PH][QW] sums of I*p; then [QH][TW] of b
    float* A = HQ + PH * QW;                                        // [QH][QW]
    float* B = A + QH * QW;                                         // [QH][QW]
    const int w = a.dw, h = a.dh, tid = threadIdx.x;
    const float ic_in = box_inv_count(R, R, 4 * R + 1, 4 * R + 1, R);  // 1 / (2R+1)^2
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const int x0 = (tile % a.tiles_x) * TW, y0 = (tile / a.tiles_x) * TH;
        const int px0 = x0 - 2 * R, py0 = y0 - 2 * R, qx0 = x0 - R, qy0 = y0 - R, xs0 = x0 - LEAD;
        const bool inner = px0 >= 0 && py0 >= 0 && px0 + PW <= w && py0 + PH <= h;
        auto stage = [&](int m, SS* buf) {
            const SS* sl = (const SS*)a.slices + (size_t)m * w * h;
            if (a.async16) {
                // xs0 and the copies are CE-aligned and w % CE == 0: a copy lies wholly inside or outside
                for (int i = tid; i < PH * NCH; i += NT) {
                    const int r = i / NCH, k = i - r * NCH, y = py0 + r, x = xs0 + k * CE;
                    const bool in = y >= 0 && y < h && x >= 0 && x < w;
                    agg_cp16(buf + r * PS + k * CE, in ? (const void*)(sl + (size_t)y * w + x) : a.slices, in);
                }
                agg_commit();
            } else {
                for (int i = tid; i < PH * PS; i += NT) {
                    const int r = i / PS, t = i - r * PS, y = py0 + r, x = xs0 + t;
                    buf[i] = (y >= 0 && y < h && x >= 0 && x < w) ? sl[(size_t)y * w + x] : agg_zero<SS>();
                }
            }
        };
        __syncthreads();  // the previous tile is done with every buffer
        stage(0, P0);
        for (int i = tid; i < PH * PW; i += NT) {
            const int r = i / PW, c = i - r * PW, x = px0 + c, y = py0 + r;
            I[r * PWI + c] = (x >= 0 && x < w && y >= 0 && y < h) ? a.guide[(size_t)y * w + x] : 0.f;
        }
        for (int i = tid; i < QW * QH; i += NT) {
            const int x = qx0 + i % QW, y = qy0 + i / QW;
            const bool in = x >= 0 && x < w && y >= 0 && y < h;
            MI[i] = in ? a.mean_i[(size_t)y * w + x] : 0.f;
            VE[i] = in ? __fadd_rn(a.var_i[(size_t)y * w + x], a.eps) : 1.f;
        }
        PeakState st[CPT];
#pragma unroll
        for (int j = 0; j < CPT; j++) st[j] = PeakState{-1.f, -1.f, -1.f, -1.f, 0.f, 0.f, 0.f, __int_as_float(0x7f800000), 0};
        const int vc = tid % TW, vr0 = (tid / TW) * CPT;  // this thread's cells: column vc, rows vr0 ..
        for (int m = 0; m < a.n; m++) {
            const SS* P = P0 + (m & 1) * PH * PS;
            if (a.async16) agg_wait_all();
            __syncthreads();  // slice m staged; the last pass of slice m-1 is done with HP and HQ
            if (m + 1 < a.n) stage(m + 1, P0 + ((m + 1) & 1) * PH * PS);
            // horizontal runs: sums of p and of I*p over rows of tile +- 2R, columns of tile +- R
            for (int it = tid; it < PH * NS1; it += NT) {
                const int r = it / NS1, c0 = (it - r * NS1) * L1;
                const SS* pr = P + r * PS + T0 + c0;
                const float* ir = I + r * PWI + c0;
                float* hp = HP + r * QW + c0;
                float* hq = HQ + r * QW + c0;
                double vp[L1 + 2 * R], vq[L1 + 2 * R], sp = 0.0, sp2 = 0.0, sq = 0.0, sq2 = 0.0;
#pragma unroll
                for (int t = 0; t < L1 + 2 * R; t++) {
                    if (QW % L1 != 0 && c0 + t - 2 * R >= QW) break;
                    const float pv = agg_f<SS>(pr[t]);
                    vp[t] = (double)pv;
                    vq[t] = (double)__fmul_rn(ir[t], pv);
                    agg_step(sp, sp2, vp, t);
                    agg_step(sq, sq2, vq, t);
                    if (t >= 2 * R) {
                        hp[t - 2 * R] = (float)sp;
                        hq[t - 2 * R] = (float)sq;
                    }
                }
            }
            __syncthreads();
            // vertical runs: mean_p and corr_Ip over tile +- R, then a and b (depth.rs:385-390)
            for (int it = tid; it < QW * NS2; it += NT) {
                const int j = it / QW, c = it - j * QW, r0 = j * L2;
                const float* hp = HP + r0 * QW + c;
                const float* hq = HQ + r0 * QW + c;
                double vp[L2 + 2 * R], vq[L2 + 2 * R], sp = 0.0, sp2 = 0.0, sq = 0.0, sq2 = 0.0;
#pragma unroll
                for (int t = 0; t < L2 + 2 * R; t++) {
                    if (QH % L2 != 0 && r0 + t - 2 * R >= QH) break;
                    vp[t] = (double)hp[t * QW];
                    vq[t] = (double)hq[t * QW];
                    agg_step(sp, sp2, vp, t);
                    agg_step(sq, sq2, vq, t);
                    if (t >= 2 * R) {
                        const int k = t - 2 * R, i = (r0 + k) * QW + c;
                        float ic = ic_in;
                        bool in = true;
                        if (!inner) {
                            const int x = qx0 + c, y = qy0 + r0 + k;
                            in = x >= 0 && x < w && y >= 0 && y < h;
                            if (in) ic = box_inv_count(x, y, w, h, R);
                        }
                        const float mp = __fmul_rn((float)sp, ic), corr = __fmul_rn((float)sq, ic), mi = MI[i];
                        const float av = __fdiv_rn(__fsub_rn(corr, __fmul_rn(mi, mp)), VE[i]);
                        A[i] = in ? av : 0.f;
                        B[i] = in ? __fsub_rn(mp, __fmul_rn(av, mi)) : 0.f;
                    }
                }
            }
            __syncthreads();
            // horizontal runs: sums of a and b over rows of tile +- R, the tile's columns
            for (int it = tid; it < QH * NS3; it += NT) {
                const int r = it / NS3, c0 = (it - r * NS3) * L3;
                const float* ar = A + r * QW + c0;
                const float* br = B + r * QW + c0;
                float* ha = HP + r * TW + c0;
                float* hb = HQ + r * TW + c0;
                double va[L3 + 2 * R], vb[L3 + 2 * R], sa = 0.0, sa2 = 0.0, sb = 0.0, sb2 = 0.0;
#pragma unroll
                for (int t = 0; t < L3 + 2 * R; t++) {
                    if (TW % L3 != 0 && c0 + t - 2 * R >= TW) break;
                    va[t] = (double)ar[t];
                    vb[t] = (double)br[t];
                    agg_step(sa, sa2, va, t);
                    agg_step(sb, sb2, vb, t);
                    if (t >= 2 * R) {
                        ha[t - 2 * R] = (float)sa;
                        hb[t - 2 * R] = (float)sb;
                    }
                }
            }
            __syncthreads();
            // vertical run down this thread's column: a-bar, b-bar, q = a-bar I + b-bar (depth.rs:404),
            // max(q, 0) (depth.rs:1146) into the tracker
            {
                const float* ha = HP + vr0 * TW + vc;
                const float* hb = HQ + vr0 * TW + vc;
                double va[CPT + 2 * R], vb[CPT + 2 * R], sa = 0.0, sa2 = 0.0, sb = 0.0, sb2 = 0.0;
#pragma unroll
                for (int t = 0; t < CPT + 2 * R; t++) {
                    va[t] = (double)ha[t * TW];
                    vb[t] = (double)hb[t * TW];
                    agg_step(sa, sa2, va, t);
                    agg_step(sb, sb2, vb, t);
                    if (t >= 2 * R) {
                        const int k = t - 2 * R, x = x0 + vc, y = y0 + vr0 + k;
                        if (inner || (x < w && y < h)) {
                            const float ic = inner ? ic_in : box_inv_count(x, y, w, h, R);
                            const float abar = __fmul_rn((float)sa, ic), bbar = __fmul_rn((float)sb, ic);
                            const float q = fmaxf(__fadd_rn(__fmul_rn(abar, I[(vr0 + k + 2 * R) * PWI + vc + 2 * R]), bbar), 0.f);
                            peak_push(st[k], q, m);
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < CPT; j++) {
            const int x = x0 + vc, y = y0 + vr0 + j;
            if (x >= w || y >= h) continue;
            const size_t o = (size_t)y * w + x, m = (size_t)w * h;
            float* S = a.state;
            S[o] = st[j].c1;
            S[m + o] = st[j].l1;
            S[2 * m + o] = st[j].r1;
            S[3 * m + o] = st[j].c2;
            S[4 * m + o] = st[j].prev;
            S[5 * m + o] = st[j].prev2;
            S[6 * m + o] = st[j].sum;
            S[7 * m + o] = st[j].cmin;
            S[8 * m + o] = __int_as_float(st[j].i1);
        }
    }
}

template <int R, int TW, int TH, class SS>
constexpr size_t guided_peaks_smem() {
    constexpr int PW = TW + 4 * R, PH = TH + 4 * R, QW = TW + 2 * R, QH = TH + 2 * R;
    constexpr int CE = 16 / (int)sizeof(SS), LEAD = (2 * R + CE - 1) / CE * CE, PS = (LEAD - 2 * R + PW + CE - 1) / CE * CE;
    return sizeof(SS) * 2 * PH * PS + sizeof(float) * ((size_t)PH * (PW | 1) + 4 * QH * QW + 2 * PH * QW);
}

// Without aggregation (agg_radius 0) the slices go to the tracker (depth.rs:547) as they are.
template <class SS>
__global__ void peaks_raw_kernel(const SS* __restrict__ slices, int n, size_t m, float* __restrict__ S) {
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < m; o += (size_t)gridDim.x * blockDim.x) {
        PeakState st{-1.f, -1.f, -1.f, -1.f, 0.f, 0.f, 0.f, __int_as_float(0x7f800000), 0};
        for (int k = 0; k < n; k++) peak_push(st, lsb_ld<SS>(slices + (size_t)k * m + o), k);
        S[o] = st.c1;
        S[m + o] = st.l1;
        S[2 * m + o] = st.r1;
        S[3 * m + o] = st.c2;
        S[4 * m + o] = st.prev;
        S[5 * m + o] = st.prev2;
        S[6 * m + o] = st.sum;
        S[7 * m + o] = st.cmin;
        S[8 * m + o] = __int_as_float(st.i1);
    }
}

size_t aggregate_smem_bytes(int r) {
    const int TWD = r <= 4 ? 64 : 32, THD = 32;
    const int PW = TWD + 4 * r, PH = THD + 4 * r, QW = TWD + 2 * r, QH = THD + 2 * r;
    return sizeof(float) * (size_t)(2 * PW * PH + 4 * QW * QH + 2 * PH * QW);
}

template <int R, int TW, int TH, class SS>
static cudaError_t launch_guided_peaks(AggArgs a, cudaStream_t s, int grid_limit) {
    constexpr size_t smem = guided_peaks_smem<R, TW, TH, SS>();
    constexpr int minb = smem <= 110 * 1024 ? 2 : 1;
    static_assert(smem <= 227 * 1024, "shared memory");
    a.tiles_x = (a.dw + TW - 1) / TW;
    a.ntiles = a.tiles_x * ((a.dh + TH - 1) / TH);
    a.async16 = a.dw % (16 / (int)sizeof(SS)) == 0 && (reinterpret_cast<uintptr_t>(a.slices) & 15) == 0;
    auto k = guided_peaks_kernel<R, TW, TH, SS, minb>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    lsb_launched(), k<<<std::min(a.ntiles, std::max(1, grid_limit)), 256, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t aggregate_peaks(AggArgs a, bool slice_fp16, cudaStream_t s, int grid_limit, bool running) {
    size_t m = (size_t)a.dw * a.dh;
    if (a.r == 0) {
        if (slice_fp16) lsb_launched(), peaks_raw_kernel<__half><<<grid1(m), 256, 0, s>>>((const __half*)a.slices, a.n, m, a.state);
        else lsb_launched(), peaks_raw_kernel<float><<<grid1(m), 256, 0, s>>>((const float*)a.slices, a.n, m, a.state);
        return cudaGetLastError();
    }
    // the reference's default radius (3) and the large-frame one (8) by moving sums
    if (running && a.r == 3)
        return slice_fp16 ? launch_guided_peaks<3, 64, 32, __half>(a, s, grid_limit) : launch_guided_peaks<3, 64, 32, float>(a, s, grid_limit);
    if (running && a.r == 8)
        return slice_fp16 ? launch_guided_peaks<8, 64, 32, __half>(a, s, grid_limit) : launch_guided_peaks<8, 64, 32, float>(a, s, grid_limit);
    const int TWD = a.r <= 4 ? 64 : 32, THD = 32;
    a.tiles_x = (a.dw + TWD - 1) / TWD;
    a.ntiles = a.tiles_x * ((a.dh + THD - 1) / THD);
    size_t smem = aggregate_smem_bytes(a.r);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    int grid = std::min(a.ntiles, std::max(1, grid_limit));
    cudaError_t e;
#define LAUNCH_AGG(TWV, SST, RTV)                                                              \
    {                                                                                          \
        auto k = aggregate_kernel<TWV, 32, SST, RTV>;                                          \
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);   \
        if (e != cudaSuccess) return e;                                                        \
        lsb_launched(), k<<<grid, 256, smem, s>>>(a);                                          \
    }
    // the reference's default radius (3) and the large-frame one (8) compiled in; others at run time
    if (TWD == 64) {
        if (a.r == 3) {
            if (slice_fp16) LAUNCH_AGG(64, __half, 3) else LAUNCH_AGG(64, float, 3)
        } else {
            if (slice_fp16) LAUNCH_AGG(64, __half, 0) else LAUNCH_AGG(64, float, 0)
        }
    } else {
        if (a.r == 8) {
            if (slice_fp16) LAUNCH_AGG(32, __half, 8) else LAUNCH_AGG(32, float, 8)
        } else {
            if (slice_fp16) LAUNCH_AGG(32, __half, 0) else LAUNCH_AGG(32, float, 0)
        }
    }
#undef LAUNCH_AGG
    return cudaGetLastError();
}

// ------------------------------------------------------------- k-th value
// depth.rs:580 and :618 `select_nth_unstable_by(total_cmp)` (the noise floor's median, p90):
// the k-th value by a two-pass 16-bit radix histogram of total-order keys.
// The key of a float in the total order (total_cmp): monotone as u32.
__device__ __forceinline__ unsigned fkey(float f) {
    unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
__global__ void hist_kernel(const float* __restrict__ v, size_t cnt, int stride, unsigned* hist, const unsigned* sel, int pass) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cnt; i += (size_t)gridDim.x * blockDim.x) {
        const unsigned k = fkey(v[i * stride]);
        if (pass == 0) atomicAdd(&hist[k >> 16], 1u);
        else if ((k >> 16) == sel[0]) atomicAdd(&hist[k & 0xffffu], 1u);
    }
}
// One block: find the bin holding rank sel[1] (pass 0) / sel[2] (pass 1).
__global__ void scan_kernel(const unsigned* hist, unsigned* sel, int pass, float* out) {
    __shared__ unsigned part[1024];
    const int t = threadIdx.x;
    unsigned s = 0;
    for (int b = t * 64; b < t * 64 + 64; b++) s += hist[b];
    part[t] = s;
    __syncthreads();
    if (t == 0) {
        unsigned want = pass == 0 ? sel[1] : sel[2], acc = 0;
        int chunk = 0;
        while (chunk < 1023 && acc + part[chunk] <= want) acc += part[chunk++];
        int b = chunk * 64;
        while (b < chunk * 64 + 63 && acc + hist[b] <= want) acc += hist[b++];
        if (pass == 0) {
            sel[0] = (unsigned)b;
            sel[2] = want - acc;
        } else {
            *out = fkey_inv((sel[0] << 16) | (unsigned)b);
        }
    }
}
__global__ void set_rank_kernel(unsigned* sel, unsigned rank) { sel[1] = rank; }

cudaError_t select_kth(const float* v, size_t cnt, int stride, size_t rank, unsigned* hist, unsigned* sel, float* out,
                       cudaStream_t s) {
    cudaMemsetAsync(hist, 0, sizeof(unsigned) * 65536, s);
    lsb_launched(), set_rank_kernel<<<1, 1, 0, s>>>(sel, (unsigned)rank);
    lsb_launched(), hist_kernel<<<grid1(cnt), 256, 0, s>>>(v, cnt, stride, hist, sel, 0);
    lsb_launched(), scan_kernel<<<1, 1024, 0, s>>>(hist, sel, 0, out);
    cudaMemsetAsync(hist, 0, sizeof(unsigned) * 65536, s);
    lsb_launched(), hist_kernel<<<grid1(cnt), 256, 0, s>>>(v, cnt, stride, hist, sel, 1);
    lsb_launched(), scan_kernel<<<1, 1024, 0, s>>>(hist, sel, 1, out);
    return cudaGetLastError();
}

// ------------------------------------------------------------ peak finish
// depth.rs:568 `finish`: the last slice's peak, the log-parabola offset, the
// confidence (prominence x peak ratio x noise gate) and the profile minimum.
__global__ void peak_finish_kernel(const float* __restrict__ S, size_t m, int n, const float* __restrict__ floor_p, float gate,
                                   float* __restrict__ depth, float* __restrict__ conf, float* __restrict__ mins) {
    const float fl = *floor_p;
    const float inv_n = __fdiv_rn(1.f, (float)n);
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < m; o += (size_t)gridDim.x * blockDim.x) {
        PeakState p{S[o], S[m + o], S[2 * m + o], S[3 * m + o], S[4 * m + o], S[5 * m + o], S[6 * m + o], S[7 * m + o],
                    __float_as_int(S[8 * m + o])};
        if (n == 1 || p.prev >= p.prev2) peak_reg(p, p.prev, n - 1, n >= 2 ? p.prev2 : -1.f, -1.f);
        const float c1 = p.c1, l = p.l1, r = p.r1;
        float delta = 0.f;
        if (l >= 0.f && r >= 0.f && c1 > 0.f) {
            const float ll = logf(fmaxf(l, 1e-12f)), lc = logf(c1), lr = logf(fmaxf(r, 1e-12f));
            const float den = __fadd_rn(__fsub_rn(ll, __fmul_rn(2.f, lc)), lr);
            if (den < 0.f) delta = fminf(fmaxf(__fdiv_rn(__fmul_rn(0.5f, __fsub_rn(ll, lr)), den), -0.5f), 0.5f);
        }
        depth[o] = __fadd_rn((float)p.i1, delta);
        float c = 0.f;
        if (c1 > 0.f) {
            const float mean = __fmul_rn(p.sum, inv_n);
            const float prom = fminf(fmaxf(__fsub_rn(1.f, __fdiv_rn(mean, c1)), 0.f), 1.f);
            const float pkr = p.c2 >= 0.f ? fminf(fmaxf(__fsub_rn(1.f, __fdiv_rn(p.c2, c1)), 0.f), 1.f) : 1.f;
            const float g = (gate > 0.f && fl > 0.f) ? fminf(fmaxf(__fdiv_rn(__fsub_rn(c1, fl), __fmul_rn(gate, fl)), 0.f), 1.f) : 1.f;
            c = __fmul_rn(__fmul_rn(prom, pkr), g);
        }
        conf[o] = c;
        mins[o] = isfinite(p.cmin) ? p.cmin : 0.f;
    }
}
cudaError_t peak_finish(const float* state, size_t m, int n, const float* floor_p, float gate, float* depth, float* conf,
                        float* mins, cudaStream_t s) {
    lsb_launched(), peak_finish_kernel<<<grid1(m), 256, 0, s>>>(state, m, n, floor_p, gate, depth, conf, mins);
    return cudaGetLastError();
}

// depth.rs:628 `median3`: 3x3 median, reflect-101.
__device__ __forceinline__ void cswap(float& a, float& b) {
    const float lo = fminf(a, b), hi = fmaxf(a, b);
    a = lo;
    b = hi;
}
__global__ void median3_kernel(const float* __restrict__ src, float* __restrict__ out, int w, int h) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    float v[9];
    int k = 0;
    for (int dy = -1; dy <= 1; dy++) {
        const float* row = src + (size_t)lsb_reflect(y + dy, h) * w;
        for (int dx = -1; dx <= 1; dx++) v[k++] = row[lsb_reflect(x + dx, w)];
    }
    // a sorting network, then the middle element
    for (int i = 0; i < 9; i++)
        for (int j = 0; j < 8 - i; j++) cswap(v[j], v[j + 1]);
    out[(size_t)y * w + x] = v[4];
}
cudaError_t median3(const float* src, float* out, int w, int h, cudaStream_t s) {
    dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    lsb_launched(), median3_kernel<<<g, b, 0, s>>>(src, out, w, h);
    return cudaGetLastError();
}

// depth.rs:615 `normalize_conf`: c = min(c / p90, 1) when p90 > 1e-6
__global__ void conf_scale_kernel(float* conf, size_t m, const float* p90) {
    const float p = *p90;
    if (!(p > 1e-6f)) return;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
        conf[i] = fminf(__fdiv_rn(conf[i], p), 1.f);
}
cudaError_t conf_scale(float* conf, size_t m, const float* p90, cudaStream_t s) {
    lsb_launched(), conf_scale_kernel<<<grid1(m), 256, 0, s>>>(conf, m, p90);
    return cudaGetLastError();
}

// depth.rs:1168 robust reweighting: w2 = c * min(tau / |d - u|, 1)
__global__ void robust_kernel(const float* __restrict__ conf, const float* __restrict__ d, const float* __restrict__ u,
                              float tau, float* __restrict__ w2, size_t m) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
        w2[i] = __fmul_rn(conf[i], fminf(__fdiv_rn(tau, fabsf(__fsub_rn(d[i], u[i]))), 1.f));
}
cudaError_t robust_weights(const float* conf, const float* d, const float* u, float tau, float* w2, size_t m, cudaStream_t s) {
    lsb_launched(), robust_kernel<<<grid1(m), 256, 0, s>>>(conf, d, u, tau, w2, m);
    return cudaGetLastError();
}

// ----------------------------------------------------------------- upsample
// depth.rs:201 `upsample_bilinear` weights for an axis position.
// depth.rs:1183-1197: depth = clamp(a-bar(x) * Y + b-bar(x), 0, n-1) with the
// coefficients bilinear from the grid (a = 0, b = u for bilinear upsampling);
// the confidence bilinear too.
__global__ void upsample_kernel(const float* __restrict__ abar, const float* __restrict__ bbar, const float* __restrict__ yfull,
                                const float* __restrict__ conf, int w, int h, int dw, int dh, int k, float max_d, int guided,
                                float* __restrict__ depth, float* __restrict__ conf_full) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const float inv = __fdiv_rn(1.f, (float)k);
    int x0, x1, y0, y1;
    float tx, ty;
    bil_axis(x, inv, dw, x0, x1, tx);
    bil_axis(y, inv, dh, y0, y1, ty);
    const size_t o = (size_t)y * w + x;
    float d;
    if (guided) d = __fadd_rn(__fmul_rn(bil(abar, dw, x0, x1, y0, y1, tx, ty), yfull[o]), bil(bbar, dw, x0, x1, y0, y1, tx, ty));
    else d = bil(bbar, dw, x0, x1, y0, y1, tx, ty);
    depth[o] = fminf(fmaxf(d, 0.f), max_d);
    conf_full[o] = bil(conf, dw, x0, x1, y0, y1, tx, ty);
}
// depth.rs:1184, guided upsampling when k == 1: q = a-bar * I + b-bar on the grid itself, clamped.
__global__ void apply_grid_kernel(const float* __restrict__ abar, const float* __restrict__ bbar, const float* __restrict__ guide,
                                  size_t m, float max_d, int guided, float* __restrict__ depth) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        const float d = guided ? __fadd_rn(__fmul_rn(abar[i], guide[i]), bbar[i]) : bbar[i];
        depth[i] = fminf(fmaxf(d, 0.f), max_d);
    }
}

cudaError_t upsample(const float* abar, const float* bbar, const float* yfull, const float* guide, const float* conf, int w,
                     int h, int dw, int dh, int k, float max_d, bool guided, float* depth, float* conf_full, cudaStream_t s) {
    if (k == 1) {
        lsb_launched(), apply_grid_kernel<<<grid1((size_t)dw * dh), 256, 0, s>>>(abar, bbar, guide, (size_t)dw * dh, max_d, guided ? 1 : 0, depth);
        cudaMemcpyAsync(conf_full, conf, sizeof(float) * dw * dh, cudaMemcpyDeviceToDevice, s);
        return cudaGetLastError();
    }
    dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    lsb_launched(), upsample_kernel<<<g, b, 0, s>>>(abar, bbar, yfull, conf, w, h, dw, dh, k, max_d, guided ? 1 : 0, depth, conf_full);
    return cudaGetLastError();
}

// ------------------------------------------------------ the weighted average
// wav.rs:84 `weight` of every cell: (c - (1 + gate) f).max(0)^power + (1e-2 f)^power + 1e-30
__global__ void wav_weight_kernel(const float* __restrict__ c, const float* __restrict__ floor, size_t m, float gate, float power,
                                  float* __restrict__ out) {
    const float g1 = __fadd_rn(1.f, gate);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        const float f = floor[i];
        const float a = fmaxf(__fsub_rn(c[i], __fmul_rn(g1, f)), 0.f);
        out[i] = __fadd_rn(__fadd_rn(powf(a, power), powf(__fmul_rn(1e-2f, f), power)), 1e-30f);
    }
}
// wav.rs:140: the guided filter's output a-bar * I + b-bar, kept a weight (>= 1e-30)
__global__ void wav_guided_kernel(const float* __restrict__ abar, const float* __restrict__ bbar, const float* __restrict__ guide, size_t m,
                                  float* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
        out[i] = fmaxf(__fadd_rn(__fmul_rn(abar[i], guide[i]), bbar[i]), 1e-30f);
}
__global__ void half_plane_kernel(const __half* __restrict__ src, size_t m, float* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) out[i] = __half2float(src[i]);
}

// wav.rs:131-145 for one frame: its contrast on the grid (the focus slice the fold took), box-smoothed
// (BoxFilter::mean, radius smooth), weighed against the floor cells, then smoothed again by the guided
// filter (guide, mean_i, var_i of radius smooth, eps) or the box mean, into out.
cudaError_t wav_weights(const void* slice, bool half, const float* floor, int dw, int dh, float gate, float power, int smooth, bool edge,
                        const float* guide, const float* mean_i, const float* var_i, float eps, WavScratch& t, float* out, cudaStream_t s) {
    const size_t m = (size_t)dw * dh;
    const float* src = (const float*)slice;
    if (half) {
        lsb_launched(), half_plane_kernel<<<grid1(m), 256, 0, s>>>((const __half*)slice, m, t.s0);
        src = t.s0;
    }
    if (smooth > 0) {
        box_mean(src, nullptr, t.tmp, t.s1, dw, dh, smooth, s);
        src = t.s1;
    }
    lsb_launched(), wav_weight_kernel<<<grid1(m), 256, 0, s>>>(src, floor, m, gate, power, t.s0);
    if (edge && smooth > 0) {
        gf_coeffs(guide, mean_i, var_i, t.s0, dw, dh, smooth, eps, t.t0, t.t1, t.t2, t.tmp, t.abar, t.bbar, s);
        lsb_launched(), wav_guided_kernel<<<grid1(m), 256, 0, s>>>(t.abar, t.bbar, guide, m, out);
    } else if (smooth > 0) {
        box_mean(t.s0, nullptr, t.tmp, out, dw, dh, smooth, s);
    } else {
        return cudaMemcpyAsync(out, t.s0, sizeof(float) * m, cudaMemcpyDeviceToDevice, s);
    }
    return cudaGetLastError();
}

cudaError_t luma_and_guide(const float* img, int w, int h, int k, float* yfull, float* guide, int dw, int dh, cudaStream_t s) {
    size_t n = (size_t)w * h;
    lsb_launched(), luma_kernel<<<grid1(n), 256, 0, s>>>(img, yfull, n);
    if (k == 1) return cudaMemcpyAsync(guide, yfull, sizeof(float) * n, cudaMemcpyDeviceToDevice, s);
    dim3 b(32, 8), g((dw + 31) / 32, (dh + 7) / 8);
    lsb_launched(), block_mean_kernel<<<g, b, 0, s>>>(yfull, w, h, k, guide, dw, dh);
    return cudaGetLastError();
}

}  // namespace lsb
