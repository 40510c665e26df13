// The fold: Burt-Adelson Laplacian pyramid + Wang-Chang region-energy
// selection over ALL frames of a stack, one launch per pyramid level.
//
// Reference semantics (crates/lapstack-core/src): per frame, pyramid.rs:203
// `build` (REDUCE pyramid.rs:86, EXPAND pyramid.rs:143, L = G - EXPAND),
// fuse.rs:200 `region_energy` (Y^2 of fuse.rs:160 through the binomial
// window of fuse.rs:168) and the strict-> winner-take-all of fuse.rs:414-451
// (ties to the earlier frame), frames folded in order.
//
// B200 layout: level-major instead of frame-major. A CTA owns a 64x32 tile of
// level l and walks the frames k = 0..n-1; for each it stages the G_l window
// (tile + halo) in shared memory, REDUCEs it to G_{l+1} (written once to HBM
// for the next level's pass), EXPANDs back, forms L_l, the luma energy and
// its window sum, and keeps the running best energy, the winning L_l
// coefficients and the winner index in registers. The accumulator is written
// once per level instead of read-modified-written once per frame. At level 0
// the source is the interleaved u16 frame itself (gains and, for aligned
// stacks, the Spline4x4 warp applied on load), and the depth pass's focus
// slice (depth.rs:1097: luma -> ring difference filter -> block mean) is
// taken from the same staged tile.
//
// Every float op on the selection path is an explicit round-to-nearest
// intrinsic in the reference's association order, so selection maps and
// coefficients are bit-identical to the reference FP32 CPU path.
#include <algorithm>

#include "lsb_common.cuh"
#include "lsb_internal.h"
#include "lsb_interp.cuh"

namespace lsb {

constexpr int TW = 64, TH = 32, NT = 256, PPT = (TW * TH) / NT;
constexpr int RMAX = 2;
constexpr int LW_MAX = TW + 2 * RMAX, LH_MAX = TH + 2 * RMAX;
constexpr int AW_MAX = LW_MAX / 2 + 5, AH_MAX = LH_MAX / 2 + 5;
constexpr int GW_MAX = 2 * AW_MAX + 4, GH_MAX = 2 * AH_MAX + 4;
constexpr int G0_MAX = GW_MAX * GH_MAX;
constexpr int SCR_MAX = GH_MAX * AW_MAX + AH_MAX * AW_MAX + AH_MAX * LW_MAX;
constexpr int YB_MAX = LW_MAX * LH_MAX;
constexpr int FOC_R = 3;
static_assert((TW + 2 * FOC_R) * (TH + 2 * FOC_R) <= SCR_MAX, "focus window must fit the scratch");
static_assert(LH_MAX * TW <= SCR_MAX, "window scratch must fit");
constexpr int SMEM_FLOATS = 3 * G0_MAX + SCR_MAX + YB_MAX + 3 * TW * TH;

// conv_sparse taps (depth.rs:417) in the per-pixel accumulation order: rows
// grouped by dy in order of first appearance, within a row in list order.
__constant__ float c_taps[3 * 64];

// binomial(R) of fuse.rs:139: C(2R, t) / 4^R, exact in f32.
template <int R>
__device__ __forceinline__ float binw(int t) {
    if (R == 1) return t == 1 ? 0.5f : 0.25f;
    if (R == 2) return t == 2 ? 0.375f : (t == 1 || t == 3 ? 0.25f : 0.0625f);
    return 1.f;
}

template <int SRC, class GS, int R, bool FOCUS, class SS>
__global__ void __launch_bounds__(NT, 2) fold_level_kernel(const FoldArgs a) {
    extern __shared__ float sm[];
    float* g0 = sm;                     // [3][gh][gw]
    float* scr = g0 + 3 * G0_MAX;       // per-channel scratch / focus luma / window rows
    float* yb = scr + SCR_MAX;          // [lh][lw] luma (then energy) of L
    float* lo = yb + YB_MAX;            // [3][TH][TW] L at the tile's own pixels
    const int tid = threadIdx.x;
    const int W = a.W, H = a.H, W1 = a.W1, H1 = a.H1;
    const float2 sc = make_float2(a.gscale, a.ginv);

    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const int x0 = (tile % a.tiles_x) * TW, y0 = (tile / a.tiles_x) * TH;
        const int xL0 = max(0, x0 - R), xL1 = min(W, x0 + TW + R);
        const int yL0 = max(0, y0 - R), yL1 = min(H, y0 + TH + R);
        const int xA0 = max(0, (xL0 >> 1) - 1), xA1 = min(W1, ((xL1 - 1) >> 1) + 2);
        const int yA0 = max(0, (yL0 >> 1) - 1), yA1 = min(H1, ((yL1 - 1) >> 1) + 2);
        const int xG0 = max(0, 2 * xA0 - 2), xG1 = min(W, 2 * xA1 + 1);
        const int yG0 = max(0, 2 * yA0 - 2), yG1 = min(H, 2 * yA1 + 1);
        const int gw = xG1 - xG0, gh = yG1 - yG0, aw = xA1 - xA0, ah = yA1 - yA0, lw = xL1 - xL0, lh = yL1 - yL0;
        if (gw > GW_MAX || gh > GH_MAX || aw > AW_MAX || ah > AH_MAX) {
            if (tid == 0) atomicOr(a.status, LSB_ERR_SHAPE);
            return;
        }
        float* tmph = scr;                       // [gh][aw]
        float* g1 = tmph + GH_MAX * AW_MAX;      // [ah][aw]
        float* exph = g1 + AH_MAX * AW_MAX;      // [ah][lw]
        const int ox1 = min(TW, W - x0), oy1 = min(TH, H - y0);  // the tile's own extent

        float best[PPT], acc[PPT][3];
        int win[PPT];
#pragma unroll
        for (int j = 0; j < PPT; j++) {
            best[j] = -1.f;  // any energy (>= 0) beats it: frame 0 fills the accumulator (fuse.rs:409-412)
            acc[j][0] = acc[j][1] = acc[j][2] = 0.f;
            win[j] = 0;
        }

        for (int k = 0; k < a.nframes; k++) {
            // ---- stage G_l over the window, three channels
            if (SRC == SRC_U16) {
                const uint16_t* f = a.src_u16 + (size_t)k * W * H * 3;
                const FrameXform xf = a.xf[k];
                for (int i = tid; i < gh * gw; i += NT) {
                    float v[3];
                    load_u16_px(f, xf, a.interp, W, H, xG0 + i % gw, yG0 + i / gw, v);
                    g0[i] = v[0];
                    g0[G0_MAX + i] = v[1];
                    g0[2 * G0_MAX + i] = v[2];
                }
            } else if (SRC == SRC_F32) {
                const float* f = a.src_f32 + (size_t)k * 3 * W * H;
                for (int c = 0; c < 3; c++)
                    for (int i = tid; i < gh * gw; i += NT)
                        g0[c * G0_MAX + i] = f[((size_t)c * H + yG0 + i / gw) * W + xG0 + i % gw];
            } else {
                const GS* f = (const GS*)a.src_g + (size_t)k * 3 * W * H;
                for (int c = 0; c < 3; c++)
                    for (int i = tid; i < gh * gw; i += NT)
                        g0[c * G0_MAX + i] = Store<GS>::ld(f + ((size_t)c * H + yG0 + i / gw) * W + xG0 + i % gw, sc);
            }
            __syncthreads();

            // ---- the focus slice of this frame (level 0): depth.rs:1097 focus_slice
            if (FOCUS) {
                const int xF0 = max(0, x0 - FOC_R), xF1 = min(W, x0 + TW + FOC_R);
                const int yF0 = max(0, y0 - FOC_R), yF1 = min(H, y0 + TH + FOC_R);
                const int fw = xF1 - xF0, fh = yF1 - yF0;
                float* yl = scr;
                for (int i = tid; i < fw * fh; i += NT) {
                    int gi = (yF0 + i / fw - yG0) * gw + (xF0 + i % fw - xG0);
                    yl[i] = lsb_luma(g0[gi], g0[G0_MAX + gi], g0[2 * G0_MAX + gi]);
                }
                __syncthreads();
                const int bk = a.bk;
                const int cx0 = x0 / bk, cy0 = y0 / bk;
                const int cw = min(TW / bk, a.dw - cx0), chh = min(TH / bk, a.dh - cy0);
                for (int i = tid; i < cw * chh; i += NT) {
                    const int cx = cx0 + i % cw, cy = cy0 + i / cw;
                    const int px0 = cx * bk, px1 = min(px0 + bk, W), py0 = cy * bk, py1 = min(py0 + bk, H);
                    float o = 0.f;
                    for (int y = py0; y < py1; y++) {
                        float rs = 0.f;
                        for (int x = px0; x < px1; x++) {
                            float m;
                            if (a.focus_kind == 0) {
                                float s = 0.f;
                                for (int t = 0; t < a.ntaps; t++) {
                                    int yy = lsb_reflect(y + (int)c_taps[3 * t], H) - yF0;
                                    int xx = lsb_reflect(x + (int)c_taps[3 * t + 1], W) - xF0;
                                    s = __fadd_rn(s, __fmul_rn(c_taps[3 * t + 2], yl[yy * fw + xx]));
                                }
                                m = fabsf(s);
                            } else {
                                const int st = a.sml_step;
                                float c = yl[(y - yF0) * fw + x - xF0];
                                float l = yl[(y - yF0) * fw + lsb_reflect(x - st, W) - xF0];
                                float r = yl[(y - yF0) * fw + lsb_reflect(x + st, W) - xF0];
                                float u = yl[(lsb_reflect(y - st, H) - yF0) * fw + x - xF0];
                                float d = yl[(lsb_reflect(y + st, H) - yF0) * fw + x - xF0];
                                float c2 = __fmul_rn(2.f, c);
                                m = __fadd_rn(fabsf(__fsub_rn(__fsub_rn(c2, l), r)), fabsf(__fsub_rn(__fsub_rn(c2, u), d)));
                            }
                            rs = __fadd_rn(rs, m);
                        }
                        o = __fadd_rn(o, rs);
                    }
                    o = __fdiv_rn(o, (float)((py1 - py0) * (px1 - px0)));
                    lsb_st<SS>((SS*)a.slice + ((size_t)k * a.dh + cy) * a.dw + cx, o);
                }
                __syncthreads();
            }

            // ---- per channel: REDUCE to G_{l+1}, EXPAND back, L = G - EXPAND(G_{l+1})
            for (int c = 0; c < 3; c++) {
                const float* G = g0 + c * G0_MAX;
                for (int i = tid; i < gh * aw; i += NT) {
                    const int r = i / aw, cc = 2 * (xA0 + i % aw);
                    const float* row = G + r * gw - xG0;
                    tmph[i] = lsb_tap5(row[lsb_reflect(cc - 2, W)], row[lsb_reflect(cc - 1, W)], row[lsb_reflect(cc, W)],
                                       row[lsb_reflect(cc + 1, W)], row[lsb_reflect(cc + 2, W)]);
                }
                __syncthreads();
                GS* dst = (GS*)a.dst_g + ((size_t)k * 3 + c) * W1 * H1;
                for (int i = tid; i < ah * aw; i += NT) {
                    const int iy = yA0 + i / aw, jx = i % aw, cc = 2 * iy;
                    const float* col = tmph + jx - yG0 * aw;
                    float v = lsb_tap5(col[lsb_reflect(cc - 2, H) * aw], col[lsb_reflect(cc - 1, H) * aw], col[lsb_reflect(cc, H) * aw],
                                       col[lsb_reflect(cc + 1, H) * aw], col[lsb_reflect(cc + 2, H) * aw]);
                    const int gx = xA0 + jx;
                    if (gx >= (x0 >> 1) && gx < ((x0 + TW) >> 1) && iy >= (y0 >> 1) && iy < ((y0 + TH) >> 1))
                        Store<GS>::st(dst + (size_t)iy * W1 + gx, v, sc);
                    // the coarse level as stored: with 16-bit storage the next level sees the rounded value
                    g1[i] = Store<GS>::as_stored(v, sc);
                }
                __syncthreads();
                for (int i = tid; i < ah * lw; i += NT) {
                    const int r = i / lw, x = xL0 + i % lw, cx = x >> 1;
                    const float* row = g1 + r * aw - xA0;
                    exph[i] = (x & 1) == 0 ? lsb_exp_even(row[lsb_reflect(cx - 1, W1)], row[lsb_reflect(cx, W1)], row[lsb_reflect(cx + 1, W1)])
                                           : lsb_exp_odd(row[lsb_reflect(cx, W1)], row[lsb_reflect(cx + 1, W1)]);
                }
                __syncthreads();
                for (int i = tid; i < lh * lw; i += NT) {
                    const int y = yL0 + i / lw, xi = i % lw, x = xL0 + xi, cy = y >> 1;
                    const float* col = exph + xi - yA0 * lw;
                    const float up = (y & 1) == 0 ? lsb_exp_even(col[lsb_reflect(cy - 1, H1) * lw], col[lsb_reflect(cy, H1) * lw], col[lsb_reflect(cy + 1, H1) * lw])
                                                   : lsb_exp_odd(col[lsb_reflect(cy, H1) * lw], col[lsb_reflect(cy + 1, H1) * lw]);
                    const float L = __fsub_rn(G[(y - yG0) * gw + x - xG0], up);
                    if (a.use_chroma) {
                        const float q = __fmul_rn(L, L);
                        yb[i] = c == 0 ? q : __fadd_rn(yb[i], q);
                    } else {
                        const float q = __fmul_rn(c == 0 ? 0.299f : (c == 1 ? 0.587f : 0.114f), L);
                        yb[i] = c == 0 ? q : __fadd_rn(yb[i], q);
                    }
                    if (x >= x0 && x < x0 + TW && y >= y0 && y < y0 + TH) lo[(c * TH + y - y0) * TW + x - x0] = L;
                }
                __syncthreads();
            }

            // ---- region energy: e = Y^2, the separable binomial window (fuse.rs:168)
            if (!a.use_chroma)
                for (int i = tid; i < lh * lw; i += NT) yb[i] = __fmul_rn(yb[i], yb[i]);
            float* eh = scr;  // [lh][TW]
            if (R > 0) {
                __syncthreads();
                for (int i = tid; i < lh * TW; i += NT) {
                    const int r = i / TW, xo = i % TW;
                    if (xo >= ox1) continue;
                    const float* row = yb + r * lw - xL0;
                    float s = 0.f;
#pragma unroll
                    for (int t = 0; t <= 2 * R; t++) s = __fadd_rn(s, __fmul_rn(binw<R>(t), row[lsb_reflect(x0 + xo + t - R, W)]));
                    eh[i] = s;
                }
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < PPT; j++) {
                const int p = tid + NT * j, px = p % TW, py = p / TW;
                if (px >= ox1 || py >= oy1) continue;
                float e;
                if (R > 0) {
                    e = 0.f;
#pragma unroll
                    for (int t = 0; t <= 2 * R; t++)
                        e = __fadd_rn(e, __fmul_rn(binw<R>(t), eh[(lsb_reflect(y0 + py + t - R, H) - yL0) * TW + px]));
                } else {
                    e = yb[(y0 + py - yL0) * lw + x0 + px - xL0];
                }
                if (e > best[j]) {
                    best[j] = e;
                    acc[j][0] = lo[(0 * TH + py) * TW + px];
                    acc[j][1] = lo[(1 * TH + py) * TW + px];
                    acc[j][2] = lo[(2 * TH + py) * TW + px];
                    win[j] = k;
                }
            }
            __syncthreads();
        }

        // ---- the level's accumulator, written once
#pragma unroll
        for (int j = 0; j < PPT; j++) {
            const int p = tid + NT * j, px = p % TW, py = p / TW;
            if (px >= ox1 || py >= oy1) continue;
            const size_t o = (size_t)(y0 + py) * W + x0 + px;
            a.acc[o] = acc[j][0];
            a.acc[(size_t)W * H + o] = acc[j][1];
            a.acc[2 * (size_t)W * H + o] = acc[j][2];
            a.best[o] = best[j];
            if (a.winner) a.winner[o] = (uint16_t)win[j];
        }
    }
}

size_t fold_smem_bytes(int, bool) { return (size_t)SMEM_FLOATS * sizeof(float); }

cudaError_t set_focus_taps(const float* taps3, int ntaps, cudaStream_t s) {
    if (ntaps > 64) return cudaErrorInvalidValue;
    return cudaMemcpyToSymbolAsync(c_taps, taps3, sizeof(float) * 3 * ntaps, 0, cudaMemcpyHostToDevice, s);
}

template <int SRC, class GS, int R, bool FOCUS, class SS>
static cudaError_t launch_fold(const FoldArgs& a, cudaStream_t s, int grid_limit) {
    auto k = fold_level_kernel<SRC, GS, R, FOCUS, SS>;
    size_t smem = fold_smem_bytes(R, FOCUS);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = std::min(a.ntiles, std::max(grid_limit, 1));
    lsb_launched(), k<<<grid, NT, smem, s>>>(a);
    return cudaGetLastError();
}

template <int SRC, class GS, int R>
static cudaError_t pick_focus(const FoldArgs& a, bool focus, cudaStream_t s, int gl) {
    if (!focus) return launch_fold<SRC, GS, R, false, float>(a, s, gl);
    // 16-bit storage keeps the focus slices in FP16 (relative precision is what the peak search needs)
    if (sizeof(GS) == 2) return launch_fold<SRC, GS, R, true, __half>(a, s, gl);
    return launch_fold<SRC, GS, R, true, float>(a, s, gl);
}

template <int SRC, class GS>
static cudaError_t pick_r(const FoldArgs& a, int r, bool focus, cudaStream_t s, int gl) {
    switch (r) {
        case 0: return pick_focus<SRC, GS, 0>(a, focus, s, gl);
        case 1: return pick_focus<SRC, GS, 1>(a, focus, s, gl);
        case 2: return pick_focus<SRC, GS, 2>(a, focus, s, gl);
        default: return cudaErrorInvalidValue;
    }
}

template <class GS>
static cudaError_t pick_src(const FoldArgs& a, int src_kind, int r, bool focus, cudaStream_t s, int gl) {
    switch (src_kind) {
        case SRC_U16: return pick_r<SRC_U16, GS>(a, r, focus, s, gl);
        case SRC_F32: return pick_r<SRC_F32, GS>(a, r, focus, s, gl);
        default: return pick_r<SRC_G, GS>(a, r, false, s, gl);
    }
}

cudaError_t fold_level(const FoldArgs& a, int src_kind, int storage, int radius, bool focus, cudaStream_t s, int grid_limit) {
    if (a.ntiles <= 0) return cudaSuccess;
    switch (storage) {
        case STORE_UNORM16: return pick_src<unorm16>(a, src_kind, radius, focus, s, grid_limit);
        case STORE_F16: return pick_src<__half>(a, src_kind, radius, focus, s, grid_limit);
        default: return pick_src<float>(a, src_kind, radius, focus, s, grid_limit);
    }
}

// ------------------------------------------------------------ residual level
// fuse.rs:207 `deviation_entropy` of each frame's top luma, one thread per
// (frame, pixel). lnp[c] = ln(c / n) as the reference's f32 ln gives it
// (computed on the host with the platform libm).
template <class GS>
__global__ void dev_ent_kernel(const ResidualArgs a, const float* __restrict__ lnp) {
    const int n2 = a.w * a.h;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.n * n2) return;
    const int k = idx / n2, pix = idx % n2, i = pix / a.w, j = pix % a.w;
    const GS* t = (const GS*)a.tops + (size_t)k * 3 * n2;
    const int r = a.radius, nwin = (2 * r + 1) * (2 * r + 1);
    const float inv_n = __fdiv_rn(1.f, (float)nwin);
    const float qscale = (float)(min(max(a.bins, 2), 65536) - 1);
    float s = 0.f, s2 = 0.f;
    int q[81];
    int m = 0;
    for (int dy = -r; dy <= r; dy++) {
        const int yy = lsb_reflect(i + dy, a.h);
        for (int dx = -r; dx <= r; dx++) {
            const int o = yy * a.w + lsb_reflect(j + dx, a.w);
            const float2 sc = make_float2(0.f, a.ginv);
            const float v = lsb_luma(Store<GS>::ld(t + o, sc), Store<GS>::ld(t + n2 + o, sc), Store<GS>::ld(t + 2 * n2 + o, sc));
            s = __fadd_rn(s, v);
            s2 = __fadd_rn(s2, __fmul_rn(v, v));
            const float vc = fminf(fmaxf(v, 0.f), 1.f);
            q[m++] = (int)__fadd_rn(__fmul_rn(vc, qscale), 0.5f);
        }
    }
    const float mean = __fmul_rn(s, inv_n);
    a.dev[idx] = fmaxf(__fsub_rn(__fmul_rn(s2, inv_n), __fmul_rn(mean, mean)), 0.f);
    // entropy over the bins in order of first touch
    float e = 0.f;
    for (int u = 0; u < m; u++) {
        bool seen = false;
        for (int v = 0; v < u; v++) seen |= q[v] == q[u];
        if (seen) continue;
        int cnt = 0;
        for (int v = u; v < m; v++) cnt += q[v] == q[u];
        const float p = __fmul_rn((float)cnt, inv_n);
        e = __fsub_rn(e, __fmul_rn(p, lnp[cnt]));
    }
    a.ent[idx] = e;
}

// fuse.rs:248 the Pareto mean (or the plain mean) over the frames per pixel.
template <class GS>
__global__ void pareto_kernel(const ResidualArgs a) {
    const int n2 = a.w * a.h;
    const int pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= n2) return;
    float o[3] = {0.f, 0.f, 0.f};
    const GS* t = (const GS*)a.tops;
    const float2 sc = make_float2(0.f, a.ginv);
    if (a.n == 1 || a.top_rule == 2) {
        const float inv = __fdiv_rn(1.f, (float)a.n);
        for (int k = 0; k < a.n; k++)
            for (int c = 0; c < 3; c++) o[c] = __fadd_rn(o[c], __fmul_rn(Store<GS>::ld(t + ((size_t)k * 3 + c) * n2 + pix, sc), inv));
    } else {
        const bool ent = a.top_rule == 0;
        auto dominated = [&](int x) {
            const float da = a.dev[(size_t)x * n2 + pix], ea = a.ent[(size_t)x * n2 + pix];
            for (int b = 0; b < a.n; b++) {
                if (b == x) continue;
                const float db = a.dev[(size_t)b * n2 + pix], eb = a.ent[(size_t)b * n2 + pix];
                const bool d = ent ? (db >= da && eb >= ea && (db > da || eb > ea)) : (db > da || (db == da && b < x));
                if (d) return true;
            }
            return false;
        };
        int kept = 0;
        for (int x = 0; x < a.n; x++) kept += !dominated(x);
        const float inv = __fdiv_rn(1.f, (float)max(kept, 1));
        for (int x = 0; x < a.n; x++)
            if (!dominated(x))
                for (int c = 0; c < 3; c++) o[c] = __fadd_rn(o[c], __fmul_rn(Store<GS>::ld(t + ((size_t)x * 3 + c) * n2 + pix, sc), inv));
    }
    for (int c = 0; c < 3; c++) a.out[(size_t)c * n2 + pix] = o[c];
}

template <class GS>
static void residual_launch(const ResidualArgs& a, const float* lnp, cudaStream_t s) {
    const int n2 = a.w * a.h;
    if (a.n > 1 && a.top_rule != 2) lsb_launched(), dev_ent_kernel<GS><<<(a.n * n2 + 127) / 128, 128, 0, s>>>(a, lnp);
    lsb_launched(), pareto_kernel<GS><<<(n2 + 127) / 128, 128, 0, s>>>(a);
}
cudaError_t fuse_residuals(const ResidualArgs& a, int storage, const float* lnp, cudaStream_t s) {
    if (a.radius > 4) return cudaErrorInvalidValue;
    if (storage == STORE_UNORM16) residual_launch<unorm16>(a, lnp, s);
    else if (storage == STORE_F16) residual_launch<__half>(a, lnp, s);
    else residual_launch<float>(a, lnp, s);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ collapse
// pyramid.rs:219: G_l = L_l + EXPAND(G_{l+1}), EXPAND horizontal then
// vertical (pyramid.rs:143) evaluated per output pixel with the same taps;
// at level 0 also fuse.rs:516 clamp and io.rs:287 u16 packing.
__device__ __forceinline__ float exp_row(const float* row, int cw, int x) {
    const int cx = x >> 1;
    return (x & 1) == 0 ? lsb_exp_even(row[lsb_reflect(cx - 1, cw)], row[lsb_reflect(cx, cw)], row[lsb_reflect(cx + 1, cw)])
                        : lsb_exp_odd(row[lsb_reflect(cx, cw)], row[lsb_reflect(cx + 1, cw)]);
}

__global__ void collapse_kernel(const float* __restrict__ acc, const float* __restrict__ coarse, float* __restrict__ out,
                                int w, int h, int cw, int ch, int last, uint16_t* __restrict__ rgb) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int cy = y >> 1;
    for (int c = 0; c < 3; c++) {
        const float* C = coarse + (size_t)c * cw * ch;
        float up;
        if ((y & 1) == 0)
            up = lsb_exp_even(exp_row(C + (size_t)lsb_reflect(cy - 1, ch) * cw, cw, x), exp_row(C + (size_t)lsb_reflect(cy, ch) * cw, cw, x),
                              exp_row(C + (size_t)lsb_reflect(cy + 1, ch) * cw, cw, x));
        else
            up = lsb_exp_odd(exp_row(C + (size_t)lsb_reflect(cy, ch) * cw, cw, x), exp_row(C + (size_t)lsb_reflect(cy + 1, ch) * cw, cw, x));
        const size_t o = (size_t)c * w * h + (size_t)y * w + x;
        float v = __fadd_rn(acc[o], up);
        if (last) {
            v = fminf(fmaxf(v, 0.f), 1.f);
            rgb[((size_t)y * w + x) * 3 + c] = (uint16_t)__fadd_rn(__fmul_rn(v, 65535.f), 0.5f);
        }
        out[o] = v;
    }
}

cudaError_t collapse_level(const float* acc, const float* coarse, float* out, int w, int h, int cw, int ch, bool last,
                           uint16_t* rgb_out, cudaStream_t s) {
    dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    lsb_launched(), collapse_kernel<<<g, b, 0, s>>>(acc, coarse, out, w, h, cw, ch, last ? 1 : 0, rgb_out);
    return cudaGetLastError();
}

// ------------------------------------------------------------ winner shares
__global__ void max_kernel(const float* __restrict__ v, int n, float* out) {
    float m = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = fmaxf(m, v[i]);
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax((int*)out, __float_as_int(m));  // non-negative floats order as ints
}
__global__ void count_kernel(const uint16_t* __restrict__ win, const float* __restrict__ best, int n, int frames,
                             const float* mx, unsigned int* counts) {
    const float fl = __fmul_rn(0.01f, *mx);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (best[i] > fl && fl > 0.f && win[i] < frames) atomicAdd(&counts[win[i]], 1u);
}
cudaError_t winner_counts(const uint16_t* win, const float* best, int cells, int frames, unsigned int* counts, float* mx,
                          cudaStream_t s) {
    cudaMemsetAsync(mx, 0, sizeof(float), s);
    cudaMemsetAsync(counts, 0, sizeof(unsigned int) * frames, s);
    int g = std::min((cells + 255) / 256, 4096);
    lsb_launched(), max_kernel<<<g, 256, 0, s>>>(best, cells, mx);
    lsb_launched(), count_kernel<<<g, 256, 0, s>>>(win, best, cells, frames, mx, counts);
    return cudaGetLastError();
}

// ------------------------------------------------------- brightness means
// brightness.rs:67 `sums` at the identity over the stride-4 grid: per frame,
// per-block f64 partial sums (a fixed tree), then the partials in order.
__global__ void means_partial_kernel(const uint16_t* __restrict__ frames, int w, int h, int nparts, double* partial) {
    const int k = blockIdx.y, part = blockIdx.x;
    const int gw = (w + 3) / 4, gh = (h + 3) / 4, ng = gw * gh;
    const int per = (ng + nparts - 1) / nparts, lo = part * per, hi = min(ng, lo + per);
    const uint16_t* f = frames + (size_t)k * w * h * 3;
    double s[3] = {0.0, 0.0, 0.0};
    for (int g = lo + threadIdx.x; g < hi; g += blockDim.x) {
        const size_t i = (size_t)(g / gw) * 4 * w + (g % gw) * 4;
        for (int c = 0; c < 3; c++) s[c] += (double)__fmul_rn((float)f[i * 3 + c], LSB_INV16);
    }
    __shared__ double red[3][256];
    for (int c = 0; c < 3; c++) red[c][threadIdx.x] = s[c];
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st)
            for (int c = 0; c < 3; c++) red[c][threadIdx.x] += red[c][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; c++) partial[((size_t)k * nparts + part) * 3 + c] = red[c][0];
}
__global__ void means_final_kernel(const double* partial, int n, int nparts, int count, double* means) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    for (int c = 0; c < 3; c++) {
        double s = 0.0;
        for (int p = 0; p < nparts; p++) s += partial[((size_t)k * nparts + p) * 3 + c];
        means[k * 3 + c] = count == 0 ? 0.0 : s / (double)count;
    }
}
cudaError_t frame_means(const uint16_t* frames, int n, int w, int h, double* partial, int nparts, double* means, cudaStream_t s) {
    dim3 g(nparts, n);
    lsb_launched(), means_partial_kernel<<<g, 256, 0, s>>>(frames, w, h, nparts, partial);
    const int count = ((w + 3) / 4) * ((h + 3) / 4);
    lsb_launched(), means_final_kernel<<<(n + 127) / 128, 128, 0, s>>>(partial, n, nparts, count, means);
    return cudaGetLastError();
}

}  // namespace lsb
