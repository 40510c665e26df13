// The fold kernels (one pyramid level, all frames) -- included by lsb_fold.cu
// inside namespace lsb.
//
// Level l of the fold runs as two kernels:
//  * reduce_level_kernel, one CTA per (frame, 32x16 tile of G_{l+1}): stages
//    the tile's G_l window, REDUCEs rows then columns (pyramid.rs:86) and
//    writes G_{l+1} once; at level 0 it also takes the frame's focus slice
//    (depth.rs:1097: luma -> ring difference filter -> block mean) from the
//    same staged window. Parallel over frames, so even the coarse levels fill
//    the GPU.
//  * select_level_kernel, persistent over 64x32 tiles of level l: walks the
//    frames in order, stages G_l over the tile +- R and G_{l+1} over what
//    EXPAND needs, forms L = G - EXPAND(G_{l+1}) (pyramid.rs:143/209), the
//    luma energy and its binomial window (fuse.rs:152/168) and keeps the
//    strict-> selection (fuse.rs:429) in registers: thread (tx, ty) owns
//    the tile pixels (tx + 32a, ty + 8b), a < 2, b < 4.
// Tiles whose windows never reach the border index without reflect-101
// (IN = true); border tiles reflect as pyramid.rs:51 does. Every float op is
// an explicit round-to-nearest intrinsic in the reference's order.
#pragma once

constexpr int NT = 256;
// resident CTAs per SM the compiler keeps the register budget for
#ifndef LSB_SEL_MINB
#define LSB_SEL_MINB 2
#endif
#ifndef LSB_RED_MINB
#define LSB_RED_MINB 3
#endif
// select: tile, own pixels per thread, windows
#ifndef LSB_TH
#define LSB_TH 32
#endif
constexpr int TW = 64, TH = LSB_TH, PPT = (TW * TH) / NT;
static_assert(TH % 16 == 0 && PPT % 2 == 0, "thread (tx, ty) owns (tx + 32a, ty + 8b)");
constexpr int RMAX = 2;
constexpr int LW_MAX = TW + 2 * RMAX, LH_MAX = TH + 2 * RMAX;
constexpr int AW_MAX = LW_MAX / 2 + 5, AH_MAX = LH_MAX / 2 + 5;
constexpr int SEL_GL = LW_MAX * LH_MAX;  // per channel
constexpr int SEL_G1 = AW_MAX * AH_MAX;
constexpr int SEL_EXP = AH_MAX * LW_MAX;
constexpr int SEL_FLOATS = 3 * (SEL_GL + SEL_G1 + SEL_EXP) + LW_MAX * LH_MAX;
static_assert(LH_MAX * TW <= 3 * SEL_EXP, "the window rows fit the EXPAND scratch");
// reduce: tile of G_{l+1}, G_l window with the focus halo
constexpr int RW = 32, RH = 16, FOC_R = 3;
constexpr int RGW = 2 * RW + 2 * FOC_R, RGH = 2 * RH + 2 * FOC_R;  // 70 x 38
constexpr int RED_WPR = (RGW * 6 + 2 + 3) / 4;  // words per staged u16 window row (with 2 bytes of slack)
constexpr int RED_FLOATS = 3 * RGW * RGH + RGW * RGH + 3 * RGH * RW + RGH * RED_WPR;

// ---- the level-0 tiles of the fused kernel (lsb_fold0.cuh) and the others
// Tiles of level 0 the fused kernel takes: columns [1, ix1) and rows [1, iy1) of the 64x32 tile grid
// (their windows, G_1 reads and slice cells lie inside the frame). 0 tiles when the frame is small.
struct Fold0Range {
    int ix1, iy1;
};
__host__ __device__ inline Fold0Range fold0_range(int W, int H, int R) {
    Fold0Range r;
    const int xs = W - 70 + (R & 1), ys = H - 38;
    r.ix1 = xs >= 64 ? xs / 64 + 1 : 1;
    r.iy1 = ys >= 32 ? ys / 32 + 1 : 1;
    return r;
}
__host__ __device__ inline bool fold0_interior(int tx, int ty, const Fold0Range& r) {
    return tx >= 1 && tx < r.ix1 && ty >= 1 && ty < r.iy1;
}
__host__ __device__ inline int fold0_count(const Fold0Range& r) { return (r.ix1 - 1) * (r.iy1 - 1); }

// The tiles the fused kernel leaves (those whose window meets the frame border), enumerated for the
// two-kernel path: row 0, then columns 0 and ix1.. of rows 1 .. iy1-1, then rows iy1.. . b < count.
__host__ __device__ inline int fold0_border_count(int tiles_x, int tiles_y, const Fold0Range& r) {
    return tiles_x * tiles_y - fold0_count(r);
}
__host__ __device__ inline int fold0_border_tile(int b, int tiles_x, const Fold0Range& r) {
    if (r.ix1 <= 1 || r.iy1 <= 1) return b;  // no interior: every tile is a border tile
    if (b < tiles_x) return b;
    b -= tiles_x;
    const int per = tiles_x - (r.ix1 - 1), mid = (r.iy1 - 1) * per;
    if (b < mid) {
        const int ty = 1 + b / per, j = b - (b / per) * per;
        return ty * tiles_x + (j == 0 ? 0 : r.ix1 + j - 1);
    }
    return r.iy1 * tiles_x + (b - mid);
}

// conv_sparse taps (depth.rs:417) in the per-pixel accumulation order: rows
// grouped by dy in order of first appearance, within a row in list order.
__constant__ float c_taps[3 * 64];
// the same taps for an interior window (rows RGW apart): offsets dy * RGW + dx and weights
__constant__ int c_tapo[64];
__constant__ float c_tapw[64];

// The default ring difference filter (r_in 1, r_out 3: a 5-tap disk at +1/5,
// a 24-tap ring at -1/24) in the order depth.rs:417 `conv_sparse` sums it
// (rows in order of first appearance, each row's taps in list order), with
// the offsets and weights as immediates. RDF_W* are the host's 1/|disk| and
// -1/|ring| in f32.
constexpr float RDF_WD = 1.0f / 5.0f, RDF_WR = -1.0f / 24.0f;
__device__ __forceinline__ float rdf13(const float* __restrict__ yc) {
    constexpr int T[29][3] = {{-1, 0, 0},  {-1, -2, 1}, {-1, -1, 1}, {-1, 1, 1}, {-1, 2, 1}, {0, -1, 0}, {0, 0, 0},  {0, 1, 0},
                              {0, -3, 1},  {0, -2, 1},  {0, 2, 1},   {0, 3, 1},  {1, 0, 0},  {1, -2, 1}, {1, -1, 1}, {1, 1, 1},
                              {1, 2, 1},   {-3, 0, 1},  {-2, -2, 1}, {-2, -1, 1}, {-2, 0, 1}, {-2, 1, 1}, {-2, 2, 1}, {2, -2, 1},
                              {2, -1, 1},  {2, 0, 1},   {2, 1, 1},   {2, 2, 1},  {3, 0, 1}};
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 29; q++) s = __fadd_rn(s, __fmul_rn(T[q][2] ? RDF_WR : RDF_WD, yc[T[q][0] * RGW + T[q][1]]));
    return s;
}

// binomial(R) of fuse.rs:139: C(2R, t) / 4^R, exact in f32.
template <int R>
__device__ __forceinline__ float binw(int t) {
    if (R == 1) return t == 1 ? 0.5f : 0.25f;
    if (R == 2) return t == 2 ? 0.375f : (t == 1 || t == 3 ? 0.25f : 0.0625f);
    return 1.f;
}

// fuse.rs:127 `halo_weight`: exp(clamp(p * ln((E + 1e-8) / 1e-4), -60, 60))
__device__ __forceinline__ float halo_weight(float e, float p) {
    const float v = __fmul_rn(p, logf(__fdiv_rn(__fadd_rn(e, 1e-8f), 1e-4f)));
    return expf(fminf(fmaxf(v, -60.f), 60.f));
}

// The level-l value of (x, y), three channels, from the level's source:
// level 0 the frame (u16 interleaved or f32 planar) times its gains
// (brightness.rs:124); above, the stored Gaussian level.
template <int SRC, class GS>
__device__ __forceinline__ void level_px(const FoldArgs& a, int k, int x, int y, float v[3]) {
    const size_t np = (size_t)a.W * a.H, o = (size_t)y * a.W + x;
    if (SRC == SRC_U16) {
        const uint16_t* p = a.src_u16 + (size_t)k * np * 3 + o * 3;
        v[0] = __fmul_rn((float)p[0], LSB_INV16);
        v[1] = __fmul_rn((float)p[1], LSB_INV16);
        v[2] = __fmul_rn((float)p[2], LSB_INV16);
    } else if (SRC == SRC_F32) {
        const float* p = a.src_f32 + (size_t)k * 3 * np + o;
        v[0] = p[0];
        v[1] = p[np];
        v[2] = p[2 * np];
    } else {
        const float2 sc = make_float2(a.xf[k].gscale, a.xf[k].ginv);
        const GS* p = (const GS*)a.src_g + (size_t)k * 3 * np + o;
        v[0] = Store<GS>::ld(p, sc);
        v[1] = Store<GS>::ld(p + np, sc);
        v[2] = Store<GS>::ld(p + 2 * np, sc);
        return;
    }
    const int gon = a.xf[k].gain_on;
    if (gon) {
        for (int c = 0; c < 3; c++)
            if (gon & (1 << c)) v[c] = __fmul_rn(v[c], a.xf[k].gain[c]);
    }
}

// 4-byte global -> shared copies that bypass the registers (cp.async)
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ------------------------------------------------------------------ REDUCE
template <int SRC, class GS, bool FOCUS, class SS, bool IN>
__device__ __forceinline__ void reduce_tile(const FoldArgs& a, float* __restrict__ sm, int k, int gx0, int gy0) {
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int W = a.W, H = a.H, W1 = a.W1, H1 = a.H1;
#define RX(i) (IN ? (i) : lsb_reflect((i), W))
#define RY(i) (IN ? (i) : lsb_reflect((i), H))
    float* g0 = sm;                      // [3][wh][ww]
    float* yl = g0 + 3 * RGW * RGH;      // [wh][ww] focus luma
    float* tmph = yl + RGW * RGH;        // [3][wh][RW]
    // the window of the tile's outputs and the focus taps' reach: RGW x RGH from (xw0, yw0); a border
    // tile's window is staged with its coordinates reflected into the level (pyramid.rs:51 reflect-101,
    // the same reflect every tap applies), so every tap below indexes it directly
    const int xw0 = 2 * gx0 - FOC_R, yw0 = 2 * gy0 - FOC_R;
    constexpr int ww = RGW, wh = RGH;
    if (SRC == SRC_U16 && IN) {
        // the interleaved u16 window rows copied as words into shared memory (each row from the
        // word at or before its first byte; fold inputs carry tail padding), then converted
        uint32_t* raw = (uint32_t*)(tmph + 3 * RGH * RW);
        const unsigned char* src = (const unsigned char*)a.src_u16;
        for (int i = threadIdx.x; i < RGH * RED_WPR; i += NT) {
            const int r = i / RED_WPR, wd = i - r * RED_WPR;
            const size_t byte = (((size_t)k * H + yw0 + r) * W + xw0) * 6;
            cp_async4(raw + i, src + (byte & ~(size_t)3) + 4 * wd);
        }
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        const int gon = a.xf[k].gain_on;
        float gain[3];
        for (int q = 0; q < 3; q++) gain[q] = a.xf[k].gain[q];
        const unsigned mis0 = (unsigned)(((((size_t)k * H + yw0) * W + xw0) * 6) & 3), rowmis = (unsigned)((W * 6) & 3);
        for (int m = threadIdx.x; m < RGH * RGW; m += NT) {  // the window's pixels over all threads
            const int r = m / RGW, c = m - r * RGW;
            const unsigned mis = (mis0 + (unsigned)r * rowmis) & 3;  // the row's first byte within its word
            const uint16_t* row = (const uint16_t*)((const unsigned char*)(raw + r * RED_WPR) + mis);
            {
                float v[3];
                for (int q = 0; q < 3; q++) {
                    v[q] = __fmul_rn((float)row[3 * c + q], LSB_INV16);
                    if (gon & (1 << q)) v[q] = __fmul_rn(v[q], gain[q]);
                }
                const int i = r * RGW + c;
                g0[i] = v[0];
                g0[RGW * RGH + i] = v[1];
                g0[2 * RGW * RGH + i] = v[2];
                if (FOCUS) yl[i] = lsb_luma(v[0], v[1], v[2]);
            }
        }
    } else if (SRC == SRC_G) {
        // a stored level: the frame's scale read once, three planes
        const float2 sc = make_float2(a.xf[k].gscale, a.xf[k].ginv);
        const size_t np = (size_t)W * H;
        const GS* f = (const GS*)a.src_g + (size_t)k * 3 * np;
        for (int m = threadIdx.x; m < wh * ww; m += NT) {  // the window's pixels over all threads
            const int r = m / ww, c = m - r * ww;
            const GS* px = f + (size_t)RY(yw0 + r) * W + RX(xw0 + c);
            {
                const int i = r * ww + c;
                g0[i] = Store<GS>::ld(px, sc);
                g0[RGW * RGH + i] = Store<GS>::ld(px + np, sc);
                g0[2 * RGW * RGH + i] = Store<GS>::ld(px + 2 * np, sc);
            }
        }
    } else
    for (int r = ty; r < wh; r += 8)
        for (int c = tx; c < ww; c += 32) {
            float v[3];
            level_px<SRC, GS>(a, k, RX(xw0 + c), RY(yw0 + r), v);
            const int i = r * ww + c;
            g0[i] = v[0];
            g0[RGW * RGH + i] = v[1];
            g0[2 * RGW * RGH + i] = v[2];
            if (FOCUS) yl[i] = lsb_luma(v[0], v[1], v[2]);
        }
    __syncthreads();
    const int ow = IN ? RW : min(RW, W1 - gx0), oh = IN ? RH : min(RH, H1 - gy0);
    // rows (pyramid.rs:90), the wh x ow outputs over all threads
    for (int m = threadIdx.x; m < wh * ow; m += NT) {
        const int r = m / ow, j = m - r * ow;
        {
            const int cc = 2 * (gx0 + j);
            const int i0 = cc - 2 - xw0, i1 = i0 + 1, i2 = i0 + 2, i3 = i0 + 3, i4 = i0 + 4;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float* row = g0 + c * RGW * RGH + r * ww;
                tmph[(c * RGH + r) * RW + j] = lsb_tap5(row[i0], row[i1], row[i2], row[i3], row[i4]);
            }
        }
    }
    if (FOCUS) {
        const int bk = a.bk;
        const int cx0 = (2 * gx0) / bk, cy0 = (2 * gy0) / bk;
        const int cw = min(2 * RW / bk, a.dw - cx0), chh = min(2 * RH / bk, a.dh - cy0);
        if (IN && bk == 2 && a.rdf13 && a.focus_kind == 0) {  // whole 2x2 blocks (interior tiles)
            // the default filter over whole 2x2 blocks (interior tiles): the generic loop, unrolled
            for (int cyy = ty; cyy < RH; cyy += 8)
                for (int cxx = tx; cxx < RW; cxx += 32) {
                    const int cx = cx0 + cxx, cy = cy0 + cyy;
                    const float* yc = yl + (2 * cy - yw0) * RGW + (2 * cx - xw0);
                    float o = 0.f;
#pragma unroll
                    for (int dy = 0; dy < 2; dy++) {
                        float rs = 0.f;
#pragma unroll
                        for (int dx = 0; dx < 2; dx++) rs = __fadd_rn(rs, fabsf(rdf13(yc + dy * RGW + dx)));
                        o = __fadd_rn(o, rs);
                    }
                    lsb_st<SS>((SS*)a.slice + ((size_t)k * a.dh + cy) * a.dw + cx, __fdiv_rn(o, 4.f));
                }
        } else
        for (int cyy = ty; cyy < chh; cyy += 8)
            for (int cxx = tx; cxx < cw; cxx += 32) {
                const int cx = cx0 + cxx, cy = cy0 + cyy;
                const int px0 = cx * bk, px1 = min(px0 + bk, W), py0 = cy * bk, py1 = min(py0 + bk, H);
                float o = 0.f;
                for (int y = py0; y < py1; y++) {
                    float rs = 0.f;
                    for (int x = px0; x < px1; x++) {
                        float m;
                        if (a.focus_kind == 0) {
                            float s = 0.f;
                            if (a.rdf13) {
                                s = rdf13(yl + (y - yw0) * RGW + (x - xw0));
                            } else {
                                const float* yc = yl + (y - yw0) * RGW + (x - xw0);
                                for (int q = 0; q < a.ntaps; q++) s = __fadd_rn(s, __fmul_rn(c_tapw[q], yc[c_tapo[q]]));
                            }
                            m = fabsf(s);
                        } else {
                            const int st = a.sml_step;
                            const float c = yl[(y - yw0) * ww + x - xw0];
                            const float l = yl[(y - yw0) * ww + x - st - xw0], r = yl[(y - yw0) * ww + x + st - xw0];
                            const float u = yl[(y - st - yw0) * ww + x - xw0], d = yl[(y + st - yw0) * ww + x - xw0];
                            const float c2 = __fmul_rn(2.f, c);
                            m = __fadd_rn(fabsf(__fsub_rn(__fsub_rn(c2, l), r)), fabsf(__fsub_rn(__fsub_rn(c2, u), d)));
                        }
                        rs = __fadd_rn(rs, m);
                    }
                    o = __fadd_rn(o, rs);
                }
                lsb_st<SS>((SS*)a.slice + ((size_t)k * a.dh + cy) * a.dw + cx, __fdiv_rn(o, (float)((py1 - py0) * (px1 - px0))));
            }
    }
    __syncthreads();
    // columns (pyramid.rs:104) -> G_{l+1}
    const float2 sc = make_float2(a.xf[k].gscale, a.xf[k].ginv);
    for (int i = ty; i < oh; i += 8) {
        const int cy = 2 * (gy0 + i);
        const int r0 = cy - 2 - yw0, r1 = r0 + 1, r2 = r0 + 2, r3 = r0 + 3, r4 = r0 + 4;
        for (int j = tx; j < ow; j += 32) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float* col = tmph + c * RGH * RW + j;
                const float v = lsb_tap5(col[r0 * RW], col[r1 * RW], col[r2 * RW], col[r3 * RW], col[r4 * RW]);
                Store<GS>::st((GS*)a.dst_g + (((size_t)k * 3 + c) * H1 + gy0 + i) * W1 + gx0 + j, v, sc);
            }
        }
    }
#undef RX
#undef RY
}

template <int SRC, class GS, bool FOCUS, class SS>
__global__ void __launch_bounds__(NT, LSB_RED_MINB) reduce_level_kernel(const FoldArgs a) {
    extern __shared__ float sm[];
    const int tiles_x = (a.W1 + RW - 1) / RW;  // the level-0 64x32 tiles' grid
    const int tile = a.fused0 ? fold0_border_tile(blockIdx.x, tiles_x, fold0_range(a.W, a.H, a.f0r)) : (int)blockIdx.x;
    const int gx0 = (tile % tiles_x) * RW, gy0 = (tile / tiles_x) * RH;
    const int k = a.red_k0 + (int)blockIdx.y;
    const bool interior = 2 * gx0 - FOC_R >= 0 && 2 * gx0 + 2 * RW + FOC_R <= a.W && 2 * gy0 - FOC_R >= 0 &&
                          2 * gy0 + 2 * RH + FOC_R <= a.H;
    if (interior) reduce_tile<SRC, GS, FOCUS, SS, true>(a, sm, k, gx0, gy0);
    else reduce_tile<SRC, GS, FOCUS, SS, false>(a, sm, k, gx0, gy0);
}

// ------------------------------------------------------------------ select
template <int R>
struct InTile {  // interior-tile window sizes (x0, y0 multiples of TW, TH)
    static constexpr int LW = TW + 2 * R, LH = TH + 2 * R;
    static constexpr int AW = ((TW + R - 1) >> 1) + ((R + 1) >> 1) + 3;
    static constexpr int AH = ((TH + R - 1) >> 1) + ((R + 1) >> 1) + 3;
};
struct TileWin {
    int x0, y0, xL0, xL1, yL0, yL1, xA0, xA1, yA0, yA1, lw, lh, aw, ah, ox1, oy1;
};

template <int SRC, class GS, int R, bool IN, bool STAGED = false>
__device__ __forceinline__ void select_frame(const FoldArgs& a, float* __restrict__ sm, int k, const TileWin& t,
                                             float (&best)[PPT], float (&acc)[PPT][3], int (&win)[PPT]) {
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int W = a.W, H = a.H, W1 = a.W1, H1 = a.H1;
#define RX(i) (IN ? (i) : lsb_reflect((i), W))
#define RY(i) (IN ? (i) : lsb_reflect((i), H))
#define RX1(i) (IN ? (i) : lsb_reflect((i), W1))
#define RY1(i) (IN ? (i) : lsb_reflect((i), H1))
    float* gl = sm;                      // [3][lh][lw]   G_l over the tile +- R
    float* g1 = gl + 3 * SEL_GL;         // [3][ah][aw]   G_{l+1} as stored
    float* exph = g1 + 3 * SEL_G1;       // [3][ah][lw]   EXPAND along rows
    float* yb = exph + 3 * SEL_EXP;      // [lh][lw]      node energy
    // staged tiles are interior: their window sizes and extents are the compile-time ones
    const int lw = STAGED ? InTile<R>::LW : t.lw, lh = STAGED ? InTile<R>::LH : t.lh;
    const int aw = STAGED ? InTile<R>::AW : t.aw, ah = STAGED ? InTile<R>::AH : t.ah;
    const int ox1 = STAGED ? TW : t.ox1, oy1 = STAGED ? TH : t.oy1;
    const float2 sc = make_float2(a.xf[k].gscale, a.xf[k].ginv);

    // ---- 1: stage G_l and G_{l+1} (STAGED: already in gl / g1 from the async copies)
    if (!STAGED) {
    for (int r = ty; r < lh; r += 8)
        for (int c = tx; c < lw; c += 32) {
            float v[3];
            level_px<SRC, GS>(a, k, t.xL0 + c, t.yL0 + r, v);
            const int i = r * lw + c;
            gl[i] = v[0];
            gl[SEL_GL + i] = v[1];
            gl[2 * SEL_GL + i] = v[2];
        }
    {
        const GS* f = (const GS*)a.dst_g + (size_t)k * 3 * W1 * H1;
        for (int c = 0; c < 3; c++)
            for (int r = ty; r < ah; r += 8) {
                const GS* row = f + ((size_t)c * H1 + t.yA0 + r) * W1 + t.xA0;
                for (int x = tx; x < aw; x += 32) g1[c * SEL_G1 + r * aw + x] = Store<GS>::ld(row + x, sc);
            }
    }
    __syncthreads();
    }

    // ---- 2: EXPAND along rows (pyramid.rs:147), the ah x lw outputs spread over all threads
    for (int m = threadIdx.x; m < ah * lw; m += NT) {
        const int i = m / lw, xi = m - i * lw;
        {
            const int x = t.xL0 + xi, cx = x >> 1;
            const bool even = (x & 1) == 0;
            const int ja = RX1(cx - 1) - t.xA0, jb = RX1(cx) - t.xA0, jc = RX1(cx + 1) - t.xA0;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float* row = g1 + c * SEL_G1 + i * aw;
                exph[c * SEL_EXP + i * lw + xi] = even ? lsb_exp_even(row[ja], row[jb], row[jc]) : lsb_exp_odd(row[jb], row[jc]);
            }
        }
    }
    __syncthreads();

    // ---- 3: EXPAND along columns, L = G - EXPAND(G_{l+1}), node energy (fuse.rs:152)
    auto lpoint = [&](int x, int y, float L[3]) -> float {
        const int xi = x - t.xL0, cy = y >> 1;
        const bool even = (y & 1) == 0;
        const int ra = (RY1(cy - 1) - t.yA0) * lw, rb = (RY1(cy) - t.yA0) * lw, rc = (RY1(cy + 1) - t.yA0) * lw;
        const int gi = (y - t.yL0) * lw + xi;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float* col = exph + c * SEL_EXP + xi;
            const float up = even ? lsb_exp_even(col[ra], col[rb], col[rc]) : lsb_exp_odd(col[rb], col[rc]);
            L[c] = __fsub_rn(gl[c * SEL_GL + gi], up);
        }
        if (a.use_chroma) return __fadd_rn(__fadd_rn(__fmul_rn(L[0], L[0]), __fmul_rn(L[1], L[1])), __fmul_rn(L[2], L[2]));
        const float Y = lsb_luma(L[0], L[1], L[2]);
        return __fmul_rn(Y, Y);
    };
    float Lr[PPT][3];
#pragma unroll
    for (int j = 0; j < PPT; j++) {
        const int px = tx + 32 * (j & 1), py = ty + 8 * (j >> 1);
        Lr[j][0] = Lr[j][1] = Lr[j][2] = 0.f;
        if (px < ox1 && py < oy1) {
            const int x = t.x0 + px, y = t.y0 + py;
            yb[(y - t.yL0) * lw + x - t.xL0] = lpoint(x, y, Lr[j]);
        }
    }
    if (R > 0 && a.halo_mode != 2) {
        // the window's halo ring around the tile, energy only, spread over all threads:
        // the full-width rows above and below the tile, then the columns beside its rows
        const int left = t.x0 - t.xL0, right = t.xL1 - (t.x0 + ox1), side = left + right;
        const int top = t.y0 - t.yL0, bot = lh - top - oy1;
        for (int m = threadIdx.x; m < (top + bot) * lw; m += NT) {
            const int rr = m / lw, xi = m - rr * lw;
            const int yi = rr < top ? rr : oy1 + rr;
            float L[3];
            yb[yi * lw + xi] = lpoint(t.xL0 + xi, t.yL0 + yi, L);
        }
        for (int m = threadIdx.x; m < oy1 * side; m += NT) {
            const int rr = m / side, c = m - rr * side;
            const int xi = c < left ? c : (lw - right) + (c - left);
            float L[3];
            yb[(top + rr) * lw + xi] = lpoint(t.xL0 + xi, t.yL0 + top + rr, L);
        }
    }
    __syncthreads();

    // ---- 4: the binomial window (fuse.rs:168) along rows, then columns + the selection
    if (a.halo_mode == 2) {
        // halo control below the guide (fuse.rs:466-470): acc = L * w for the first frame,
        // then acc += w * L; best = the sum of the weights
#pragma unroll
        for (int j = 0; j < PPT; j++) {
            const int px = tx + 32 * (j & 1), py = ty + 8 * (j >> 1);
            if (px >= ox1 || py >= oy1) continue;
            const float wv = a.halo_w[((size_t)k * H + t.y0 + py) * W + t.x0 + px];
#pragma unroll
            for (int c = 0; c < 3; c++) acc[j][c] = k == 0 ? __fmul_rn(Lr[j][c], wv) : __fadd_rn(acc[j][c], __fmul_rn(wv, Lr[j][c]));
            best[j] = k == 0 ? wv : __fadd_rn(best[j], wv);
        }
        __syncthreads();
        return;
    }
    float* eh = exph;
    if (R > 0) {
        for (int m = threadIdx.x; m < lh * ox1; m += NT) {  // the lh x ox1 row sums over all threads
            const int r = m / ox1, xo = m - r * ox1;
            {
                const float* row = yb + r * lw - t.xL0;
                float s = 0.f;
#pragma unroll
                for (int q = 0; q <= 2 * R; q++) s = __fadd_rn(s, __fmul_rn(binw<R>(q), row[RX(t.x0 + xo + q - R)]));
                eh[r * TW + xo] = s;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < PPT; j++) {
        const int px = tx + 32 * (j & 1), py = ty + 8 * (j >> 1);
        if (px >= ox1 || py >= oy1) continue;
        float e;
        if (R > 0) {
            e = 0.f;
#pragma unroll
            for (int q = 0; q <= 2 * R; q++) e = __fadd_rn(e, __fmul_rn(binw<R>(q), eh[(RY(t.y0 + py + q - R) - t.yL0) * TW + px]));
        } else {
            e = yb[(py + t.y0 - t.yL0) * lw + px + t.x0 - t.xL0];
        }
        if (a.halo_mode == 1) a.halo_w[((size_t)k * H + t.y0 + py) * W + t.x0 + px] = halo_weight(e, a.halo_p);
        if (e > best[j]) {
            best[j] = e;
            acc[j][0] = Lr[j][0];
            acc[j][1] = Lr[j][1];
            acc[j][2] = Lr[j][2];
            win[j] = k;
        }
    }
    __syncthreads();  // the next frame restages gl / g1 / exph
#undef RX
#undef RY
#undef RX1
#undef RY1
}

// ------------------------------------------------------- async tile staging
// For interior tiles the next frame's window rows (G_l over the tile +- R, and
// G_{l+1} over what EXPAND reads) are copied global -> shared with cp.async
// while the current frame computes, so the loads' latency is off the critical
// path. Rows are copied as 4-byte words from the word boundary at or before
// the row's first byte (`mis` bytes of slack in front); every fold input is
// allocated with 64 bytes of tail padding for the word after a row's end.
template <int SRC, class GS, int R>
struct Staging {
    static constexpr bool INTERLEAVED = SRC == SRC_U16;
    static constexpr int G0_EB = SRC == SRC_U16 ? 6 : (SRC == SRC_F32 ? 4 : (int)sizeof(GS));  // bytes per px in a row
    static constexpr int G0_ROWS = INTERLEAVED ? InTile<R>::LH : 3 * InTile<R>::LH;
    static constexpr int G0_WPR = (InTile<R>::LW * G0_EB + 2 + 3) / 4;  // words per row, with 2 bytes of slack
    static constexpr int G1_ROWS = 3 * InTile<R>::AH;
    static constexpr int G1_WPR = (InTile<R>::AW * (int)sizeof(GS) + 2 + 3) / 4;
    static constexpr int WORDS = G0_ROWS * G0_WPR + G1_ROWS * G1_WPR;  // one stage
    // two stages beside the compute buffers, if two CTAs still fit an SM
    static constexpr bool ON = SRC != SRC_F32 && sizeof(GS) == 2 && (2 * WORDS + SEL_FLOATS) * 4 <= 110 * 1024;
    static constexpr size_t SMEM = (size_t)(SEL_FLOATS + (ON ? 2 * WORDS : 0)) * 4;
};


// Issue the copies of frame k's interior window into `raw` (one stage).
template <int SRC, class GS, int R>
__device__ __forceinline__ void stage_issue(const FoldArgs& a, int k, const TileWin& t, uint32_t* raw) {
    using S = Staging<SRC, GS, R>;
    const int W = a.W, H = a.H, W1 = a.W1, H1 = a.H1;
    const size_t np = (size_t)W * H, np1 = (size_t)W1 * H1;
    for (int i = threadIdx.x; i < S::G0_ROWS * S::G0_WPR; i += NT) {
        const int row = i / S::G0_WPR, wd = i - row * S::G0_WPR;
        size_t byte;
        if (SRC == SRC_U16) {
            byte = (((size_t)k * np + (size_t)(t.yL0 + row) * W + t.xL0) * 3) * 2;
        } else {
            const int c = row / InTile<R>::LH, r = row - c * InTile<R>::LH;
            byte = ((((size_t)k * 3 + c) * H + t.yL0 + r) * W + t.xL0) * sizeof(GS);
        }
        const unsigned char* base = SRC == SRC_U16 ? (const unsigned char*)a.src_u16 : (const unsigned char*)a.src_g;
        cp_async4(raw + i, base + (byte & ~(size_t)3) + 4 * wd);
    }
    uint32_t* raw1 = raw + S::G0_ROWS * S::G0_WPR;
    for (int i = threadIdx.x; i < S::G1_ROWS * S::G1_WPR; i += NT) {
        const int row = i / S::G1_WPR, wd = i - row * S::G1_WPR;
        const int c = row / InTile<R>::AH, r = row - c * InTile<R>::AH;
        const size_t byte = ((((size_t)k * 3 + c) * H1 + t.yA0 + r) * W1 + t.xA0) * sizeof(GS);
        cp_async4(raw1 + i, (const unsigned char*)a.dst_g + (byte & ~(size_t)3) + 4 * wd);
    }
    (void)np1;
}
// The staged words of frame k -> the f32 windows gl / g1 select_frame reads
// (level_px's conversion and gains, Store<GS>::ld for the stored levels).
template <int SRC, class GS, int R>
__device__ __forceinline__ void stage_convert(const FoldArgs& a, int k, const TileWin& t, const uint32_t* raw, float* sm) {
    using S = Staging<SRC, GS, R>;
    using T = InTile<R>;
    const int W = a.W, H = a.H, W1 = a.W1, H1 = a.H1;
    const size_t np = (size_t)W * H;
    float* gl = sm;
    float* g1 = gl + 3 * SEL_GL;
    const float2 sc = make_float2(a.xf[k].gscale, a.xf[k].ginv);
    int gon = 0;
    float gain[3] = {1.f, 1.f, 1.f};
    if (SRC == SRC_U16) {
        gon = a.xf[k].gain_on;
        for (int c = 0; c < 3; c++) gain[c] = a.xf[k].gain[c];
    }
    for (int i = threadIdx.x; i < T::LH * T::LW; i += NT) {
        const int r = i / T::LW, x = i - r * T::LW;
        float v[3];
        if (SRC == SRC_U16) {
            const size_t byte = (((size_t)k * np + (size_t)(t.yL0 + r) * W + t.xL0) * 3) * 2;
            const uint16_t* p = (const uint16_t*)((const unsigned char*)(raw + r * S::G0_WPR) + (byte & 3)) + 3 * x;
            for (int c = 0; c < 3; c++) {
                v[c] = __fmul_rn((float)p[c], LSB_INV16);
                if (gon & (1 << c)) v[c] = __fmul_rn(v[c], gain[c]);
            }
        } else {
            for (int c = 0; c < 3; c++) {
                const size_t byte = ((((size_t)k * 3 + c) * H + t.yL0 + r) * W + t.xL0) * sizeof(GS);
                const GS* p = (const GS*)((const unsigned char*)(raw + (c * T::LH + r) * S::G0_WPR) + (byte & 3)) + x;
                v[c] = Store<GS>::ld(p, sc);
            }
        }
        const int o = r * T::LW + x;
        gl[o] = v[0];
        gl[SEL_GL + o] = v[1];
        gl[2 * SEL_GL + o] = v[2];
    }
    const uint32_t* raw1 = raw + S::G0_ROWS * S::G0_WPR;
    for (int i = threadIdx.x; i < 3 * T::AH * T::AW; i += NT) {
        const int c = i / (T::AH * T::AW), rem = i - c * (T::AH * T::AW), r = rem / T::AW, x = rem - r * T::AW;
        const size_t byte = ((((size_t)k * 3 + c) * H1 + t.yA0 + r) * W1 + t.xA0) * sizeof(GS);
        const GS* p = (const GS*)((const unsigned char*)(raw1 + (c * T::AH + r) * S::G1_WPR) + (byte & 3)) + x;
        g1[c * SEL_G1 + r * T::AW + x] = Store<GS>::ld(p, sc);
    }
}

template <int SRC, class GS, int R>
__global__ void __launch_bounds__(NT, LSB_SEL_MINB) select_level_kernel(const FoldArgs a) {
    extern __shared__ float sm[];
    const int W = a.W, H = a.H, W1 = a.W1, H1 = a.H1;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int G = a.sel_groups > 1 ? a.sel_groups : 1;
    for (int wi = blockIdx.x; wi < a.ntiles * G; wi += gridDim.x) {
        const int tile = a.fused0 ? fold0_border_tile(wi % a.ntiles, a.tiles_x, fold0_range(W, H, a.f0r)) : wi % a.ntiles;
        const int g = wi / a.ntiles;
        const int k0 = G > 1 ? a.sel_k0 + (a.sel_k1 - a.sel_k0) * g / G : a.sel_k0;
        const int k1 = G > 1 ? a.sel_k0 + (a.sel_k1 - a.sel_k0) * (g + 1) / G : a.sel_k1;
        TileWin t;
        t.x0 = (tile % a.tiles_x) * TW;
        t.y0 = (tile / a.tiles_x) * TH;
        const int uxL0 = t.x0 - R, uxL1 = t.x0 + TW + R, uyL0 = t.y0 - R, uyL1 = t.y0 + TH + R;
        const bool interior = ((uxL0 >> 1) - 1) >= 0 && uxL1 <= W && ((uxL1 - 1) >> 1) + 2 <= W1 && ((uyL0 >> 1) - 1) >= 0 &&
                              uyL1 <= H && ((uyL1 - 1) >> 1) + 2 <= H1;
        t.xL0 = max(0, uxL0);
        t.xL1 = min(W, uxL1);
        t.yL0 = max(0, uyL0);
        t.yL1 = min(H, uyL1);
        t.xA0 = max(0, (t.xL0 >> 1) - 1);
        t.xA1 = min(W1, ((t.xL1 - 1) >> 1) + 2);
        t.yA0 = max(0, (t.yL0 >> 1) - 1);
        t.yA1 = min(H1, ((t.yL1 - 1) >> 1) + 2);
        t.lw = t.xL1 - t.xL0;
        t.lh = t.yL1 - t.yL0;
        t.aw = t.xA1 - t.xA0;
        t.ah = t.yA1 - t.yA0;
        t.ox1 = min(TW, W - t.x0);
        t.oy1 = min(TH, H - t.y0);
        if (t.lw > LW_MAX || t.lh > LH_MAX || t.aw > AW_MAX || t.ah > AH_MAX) {
            if (threadIdx.x == 0) atomicOr(a.status, LSB_ERR_SHAPE);
            return;
        }
        float best[PPT], acc[PPT][3];
        int win[PPT];
#pragma unroll
        for (int j = 0; j < PPT; j++) {
            best[j] = -1.f;  // any energy (>= 0) beats it: frame 0 fills the accumulator (fuse.rs:409-412)
            acc[j][0] = acc[j][1] = acc[j][2] = 0.f;
            win[j] = 0;
            const int px = tx + 32 * (j & 1), py = ty + 8 * (j >> 1);
            if (g == 0 && a.sel_k0 > 0 && px < t.ox1 && py < t.oy1) {  // resume: the state the frames before left
                const size_t o = (size_t)(t.y0 + py) * W + t.x0 + px;
                acc[j][0] = a.acc[o];
                acc[j][1] = a.acc[(size_t)W * H + o];
                acc[j][2] = a.acc[2 * (size_t)W * H + o];
                best[j] = a.best[o];
                if (a.winner) win[j] = a.winner[o];
            }
        }
        using S = Staging<SRC, GS, R>;
        if (S::ON && interior) {
            if (t.lw != InTile<R>::LW || t.lh != InTile<R>::LH || t.aw != InTile<R>::AW || t.ah != InTile<R>::AH) {
                if (threadIdx.x == 0) atomicOr(a.status, LSB_ERR_SHAPE);
                return;
            }
            uint32_t* raw = (uint32_t*)(sm + SEL_FLOATS);
            stage_issue<SRC, GS, R>(a, k0, t, raw);
            cp_async_commit();
            for (int k = k0; k < k1; k++) {
                uint32_t* cur = raw + ((k - k0) & 1) * S::WORDS;
                if (k + 1 < k1) {
                    stage_issue<SRC, GS, R>(a, k + 1, t, raw + ((k + 1 - k0) & 1) * S::WORDS);
                    cp_async_commit();
                    cp_async_wait<1>();
                } else {
                    cp_async_wait<0>();
                }
                __syncthreads();
                stage_convert<SRC, GS, R>(a, k, t, cur, sm);
                __syncthreads();
                select_frame<SRC, GS, R, true, true>(a, sm, k, t, best, acc, win);
            }
        } else {
            for (int k = k0; k < k1; k++) {
                if (interior) select_frame<SRC, GS, R, true>(a, sm, k, t, best, acc, win);
                else select_frame<SRC, GS, R, false>(a, sm, k, t, best, acc, win);
            }
        }
#pragma unroll
        for (int j = 0; j < PPT; j++) {
            const int px = tx + 32 * (j & 1), py = ty + 8 * (j >> 1);
            if (px >= t.ox1 || py >= t.oy1) continue;
            const size_t o = (size_t)(t.y0 + py) * W + t.x0 + px, np = (size_t)W * H;
            if (G > 1) {  // this group's state, merged by select_merge_kernel
                float* ga = a.gacc + (size_t)g * 3 * np;
                ga[o] = acc[j][0];
                ga[np + o] = acc[j][1];
                ga[2 * np + o] = acc[j][2];
                a.gbest[(size_t)g * np + o] = best[j];
                a.gwin[(size_t)g * np + o] = win[j];
                continue;
            }
            a.acc[o] = acc[j][0];
            a.acc[np + o] = acc[j][1];
            a.acc[2 * np + o] = acc[j][2];
            a.best[o] = best[j];
            if (a.winner) a.winner[o] = (uint16_t)win[j];
        }
    }
}

// --------------------------------------------------------------------- warp
// align.rs:489 `warp_with` of every aligned frame (stack.rs:662-679: the pixel
// as shot where the source point leaves the frame), written once: f32 planar
// (FP32 storage) or u16 interleaved (16-bit storage, rounded to the u16 step).
template <bool U16OUT>
__global__ void __launch_bounds__(NT) warp_frames_kernel(const uint16_t* __restrict__ frames, const FrameXform* __restrict__ xf,
                                                         int interp, int W, int H, void* __restrict__ out) {
    const int k = blockIdx.z;
    const int x = blockIdx.x * 32 + (threadIdx.x & 31), y = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (x >= W || y >= H) return;
    const size_t np = (size_t)W * H;
    const FrameXform X = xf[k];
    float v[3];
    load_px_core(frames + (size_t)k * np * 3, X.inv, X.warp, X.affine, interp, W, H, x, y, v);
    const size_t o = (size_t)y * W + x;
    if (U16OUT) {
        uint16_t* p = (uint16_t*)out + ((size_t)k * np + o) * 3;
        for (int c = 0; c < 3; c++) p[c] = (uint16_t)fminf(fmaxf(__fadd_rn(__fmul_rn(v[c], 65535.f), 0.5f), 0.f), 65535.f);
    } else {
        float* p = (float*)out + (size_t)k * 3 * np + o;
        p[0] = v[0];
        p[np] = v[1];
        p[2 * np] = v[2];
    }
}

// The same warp for the Spline4x4 kernel (align.rs:416, the default) over
// 64x16 output tiles: the tile's source footprint (the images of its corners,
// the taps' reach and a pixel of margin, clamped to the frame like the taps) is converted
// to f32 once into shared memory, so each source sample is read and scaled
// once instead of by every one of the 16 output pixels whose taps reach it.
// The taps, weights and sums are those of load_px_core, in its order; a tile
// whose footprint does not fit (a large rotation or magnification) takes the
// direct path.
constexpr int WT_W = 64, WT_H = 16, WB_W = WT_W + 16, WB_H = WT_H + 16;
template <bool U16OUT>
__global__ void __launch_bounds__(NT) warp_tile_kernel(const uint16_t* __restrict__ frames, const FrameXform* __restrict__ xf, int W,
                                                       int H, void* __restrict__ out) {
    __shared__ float4 box[WB_H][WB_W];
    const int k = blockIdx.z, x0 = blockIdx.x * WT_W, y0 = blockIdx.y * WT_H;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const size_t np = (size_t)W * H;
    const uint16_t* f = frames + (size_t)k * np * 3;
    const FrameXform X = xf[k];
    int bx0 = 0, by0 = 0, bw = 0, bh = 0;
    bool fits = false;
    if (X.warp) {
        double mnx = 1e300, mxx = -1e300, mny = 1e300, mxy = -1e300;
        const int cx[2] = {x0, min(x0 + WT_W - 1, W - 1)}, cy[2] = {y0, min(y0 + WT_H - 1, H - 1)};
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) {
                double sx, sy;
                const double* m = X.inv;
                const double xd = (double)cx[a], yd = (double)cy[b];
                if (X.affine) {
                    sx = __dadd_rn(__dadd_rn(__dmul_rn(m[1], yd), m[2]), __dmul_rn(m[0], xd));
                    sy = __dadd_rn(__dadd_rn(__dmul_rn(m[4], yd), m[5]), __dmul_rn(m[3], xd));
                } else {
                    const double d = __dadd_rn(__dadd_rn(__dmul_rn(m[6], xd), __dmul_rn(m[7], yd)), m[8]);
                    sx = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[0], xd), __dmul_rn(m[1], yd)), m[2]), d);
                    sy = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[3], xd), __dmul_rn(m[4], yd)), m[5]), d);
                }
                mnx = fmin(mnx, sx);
                mxx = fmax(mxx, sx);
                mny = fmin(mny, sy);
                mxy = fmax(mxy, sy);
            }
        // only affine footprints are the corners' hull for sure; projective tiles go direct
        if (X.affine && mnx > -1e9 && mxx < 1e9 && mny > -1e9 && mxy < 1e9) {
            // one pixel of margin each side: an inner pixel's rounded source point may pass a corner's by an ulp
            bx0 = (int)floor(mnx) - 2;
            by0 = (int)floor(mny) - 2;
            bw = (int)floor(mxx) + 3 - bx0 + 1;
            bh = (int)floor(mxy) + 3 - by0 + 1;
            fits = bw <= WB_W && bh <= WB_H;
        }
    }
    if (fits) {
        // the footprint's elements over all threads; m / bw by a multiply (exact for m < 2^16, bw <= 80)
        const unsigned magic = (unsigned)((0xffffffffull + bw) / bw);
        for (int m = threadIdx.x; m < bw * bh; m += NT) {
            const int r = (int)__umulhi((unsigned)m, magic), c = m - r * bw;
            const uint16_t* p = f + ((size_t)min(max(by0 + r, 0), H - 1) * W + min(max(bx0 + c, 0), W - 1)) * 3;
            box[r][c] = make_float4(__fmul_rn((float)p[0], LSB_INV16), __fmul_rn((float)p[1], LSB_INV16),
                                    __fmul_rn((float)p[2], LSB_INV16), 0.f);
        }
        __syncthreads();
    }
#pragma unroll 1
    for (int q = 0; q < 4; q++) {
        const int x = x0 + tx + 32 * (q & 1), y = y0 + ty + 8 * (q >> 1);
        if (x >= W || y >= H) continue;
        float v[3];
        if (fits) {
            const double* m = X.inv;
            const double xd = (double)x, yd = (double)y;
            const double sx = __dadd_rn(__dadd_rn(__dmul_rn(m[1], yd), m[2]), __dmul_rn(m[0], xd));
            const double sy = __dadd_rn(__dadd_rn(__dmul_rn(m[4], yd), m[5]), __dmul_rn(m[3], xd));
            if (sx >= 0.0 && sx <= (double)(W - 1) && sy >= 0.0 && sy <= (double)(H - 1)) {
                const double fx = floor(sx), fy = floor(sy);
                const int ix = (int)fx - 1 - bx0, iy = (int)fy - 1 - by0;
                float wx[4], wy[4];
                spline4_d(__dsub_rn(sx, fx), wx);
                spline4_d(__dsub_rn(sy, fy), wy);
                float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    float r0 = 0.f, r1 = 0.f, r2 = 0.f;
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const float4 s4 = box[iy + j][ix + i];
                        r0 = __fadd_rn(r0, __fmul_rn(wx[i], s4.x));
                        r1 = __fadd_rn(r1, __fmul_rn(wx[i], s4.y));
                        r2 = __fadd_rn(r2, __fmul_rn(wx[i], s4.z));
                    }
                    a0 = __fadd_rn(a0, __fmul_rn(wy[j], r0));
                    a1 = __fadd_rn(a1, __fmul_rn(wy[j], r1));
                    a2 = __fadd_rn(a2, __fmul_rn(wy[j], r2));
                }
                v[0] = a0;
                v[1] = a1;
                v[2] = a2;
            } else {
                const uint16_t* p = f + ((size_t)y * W + x) * 3;
                for (int c = 0; c < 3; c++) v[c] = __fmul_rn((float)p[c], LSB_INV16);
            }
        } else {
            load_px_core(f, X.inv, X.warp, X.affine, 3, W, H, x, y, v);
        }
        const size_t o = (size_t)y * W + x;
        if (U16OUT) {
            uint16_t* p = (uint16_t*)out + ((size_t)k * np + o) * 3;
            for (int c = 0; c < 3; c++) p[c] = (uint16_t)fminf(fmaxf(__fadd_rn(__fmul_rn(v[c], 65535.f), 0.5f), 0.f), 65535.f);
        } else {
            float* p = (float*)out + (size_t)k * 3 * np + o;
            p[0] = v[0];
            p[np] = v[1];
            p[2 * np] = v[2];
        }
    }
}

