// The level-0 fold in ONE kernel (included by lsb_fold.cu inside namespace
// lsb, after lsb_level.cuh).
//
// reduce_level_kernel + select_level_kernel read every level-0 frame from HBM
// twice (once to REDUCE it to G_1 and take its focus slice, once to select
// its Laplacian coefficients). fold0_kernel does both from one staged copy of
// the frame: a CTA owns a 64x32 tile of level 0 and walks the frames in
// order; for each frame it
//   1. copies the tile's u16 window (tile + 6..7 px) into shared memory with
//      one bulk copy per row (cp.async.bulk, completion on an mbarrier; the
//      next frame's copy is issued as soon as this one is converted),
//   2. converts it to f32 planes with the frame's gains and takes its luma,
//   3. runs the ring difference filter and the 2x2 block mean (the focus slice,
//      depth.rs:1097 / :417 / :174),
//   4. REDUCEs the window to G_1 over what EXPAND needs (pyramid.rs:86) and
//      writes the tile's own G_1 in the storage type,
//   5. EXPANDs back, forms L = G - EXPAND(G_1 as stored) in place of G and the
//      luma energy (fuse.rs:152); each thread takes the binomial window
//      (fuse.rs:168) of the pixels it owns and keeps their strict-> selection
//      (fuse.rs:429) in registers.
// The arithmetic is the reference's, op for op and in its order (round-to-
// nearest f32 adds and multiplies, never contracted); pairs of independent
// results (two rows, or two neighbouring pixels) go through one packed
// f32x2 instruction, which rounds each lane exactly as the scalar op would.
// The results are therefore bit-identical to the two-kernel path, which stays
// for the tiles whose window reaches the frame border.
#pragma once

// ------------------------------------------------------------ f32x2 helpers
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2,%3};\n\tmov.b64 rb, {%4,%5};\n\tadd.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0,%1}, rd;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2,%3};\n\tmov.b64 rb, {%4,%5};\n\tsub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0,%1}, rd;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2,%3};\n\tmov.b64 rb, {%4,%5};\n\tmul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0,%1}, rd;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 splat(float v) { return make_float2(v, v); }
// ptxas contracts a packed multiply that feeds a packed add into one fused multiply-add, whatever
// the .rn modifiers, which changes the rounding. So a packed add follows a packed multiply only when
// the product is exact (a power-of-two factor: 1/16, 1/4, 1/8, 1/2, where contraction changes
// nothing); an inexact product is added lane by lane, with scalar round-to-nearest adds.
__device__ __forceinline__ float2 addl(float2 a, float2 p) { return make_float2(__fadd_rn(a.x, p.x), __fadd_rn(a.y, p.y)); }
// pyramid.rs:95 tap5 on two independent lanes (K0 = 1/16, K1 = 1/4 exact; K2 = 6/16 not)
__device__ __forceinline__ float2 tap5x2(float2 s0, float2 s1, float2 s2, float2 s3, float2 s4) {
    float2 a = mul2(splat(LSB_K0), s0);
    a = add2(a, mul2(splat(LSB_K1), s1));
    a = addl(a, mul2(splat(LSB_K2), s2));
    a = add2(a, mul2(splat(LSB_K1), s3));
    return add2(a, mul2(splat(LSB_K0), s4));
}
// pyramid.rs:128-166 EXPAND taps on two lanes (E0 = 1/8 and OD = 1/2 exact; E1 = 3/4 not)
__device__ __forceinline__ float2 exp_even2(float2 a, float2 b, float2 c) {
    return add2(addl(mul2(splat(LSB_E0), a), mul2(splat(LSB_E1), b)), mul2(splat(LSB_E0), c));
}
__device__ __forceinline__ float2 exp_odd2(float2 a, float2 b) { return mul2(splat(LSB_OD), add2(a, b)); }
// fuse.rs:160 luma on two lanes (no weight is a power of two)
__device__ __forceinline__ float2 luma2(float2 r, float2 g, float2 b) {
    return addl(addl(mul2(splat(0.299f), r), mul2(splat(0.587f), g)), mul2(splat(0.114f), b));
}
// w * v added to s, the product exact when w is a power of two
template <bool EXACT>
__device__ __forceinline__ float2 acc2(float2 s, float w, float2 v) {
    return EXACT ? add2(s, mul2(splat(w), v)) : addl(s, mul2(splat(w), v));
}
// binw<R>(q) is a power of two except 6/16 (R = 2, q = 2)
template <int R>
__device__ __forceinline__ constexpr bool binw_exact(int q) {
    return !(R == 2 && q == 2);
}

// ------------------------------------------------- bulk copies on an mbarrier
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* m) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(m)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect(uint64_t* m, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}
// global -> this CTA's shared memory, 16-byte aligned addresses, size a multiple of 16 (no multicast)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(m))
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* m, unsigned parity) {
    unsigned ok;
    asm volatile("{.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;}"
                 : "=r"(ok)
                 : "r"(smem_u32(m)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// Waits for phase `parity` of m; gives up after `limit` polls (each try_wait itself blocks for a
// while), returning false. The copies it waited for may then still be in flight.
__device__ __forceinline__ bool mbar_wait(uint64_t* m, unsigned parity, unsigned limit) {
    for (unsigned i = 0; i < limit; i++)
        if (mbar_test(m, parity)) return true;
    return false;
}

// ---------------------------------------------------------------- geometry
// Tile 64x32 of level 0, 256 threads. The u16 window spans columns
// x0 - 6 - (R & 1) .. +76 and rows y0 - 6 .. +44: every G_1 value EXPAND reads
// at the tile +- R (columns x0/2 - 2 .. +36, rows y0/2 - 2 .. +20), the ring
// difference filter's reach (3 px) and the Laplacian at the tile +- R. The
// odd-R column shift keeps the Laplacian's pixel pairs 8-byte aligned.
namespace f0 {
constexpr int TW0 = 64, TH0 = 32, NT0 = 256;
constexpr int WW = 76, WH = 44;          // u16 window
constexpr int RAW_ROW = 480;             // bytes per staged row: 76 * 6 + up to 14 of slack, to 16
constexpr int G1W = 40, G1H = 20;        // G_1 over what EXPAND reads (36 used; 40 keeps reads in bounds)
constexpr int LYW = 72, LYH = 38;        // luma over the filter's reach: x0-3 .., y0-3 ..
constexpr int EXW = 72;                  // EXPAND along rows: 64 + 2R columns (<= 68), 9 groups of 8
constexpr int YBW = 68, YBH = 36;        // energies over the tile +- R
// shared memory, in bytes (the luma planes are dead once the filter ran and hold the energies after;
// the row sums of REDUCE are dead once G_1 exists and hold the EXPAND row pass after)
constexpr int OFF_MBAR = 0;                                   // the copies' mbarrier
constexpr int OFF_MIS = 16;                                   // [WH] each staged row's first byte within its slot
constexpr int OFF_RAW = 192;
constexpr int OFF_G0 = OFF_RAW + WH * RAW_ROW;                 // [3][WH][WW] f32: G, then L
constexpr int OFF_LY = OFF_G0 + 3 * WH * WW * 4;               // [LYH][LYW] luma and [LYH][LYW] luma shifted by one
constexpr int OFF_YB = OFF_LY;                                 // [YBH][YBW] energies  (after the filter)
constexpr int OFF_TMP = OFF_LY + 2 * LYH * LYW * 4;            // [3][WH][36] REDUCE rows; then [3][G1H][EXW] EXPAND rows
constexpr int TMPW = 36;
constexpr int OFF_G1 = OFF_TMP + 3 * WH * TMPW * 4;            // [3][G1H][G1W] G_1 as stored
constexpr int SMEM = OFF_G1 + 3 * G1H * G1W * 4;
static_assert(OFF_YB + YBH * YBW * 4 <= OFF_TMP, "the energies fit the luma planes");
static_assert(3 * G1H * EXW <= 3 * WH * TMPW, "the EXPAND rows fit the REDUCE rows' space");
static_assert(OFF_RAW % 16 == 0 && RAW_ROW % 16 == 0, "bulk copy destinations are 16-byte aligned");
static_assert(SMEM <= 113 * 1024, "two CTAs per SM");
}  // namespace f0

// ---- phase 1: the staged u16 rows -> G (three f32 planes [WH][WW]) with the frame's gains
// (io.rs:89 v * (1/65535), brightness.rs:124), and the luma (fuse.rs:160) over the filter's reach into
// Ly [LYH][LYW] (column 0 = x0 - 3) and Ls (Ly shifted by one column: Ls[c] = Ly[c + 1]).
// Pixel pairs: 12 staged bytes -> six u16 -> three lane pairs (R, G, B of two pixels); a u16 u is
// made a float exactly as the bits 0x4B000000 | u less 2^23.
template <int R, bool FOCUS>
__device__ __forceinline__ void f0_convert(const unsigned char* __restrict__ raw, const int* __restrict__ mis, float* __restrict__ G,
                                           float* __restrict__ Ly, float* __restrict__ Ls, int gon, const float (&gain)[3]) {
    using namespace f0;
    constexpr int PPR = WW / 2;  // pixel pairs per row
    for (int it = threadIdx.x; it < WH * PPR; it += NT0) {
        const int r = it / PPR, p = it - r * PPR;
        const int byte = mis[r] + 12 * p;
        const uint32_t* w = (const uint32_t*)(raw + r * RAW_ROW + (byte & ~3));
        uint32_t w0 = w[0], w1 = w[1], w2 = w[2];
        if (byte & 2) {  // the pair starts half way into a word
            const uint32_t w3 = w[3];
            w0 = __funnelshift_r(w0, w1, 16);
            w1 = __funnelshift_r(w1, w2, 16);
            w2 = __funnelshift_r(w2, w3, 16);
        }
        const float2 m23 = splat(8388608.f);
        float2 cr = sub2(make_float2(__int_as_float(__byte_perm(w0, 0x4B00, 0x5410)), __int_as_float(__byte_perm(w1, 0x4B00, 0x5432))), m23);
        float2 cg = sub2(make_float2(__int_as_float(__byte_perm(w0, 0x4B00, 0x5432)), __int_as_float(__byte_perm(w2, 0x4B00, 0x5410))), m23);
        float2 cb = sub2(make_float2(__int_as_float(__byte_perm(w1, 0x4B00, 0x5410)), __int_as_float(__byte_perm(w2, 0x4B00, 0x5432))), m23);
        cr = mul2(cr, splat(LSB_INV16));
        cg = mul2(cg, splat(LSB_INV16));
        cb = mul2(cb, splat(LSB_INV16));
        if (gon & 1) cr = mul2(cr, splat(gain[0]));
        if (gon & 2) cg = mul2(cg, splat(gain[1]));
        if (gon & 4) cb = mul2(cb, splat(gain[2]));
        const int o = r * WW + 2 * p;
        *(float2*)(G + o) = cr;
        *(float2*)(G + WH * WW + o) = cg;
        *(float2*)(G + 2 * WH * WW + o) = cb;
        if (FOCUS && r >= 3 && r < 3 + LYH) {
            const int lc = 2 * p - 3 - (R & 1);  // the luma column of the pair's first pixel
            if (lc >= -1 && lc < 70) {
                const float2 y = luma2(cr, cg, cb);
                float* ly = Ly + (r - 3) * LYW;
                float* ls = Ls + (r - 3) * LYW;
                if (lc >= 0) ly[lc] = y.x;
                if (lc + 1 < 70) ly[lc + 1] = y.y;
                if (lc >= 1) ls[lc - 1] = y.x;
                if (lc >= 0 && lc < 68) ls[lc] = y.y;
            }
        }
    }
}

// ---- phase 2: the focus slice of the tile (depth.rs:1097): per 2x2 block of level 0, the ring
// difference filter of each pixel (depth.rs:417, taps in order, s += w * y), |.|, the row sums, their
// sum, / 4 (depth.rs:174 block_mean). Pixel pairs (x, x+1) run as lanes; a tap with odd dx reads the
// pair from Ly at an even column, one with even dx from Ls.
template <class SS>
__device__ __forceinline__ void f0_focus(const FoldArgs& a, const float* __restrict__ Ly, const float* __restrict__ Ls, int k, int x0,
                                         int y0) {
    using namespace f0;
    const float2 wd = splat(RDF_WD), wr = splat(RDF_WR);
    // depth.rs:454 rdf_taps(1, 3) in depth.rs:417 conv_sparse's order (dy, dx, ring): rdf13's table
    constexpr int T[29][3] = {{-1, 0, 0},  {-1, -2, 1}, {-1, -1, 1}, {-1, 1, 1},  {-1, 2, 1}, {0, -1, 0},  {0, 0, 0},  {0, 1, 0},
                              {0, -3, 1},  {0, -2, 1},  {0, 2, 1},   {0, 3, 1},   {1, 0, 0},  {1, -2, 1},  {1, -1, 1}, {1, 1, 1},
                              {1, 2, 1},   {-3, 0, 1},  {-2, -2, 1}, {-2, -1, 1}, {-2, 0, 1}, {-2, 1, 1},  {-2, 2, 1}, {2, -2, 1},
                              {2, -1, 1},  {2, 0, 1},   {2, 1, 1},   {2, 2, 1},   {3, 0, 1}};
#pragma unroll 1
    for (int j = 0; j < 2; j++) {
        const int cx = threadIdx.x & 31, cy = (threadIdx.x >> 5) + 8 * j;
        float o = 0.f;
#pragma unroll
        for (int dy0 = 0; dy0 < 2; dy0++) {
            const int row = 2 * cy + dy0 + 3, col = 2 * cx + 3;
            float2 s = make_float2(0.f, 0.f);
#pragma unroll
            for (int q = 0; q < 29; q++) {
                const int dy = T[q][0], dx = T[q][1];
                const float2 v = (dx & 1) ? *(const float2*)(Ly + (row + dy) * LYW + col + dx)
                                          : *(const float2*)(Ls + (row + dy) * LYW + col + dx - 1);
                const float2 t = mul2(T[q][2] ? wr : wd, v);  // 1/5, -1/24: inexact products, added lane by lane
                s = q == 0 ? t : addl(s, t);
            }
            const float rs = __fadd_rn(fabsf(s.x), fabsf(s.y));
            o = dy0 == 0 ? rs : __fadd_rn(o, rs);
        }
        lsb_st<SS>((SS*)a.slice + ((size_t)k * a.dh + (y0 >> 1) + cy) * a.dw + (x0 >> 1) + cx, __fmul_rn(o, 0.25f));
    }
}

// ---- phase 3: REDUCE along rows (pyramid.rs:90) of every window row, at the G_1 columns
// x0/2 - 2 + a, a < 36: tmp[c][r][a]. Two rows per thread as lanes; the lanes of a warp take consecutive
// outputs, so their taps (window columns 2a .. 2a + 4, read as two 8-byte pairs and one word) are
// contiguous in shared memory.
template <int R>
__device__ __forceinline__ void f0_reduce_rows(const float* __restrict__ G, float* __restrict__ tmp) {
    using namespace f0;
    constexpr int ITEMS = 3 * (WH / 2) * TMPW;
    for (int it = threadIdx.x; it < ITEMS; it += NT0) {
        const int c = it / ((WH / 2) * TMPW), rem = it - c * ((WH / 2) * TMPW);
        const int rp = rem / TMPW, a = rem - rp * TMPW;
        const int r0 = 2 * rp;
        const float* p0 = G + (c * WH + r0) * WW + 2 * a + (R & 1);
        float2 v[5];
        if (R & 1) {  // odd columns: one word, then two pairs
            v[0] = make_float2(p0[0], p0[WW]);
            const float2 a1 = *(const float2*)(p0 + 1), b1 = *(const float2*)(p0 + WW + 1);
            const float2 a3 = *(const float2*)(p0 + 3), b3 = *(const float2*)(p0 + WW + 3);
            v[1] = make_float2(a1.x, b1.x);
            v[2] = make_float2(a1.y, b1.y);
            v[3] = make_float2(a3.x, b3.x);
            v[4] = make_float2(a3.y, b3.y);
        } else {  // even columns: two pairs, then one word
            const float2 a0 = *(const float2*)(p0), b0 = *(const float2*)(p0 + WW);
            const float2 a2 = *(const float2*)(p0 + 2), b2 = *(const float2*)(p0 + WW + 2);
            v[0] = make_float2(a0.x, b0.x);
            v[1] = make_float2(a0.y, b0.y);
            v[2] = make_float2(a2.x, b2.x);
            v[3] = make_float2(a2.y, b2.y);
            v[4] = make_float2(p0[4], p0[WW + 4]);
        }
        const float2 o = tap5x2(v[0], v[1], v[2], v[3], v[4]);
        tmp[(c * WH + r0) * TMPW + a] = o.x;
        tmp[(c * WH + r0 + 1) * TMPW + a] = o.y;
    }
}

// ---- phase 4: REDUCE along columns (pyramid.rs:104) -> G_1 rows y0/2 - 2 + b, b < 20, as the storage
// type gives it back (what the next level's pass and EXPAND read), into G1s[c][b][a]; the tile's own
// 16x32 block (b in [2, 18), a in [2, 34)) is also written to HBM. Two columns per thread as lanes,
// five outputs from 13 loads.
template <class GS>
__device__ __forceinline__ void f0_reduce_cols(const FoldArgs& a, const float* __restrict__ tmp, float* __restrict__ G1s, int k, int x0,
                                               int y0, float2 sc) {
    using namespace f0;
    constexpr int ITEMS = 3 * (TMPW / 2) * 4;
    const int W1 = a.W1, H1 = a.H1;
    for (int it = threadIdx.x; it < ITEMS; it += NT0) {
        const int c = it / ((TMPW / 2) * 4), rem = it - c * ((TMPW / 2) * 4);
        const int bg = rem / (TMPW / 2), ap = rem - bg * (TMPW / 2);
        const int aa = 2 * ap, b0 = 5 * bg;
        const float* col = tmp + (c * WH + 2 * b0) * TMPW + aa;
        float2 v[13];
#pragma unroll
        for (int t = 0; t < 13; t++) v[t] = *(const float2*)(col + t * TMPW);
#pragma unroll
        for (int i = 0; i < 5; i++) {
            const int b = b0 + i;
            const float2 o = tap5x2(v[2 * i], v[2 * i + 1], v[2 * i + 2], v[2 * i + 3], v[2 * i + 4]);
            *(float2*)(G1s + (c * G1H + b) * G1W + aa) = make_float2(Store<GS>::as_stored(o.x, sc), Store<GS>::as_stored(o.y, sc));
            if (b >= 2 && b < 18 && aa >= 2 && aa < 34) {
                GS* d = (GS*)a.dst_g + (((size_t)k * 3 + c) * H1 + (y0 >> 1) - 2 + b) * W1 + (x0 >> 1) - 2 + aa;
                Store<GS>::st(d, o.x, sc);
                Store<GS>::st(d + 1, o.y, sc);
            }
        }
    }
}

// ---- phase 5: EXPAND along rows (pyramid.rs:147) of G_1 as stored: exph[c][b][x'] at level-0
// columns x0 - R + x', x' < 64 + 2R. Two G_1 rows per thread as lanes, eight outputs from eight loads;
// the last column group also takes the 2R columns past 64, so that the 240 items take one round.
template <int R>
__device__ __forceinline__ void f0_expand_rows(const float* __restrict__ G1s, float* __restrict__ exph) {
    using namespace f0;
    constexpr int NG = TW0 / 8, ITEMS = 3 * (G1H / 2) * NG;
    constexpr int A0 = R == 2 ? 0 : 1;  // the group's first G_1 column, less 4g
    for (int it = threadIdx.x; it < ITEMS; it += NT0) {
        const int c = it / ((G1H / 2) * NG), rem = it - c * ((G1H / 2) * NG);
        const int bp = rem / NG, g = rem - bp * NG;
        const int b0 = 2 * bp;
        const float* src = G1s + (c * G1H + b0) * G1W + 4 * g + A0;
        float2 u[8];
#pragma unroll
        for (int t = 0; t < 8; t++) u[t] = make_float2(src[t], src[G1W + t]);
        float* d0 = exph + (c * G1H + b0) * EXW + 8 * g;
        const int ni = g == NG - 1 ? 8 + 2 * R : 8;
#pragma unroll
        for (int i = 0; i < 8 + 2 * R; i++) {
            if (i >= ni) break;
            const int m = i - R;                   // its parity is that of the level-0 column
            const int j = ((m >> 1) + 2) - A0;     // the G_1 column of x >> 1 within u
            const float2 o = (m & 1) == 0 ? exp_even2(u[j - 1], u[j], u[j + 1]) : exp_odd2(u[j], u[j + 1]);
            d0[i] = o.x;
            d0[EXW + i] = o.y;
        }
    }
}

// ---- phase 6: EXPAND along columns, L = G - EXPAND(G_1) (pyramid.rs:209) written over G, and the
// node energy (fuse.rs:152: luma squared, or the squared channels with chroma) into yb[r][x'] over
// the tile +- R (level-0 row y0 - R + r, column x0 - R + x'). Pixel pairs as lanes.
template <int R>
__device__ __forceinline__ void f0_laplace(const float* __restrict__ exph, float* __restrict__ G, float* __restrict__ yb, int chroma) {
    using namespace f0;
    constexpr int EW = TW0 + 2 * R, EH = TH0 + 2 * R, PPR = EW / 2, ITEMS = EH * PPR;
    for (int it = threadIdx.x; it < ITEMS; it += NT0) {
        const int r = it / PPR, p = it - r * PPR, xq = 2 * p;
        const int m = r - R, b = (m >> 1) + 2;  // the G_1 row of y >> 1
        const int wr = r - R + 6, wc = xq - R + 6 + (R & 1);
        float2 L[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float* e = exph + c * G1H * EXW + xq;
            const float2 up = (m & 1) == 0 ? exp_even2(*(const float2*)(e + (b - 1) * EXW), *(const float2*)(e + b * EXW),
                                                       *(const float2*)(e + (b + 1) * EXW))
                                           : exp_odd2(*(const float2*)(e + b * EXW), *(const float2*)(e + (b + 1) * EXW));
            float2* gp = (float2*)(G + (c * WH + wr) * WW + wc);
            L[c] = sub2(*gp, up);
            *gp = L[c];
        }
        float2 en;
        if (chroma) {
            en = addl(addl(mul2(L[0], L[0]), mul2(L[1], L[1])), mul2(L[2], L[2]));
        } else {
            const float2 y = luma2(L[0], L[1], L[2]);
            en = mul2(y, y);
        }
        *(float2*)(yb + r * YBW + xq) = en;
    }
}

// ---- phase 7: the binomial window (fuse.rs:168) and the strict-> selection (fuse.rs:429): thread
// (tx, ty) owns the pixel pairs (x0 + 2tx, +1) of rows y0 + 4ty .. +3. It forms the row sums of the
// 4 + 2R energy rows it needs itself (sum_q binw(q) yb[r][x' + q], in order), then the column sums, and
// reads the winning coefficients from L only when a frame wins. R = 0: the node energy itself.
template <int R>
__device__ __forceinline__ void f0_select(const float* __restrict__ yb, const float* __restrict__ G, int k, float (&best)[8],
                                          float (&acc)[8][3], int (&win)[8]) {
    using namespace f0;
    constexpr int NV = 4 + 2 * R;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5, px = 2 * tx;
    float2 v[NV];
#pragma unroll
    for (int t = 0; t < NV; t++) {
        const float* row = yb + (4 * ty + t) * YBW + px;
        if (R == 0) {
            v[t] = *(const float2*)row;
        } else {
            float y[2 + 2 * R];
#pragma unroll
            for (int q = 0; q < 2 + 2 * R; q += 2) {
                const float2 p2 = *(const float2*)(row + q);
                y[q] = p2.x;
                y[q + 1] = p2.y;
            }
            float2 h = mul2(splat(binw<R>(0)), make_float2(y[0], y[1]));
#pragma unroll
            for (int q = 1; q <= 2 * R; q++)
                h = binw_exact<R>(q) ? add2(h, mul2(splat(binw<R>(q)), make_float2(y[q], y[q + 1])))
                                     : addl(h, mul2(splat(binw<R>(q)), make_float2(y[q], y[q + 1])));
            v[t] = h;
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float2 e = v[j];
        if (R > 0) {
            e = mul2(splat(binw<R>(0)), v[j]);
#pragma unroll
            for (int q = 1; q <= 2 * R; q++) e = binw_exact<R>(q) ? add2(e, mul2(splat(binw<R>(q)), v[j + q]))
                                                                : addl(e, mul2(splat(binw<R>(q)), v[j + q]));
        }
        const int wr = 4 * ty + j + 6, wc = px + 6 + (R & 1);
#pragma unroll
        for (int l = 0; l < 2; l++) {
            const float ev = l ? e.y : e.x;
            const int i = 2 * j + l;
            if (ev > best[i]) {
                best[i] = ev;
#pragma unroll
                for (int c = 0; c < 3; c++) acc[i][c] = G[(c * WH + wr) * WW + wc + l];
                win[i] = k;
            }
        }
    }
}

// The bulk copies of frame k's window for tile t (warp 0): one per row, from the 16-byte boundary at
// or before the row's first byte, rounded up to 16 bytes (fold inputs carry 64 bytes of tail
// padding); the row's offset within its slot goes to mis[].
template <int R>
__device__ __forceinline__ void f0_issue(const FoldArgs& a, int t, int k, int nix, unsigned char* raw, int* mis, uint64_t* mbar) {
    using namespace f0;
    const int lane = threadIdx.x & 31;
    const int x0 = (1 + t % nix) * TW0, y0 = (1 + t / nix) * TH0;
    const int gx0 = x0 - 6 - (R & 1), gy0 = y0 - 6;
    const unsigned char* src = (const unsigned char*)a.src_u16;
    size_t from[2] = {0, 0};
    unsigned len[2] = {0, 0}, total = 0;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const int r = lane + 32 * i;
        if (r < WH) {
            const size_t b0 = (((size_t)k * a.H + gy0 + r) * a.W + gx0) * 6;
            from[i] = b0 & ~(size_t)15;
            const int m = (int)(b0 - from[i]);
            len[i] = (unsigned)((m + WW * 6 + 15) & ~15);
            mis[r] = m;
            total += len[i];
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
    if (lane == 0) mbar_expect(mbar, total);
    // the rows' previous contents were read through the generic proxy (ordered by the CTA barrier)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 2; i++)
        if (len[i]) bulk_g2s(raw + (lane + 32 * i) * RAW_ROW, src + from[i], len[i], mbar);
}

#ifndef LSB_F0_SPIN_LIMIT
#define LSB_F0_SPIN_LIMIT (1u << 22)
#endif

// The fused level-0 fold over frames sel_k0 .. sel_k1-1 (their REDUCE, focus slices and selection;
// red_k0 == sel_k0 and red_n == sel_k1 - sel_k0), persistent over the interior tiles. The selection
// resumes from acc / best / winner when sel_k0 > 0. A copy that does not land within the wait limit
// raises LSB_ERR_TIMEOUT in the status word and the CTA returns (after waiting once more, within
// the limit, for its copies in flight).
template <class GS, int R, bool FOCUS, class SS>
__global__ void __launch_bounds__(f0::NT0, 2) fold0_kernel(const FoldArgs a) {
    using namespace f0;
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* mbar = (uint64_t*)(smem + OFF_MBAR);
    int* mis = (int*)(smem + OFF_MIS);
    unsigned char* raw = smem + OFF_RAW;
    float* G = (float*)(smem + OFF_G0);
    float* Ly = (float*)(smem + OFF_LY);
    float* Ls = Ly + LYH * LYW;
    float* yb = (float*)(smem + OFF_YB);
    float* tmp = (float*)(smem + OFF_TMP);
    float* G1s = (float*)(smem + OFF_G1);
    const int W = a.W, H = a.H;
    const Fold0Range rg = fold0_range(W, H, R);
    const int nix = rg.ix1 - 1, ntiles = fold0_count(rg);
    const int k0 = a.sel_k0, k1 = a.sel_k1;
    if ((int)blockIdx.x >= ntiles || k1 <= k0) return;
    if (threadIdx.x == 0) mbar_init(mbar);
    for (int i = threadIdx.x; i < 3 * G1H * (G1W - TMPW); i += NT0)  // G_1 columns past 36: read, never used
        G1s[(i / (G1W - TMPW)) * G1W + TMPW + i % (G1W - TMPW)] = 0.f;
    __syncthreads();
    if (threadIdx.x < 32) f0_issue<R>(a, blockIdx.x, k0, nix, raw, mis, mbar);
    unsigned phase = 0;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const size_t np = (size_t)W * H;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int x0 = (1 + t % nix) * TW0, y0 = (1 + t / nix) * TH0;
        float best[8], acc[8][3];
        int win[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            best[i] = -1.f;  // any energy (>= 0) beats it: the first frame fills the accumulator
            acc[i][0] = acc[i][1] = acc[i][2] = 0.f;
            win[i] = 0;
            if (k0 > 0) {  // resume: the state the frames before left
                const size_t o = (size_t)(y0 + 4 * ty + (i >> 1)) * W + x0 + 2 * tx + (i & 1);
                acc[i][0] = a.acc[o];
                acc[i][1] = a.acc[np + o];
                acc[i][2] = a.acc[2 * np + o];
                best[i] = a.best[o];
                if (a.winner) win[i] = a.winner[o];
            }
        }
        for (int k = k0; k < k1; k++) {
            const bool ok = mbar_wait(mbar, phase & 1, LSB_F0_SPIN_LIMIT);
            phase++;
            if (__syncthreads_or(!ok)) {
                if (threadIdx.x == 0) atomicOr(a.status, LSB_ERR_TIMEOUT);
                mbar_wait(mbar, (phase - 1) & 1, LSB_F0_SPIN_LIMIT);
                return;
            }
            const FrameXform& X = a.xf[k];
            const int gon = X.gain_on;
            const float gain[3] = {X.gain[0], X.gain[1], X.gain[2]};
            const float2 sc = make_float2(X.gscale, X.ginv);
            f0_convert<R, FOCUS>(raw, mis, G, Ly, Ls, gon, gain);
            __syncthreads();
            // the next window: this tile's next frame, or the first frame of this CTA's next tile
            if (threadIdx.x < 32) {
                if (k + 1 < k1) f0_issue<R>(a, t, k + 1, nix, raw, mis, mbar);
                else if (t + (int)gridDim.x < ntiles) f0_issue<R>(a, t + gridDim.x, k0, nix, raw, mis, mbar);
            }
            if (FOCUS) f0_focus<SS>(a, Ly, Ls, k, x0, y0);
            f0_reduce_rows<R>(G, tmp);
            __syncthreads();
            f0_reduce_cols<GS>(a, tmp, G1s, k, x0, y0, sc);
            __syncthreads();
            f0_expand_rows<R>(G1s, tmp);
            __syncthreads();
            f0_laplace<R>(tmp, G, yb, a.use_chroma);
            __syncthreads();
            f0_select<R>(yb, G, k, best, acc, win);
            __syncthreads();  // the next frame's conversion overwrites G and the luma planes
        }
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const size_t o = (size_t)(y0 + 4 * ty + (i >> 1)) * W + x0 + 2 * tx + (i & 1);
            a.acc[o] = acc[i][0];
            a.acc[np + o] = acc[i][1];
            a.acc[2 * np + o] = acc[i][2];
            a.best[o] = best[i];
            if (a.winner) a.winner[o] = (uint16_t)win[i];
        }
    }
}
