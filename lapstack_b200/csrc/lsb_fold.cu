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
#include <map>
#include <mutex>
#include <vector>

#include "lsb_common.cuh"
#include "lsb_internal.h"
#include "lsb_interp.cuh"

namespace lsb {

#include "lsb_level.cuh"
#include "lsb_fold0.cuh"

size_t fold_smem_bytes(int, bool) { return (size_t)SEL_FLOATS * sizeof(float); }

// The taps live in constant memory, one copy per device for every engine on it: they are written
// (stream-ordered on s) only when they change, and an engine that finds them already requested
// makes its stream wait for that write. Engines that run at the same time must ask for the same taps.
static std::mutex g_taps_mu;
static std::map<int, std::pair<std::vector<float>, cudaEvent_t>> g_taps;
cudaError_t set_focus_taps(const float* taps3, int ntaps, cudaStream_t s) {
    if (ntaps > 64) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t de = cudaGetDevice(&dev);
    if (de != cudaSuccess) return de;
    std::lock_guard<std::mutex> lk(g_taps_mu);
    auto& cur = g_taps[dev];
    const std::vector<float> want(taps3, taps3 + 3 * ntaps);
    if (cur.second && cur.first == want) return cudaStreamWaitEvent(s, cur.second, 0);
    if (!cur.second) {
        de = cudaEventCreateWithFlags(&cur.second, cudaEventDisableTiming);
        if (de != cudaSuccess) {
            cur.second = nullptr;
            return de;
        }
    }
    int off[64];
    float wgt[64];
    for (int q = 0; q < ntaps; q++) {
        off[q] = (int)taps3[3 * q] * RGW + (int)taps3[3 * q + 1];
        wgt[q] = taps3[3 * q + 2];
    }
    cudaError_t e = cudaMemcpyToSymbolAsync(c_taps, taps3, sizeof(float) * 3 * ntaps, 0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyToSymbolAsync(c_tapo, off, sizeof(int) * ntaps, 0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyToSymbolAsync(c_tapw, wgt, sizeof(float) * ntaps, 0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(cur.second, s);
    cur.first = e == cudaSuccess ? want : std::vector<float>();
    return e;
}

template <class K>
static cudaError_t with_smem(K k, size_t smem) {
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// fuse.rs:429 strict `>` across frame groups: the groups' selection states merged in group order: the first group
// holding the largest energy wins, and within it its first frame did.
__global__ void select_merge_kernel(const FoldArgs a, int G) {
    const size_t np = (size_t)a.W * a.H;
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < np; o += (size_t)gridDim.x * blockDim.x) {
        int bg = 0;
        float best = a.gbest[o];
        for (int g = 1; g < G; g++) {
            const float b = a.gbest[(size_t)g * np + o];
            if (b > best) {
                best = b;
                bg = g;
            }
        }
        const float* ga = a.gacc + (size_t)bg * 3 * np;
        a.acc[o] = ga[o];
        a.acc[np + o] = ga[np + o];
        a.acc[2 * np + o] = ga[2 * np + o];
        a.best[o] = best;
        if (a.winner) a.winner[o] = (uint16_t)a.gwin[(size_t)bg * np + o];
    }
}

// The fused level-0 kernel applies: 16-bit frames, one call doing the REDUCE and the selection of the
// same frames, no halo control, no focus slice or the default one (ring difference filter r 1..3 on
// 2x2 blocks), and a frame with interior tiles. It walks all the frames per tile, so the level is then
// selected without frame groups.
static bool fold0_applies(const FoldArgs& a, int src, bool focus, int R) {
    if (src != SRC_U16 || a.level != 0 || a.halo_mode != 0 || !a.select || a.red_n <= 0) return false;
    if (a.red_k0 != a.sel_k0 || a.red_n != a.sel_k1 - a.sel_k0) return false;
    if (focus && !(a.rdf13 && a.bk == 2 && a.focus_kind == 0)) return false;
    return fold0_count(fold0_range(a.W, a.H, R)) > 0;
}

// One level: REDUCE the frames asked for (and take their focus slices at level 0), then select.
// Level 0 of 16-bit frames: the fused kernel on the interior tiles, the two kernels on the others.
template <int SRC, class GS, int R, bool FOCUS, class SS>
static cudaError_t launch_level(const FoldArgs& a0, cudaStream_t s, int grid_limit) {
    const size_t rsm = (size_t)RED_FLOATS * sizeof(float), ssm = Staging<SRC, GS, R>::SMEM;
    auto kr = reduce_level_kernel<SRC, GS, FOCUS, SS>;
    auto ks = select_level_kernel<SRC, GS, R>;
    cudaError_t e = with_smem(kr, rsm);
    if (e == cudaSuccess) e = with_smem(ks, ssm);
    if (e != cudaSuccess) return e;
    FoldArgs a = a0;
    int rtiles = ((a.W1 + RW - 1) / RW) * ((a.H1 + RH - 1) / RH);
    // beside the registration chain: one persistent CTA per SM at most
    const size_t ssm_run = a.beside ? std::max(ssm, BESIDE_SMEM) : ssm;
    if (a.beside && (e = with_smem(ks, ssm_run)) != cudaSuccess) return e;
    if (SRC == SRC_U16 && !a0.no_fused && fold0_applies(a0, SRC, FOCUS, R)) {
        auto kf = fold0_kernel<GS, R, FOCUS, SS>;
        const size_t fsm = a.beside ? std::max((size_t)f0::SMEM, BESIDE_SMEM) : (size_t)f0::SMEM;
        e = with_smem(kf, fsm);
        if (e != cudaSuccess) return e;
        const Fold0Range rg = fold0_range(a.W, a.H, R);
        const int nf = fold0_count(rg);
        lsb_launched(), kf<<<std::min(nf, std::max(grid_limit, 1)), f0::NT0, fsm, s>>>(a);
        if (a.after_fused) cudaEventRecord(a.after_fused, s);
        if (a.between) cudaEventRecord(a.between, s);
        a.between = nullptr;
        a.sel_groups = 1;  // the border tiles too: a group merge would run over the whole level
        a.fused0 = 1;
        a.f0r = R;
        a.ntiles = fold0_border_count(a.tiles_x, a.tiles_y, rg);
        rtiles = a.ntiles;  // the REDUCE's tiles are the level-0 tiles' G_1 blocks
        if (a.ntiles <= 0) return cudaGetLastError();
    }
    if (a.red_n > 0) lsb_launched(), kr<<<dim3(rtiles, a.red_n), NT, rsm, s>>>(a);
    if (a.between) cudaEventRecord(a.between, s);
    const int groups = std::max(a.sel_groups, 1);
    if (a.select) lsb_launched(), ks<<<std::min(a.ntiles * groups, std::max(grid_limit, 1)), NT, ssm_run, s>>>(a);
    if (a.select && groups > 1) {
        const size_t np = (size_t)a.W * a.H;
        lsb_launched(), select_merge_kernel<<<(unsigned)std::min<size_t>((np + 255) / 256, 148 * 8), 256, 0, s>>>(a, groups);
    }
    return cudaGetLastError();
}

template <int SRC, class GS, int R>
static cudaError_t pick_focus(const FoldArgs& a, bool focus, cudaStream_t s, int gl) {
    if (!focus) return launch_level<SRC, GS, R, false, float>(a, s, gl);
    // 16-bit storage keeps the focus slices in FP16 (relative precision is what the peak search needs)
    if (sizeof(GS) == 2) return launch_level<SRC, GS, R, true, __half>(a, s, gl);
    return launch_level<SRC, GS, R, true, float>(a, s, gl);
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

// wav.rs:146-161 the weighted average's accumulation over the frames as folded (level 0's source and
// gains): per pixel, frame by frame in order, w = the frame's weight plane taken bilinearly to the pixel
// (depth.rs:201 upsample_bilinear), acc += w * v per channel, wsum += w; then acc / wsum clamped to [0, 1].
template <int SRC>
__global__ void wav_accumulate_kernel(const FoldArgs a, const float* __restrict__ wts, int n, int dw, int dh, int k,
                                      float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.W || y >= a.H) return;
    const float inv = __fdiv_rn(1.f, (float)k);
    int x0, x1, y0, y1;
    float tx, ty;
    bil_axis(x, inv, dw, x0, x1, tx);
    bil_axis(y, inv, dh, y0, y1, ty);
    const size_t m = (size_t)dw * dh, np = (size_t)a.W * a.H, o = (size_t)y * a.W + x;
    float acc[3] = {0.f, 0.f, 0.f}, ws = 0.f;
    for (int f = 0; f < n; f++) {
        const float wv = bil(wts + (size_t)f * m, dw, x0, x1, y0, y1, tx, ty);
        float v[3];
        level_px<SRC, float>(a, f, x, y, v);
#pragma unroll
        for (int c = 0; c < 3; c++) acc[c] = __fadd_rn(acc[c], __fmul_rn(wv, v[c]));
        ws = __fadd_rn(ws, wv);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) out[c * np + o] = fminf(fmaxf(__fdiv_rn(acc[c], ws), 0.f), 1.f);
}

cudaError_t wav_accumulate(const FoldArgs& a, int src_kind, const float* wts, int n, int dw, int dh, int k, float* out, cudaStream_t s) {
    dim3 b(32, 8), g((a.W + 31) / 32, (a.H + 7) / 8);
    if (src_kind == SRC_F32) lsb_launched(), wav_accumulate_kernel<SRC_F32><<<g, b, 0, s>>>(a, wts, n, dw, dh, k, out);
    else if (src_kind == SRC_U16) lsb_launched(), wav_accumulate_kernel<SRC_U16><<<g, b, 0, s>>>(a, wts, n, dw, dh, k, out);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t fold_level(const FoldArgs& a0, int src_kind, int storage, int radius, bool focus, cudaStream_t s, int grid_limit) {
    FoldArgs a = a0;  // the select kernel's tiling
    a.tiles_x = (a.W + TW - 1) / TW;
    a.tiles_y = (a.H + TH - 1) / TH;
    a.ntiles = a.tiles_x * a.tiles_y;
    if (a.ntiles <= 0) return cudaSuccess;
    switch (storage) {
        case STORE_UNORM16: return pick_src<unorm16>(a, src_kind, radius, focus, s, grid_limit);
        case STORE_F16: return pick_src<__half>(a, src_kind, radius, focus, s, grid_limit);
        default: return pick_src<float>(a, src_kind, radius, focus, s, grid_limit);
    }
}

cudaError_t warp_frames(const uint16_t* frames, const FrameXform* xf, int interp, int w, int h, int n, bool u16_out, void* out,
                        cudaStream_t s) {
    if (interp == 3) {  // Spline4x4: the tiled form
        dim3 g((w + WT_W - 1) / WT_W, (h + WT_H - 1) / WT_H, n);
        if (u16_out) lsb_launched(), warp_tile_kernel<true><<<g, NT, 0, s>>>(frames, xf, w, h, out);
        else lsb_launched(), warp_tile_kernel<false><<<g, NT, 0, s>>>(frames, xf, w, h, out);
        return cudaGetLastError();
    }
    dim3 g((w + 31) / 32, (h + 7) / 8, n);
    if (u16_out) lsb_launched(), warp_frames_kernel<true><<<g, NT, 0, s>>>(frames, xf, interp, w, h, out);
    else lsb_launched(), warp_frames_kernel<false><<<g, NT, 0, s>>>(frames, xf, interp, w, h, out);
    return cudaGetLastError();
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
            const float2 sc = make_float2(0.f, a.xf[k].ginv);
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
    if (a.n == 1 || a.top_rule == 2) {
        const float inv = __fdiv_rn(1.f, (float)a.n);
        for (int k = 0; k < a.n; k++) {
            const float2 sc = make_float2(0.f, a.xf[k].ginv);
            for (int c = 0; c < 3; c++) o[c] = __fadd_rn(o[c], __fmul_rn(Store<GS>::ld(t + ((size_t)k * 3 + c) * n2 + pix, sc), inv));
        }
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
            if (!dominated(x)) {
                const float2 sc = make_float2(0.f, a.xf[x].ginv);
                for (int c = 0; c < 3; c++) o[c] = __fadd_rn(o[c], __fmul_rn(Store<GS>::ld(t + ((size_t)x * 3 + c) * n2 + pix, sc), inv));
            }
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

// ------------------------------------------------------------- halo control
// pyramid.rs:86 REDUCE of one f32 plane per frame: the 5 reflected rows each
// reduced along x (the row pass), then those 5 values along y (the column
// pass) -- the same operations, in the same order, as the two passes.
__global__ void reduce_weights_kernel(const float* __restrict__ src, int w, int h, float* __restrict__ dst, int w1, int h1) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (j >= w1 || i >= h1) return;
    const float* p = src + (size_t)k * w * h;
    float r[5];
    for (int t = 0; t < 5; t++) {
        const float* row = p + (size_t)lsb_reflect(2 * i + t - 2, h) * w;
        r[t] = lsb_tap5(row[lsb_reflect(2 * j - 2, w)], row[lsb_reflect(2 * j - 1, w)], row[lsb_reflect(2 * j, w)],
                        row[lsb_reflect(2 * j + 1, w)], row[lsb_reflect(2 * j + 2, w)]);
    }
    dst[(size_t)k * w1 * h1 + (size_t)i * w1 + j] = lsb_tap5(r[0], r[1], r[2], r[3], r[4]);
}
cudaError_t reduce_weights(const float* src, int w, int h, int n, float* dst, int w1, int h1, cudaStream_t s) {
    dim3 b(32, 8), g((w1 + 31) / 32, (h1 + 7) / 8, n);
    lsb_launched(), reduce_weights_kernel<<<g, b, 0, s>>>(src, w, h, dst, w1, h1);
    return cudaGetLastError();
}
// fuse.rs:466-470 at the top level: acc = G * w for frame 0, then acc += w * G; best = sum w
template <class GS>
__global__ void halo_top_kernel(const GS* __restrict__ tops, const FrameXform* __restrict__ xf, const float* __restrict__ wts, int n, int w,
                                int h, float* __restrict__ acc, float* __restrict__ best) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t n2 = (size_t)w * h, o = (size_t)y * w + x;
    float a[3] = {0.f, 0.f, 0.f}, b = 0.f;
    for (int k = 0; k < n; k++) {
        const float2 sc = make_float2(xf[k].gscale, xf[k].ginv);
        const float wv = wts[(size_t)k * n2 + o];
        for (int c = 0; c < 3; c++) {
            const float g = Store<GS>::ld(tops + ((size_t)k * 3 + c) * n2 + o, sc);
            a[c] = k == 0 ? __fmul_rn(g, wv) : __fadd_rn(a[c], __fmul_rn(wv, g));
        }
        b = k == 0 ? wv : __fadd_rn(b, wv);
    }
    for (int c = 0; c < 3; c++) acc[c * n2 + o] = a[c];
    best[o] = b;
}
cudaError_t halo_top(const void* tops, int storage, const FrameXform* xf, const float* wts, int n, int w, int h, float* acc, float* best,
                     cudaStream_t s) {
    dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    if (storage == STORE_UNORM16) lsb_launched(), halo_top_kernel<unorm16><<<g, b, 0, s>>>((const unorm16*)tops, xf, wts, n, w, h, acc, best);
    else if (storage == STORE_F16) lsb_launched(), halo_top_kernel<__half><<<g, b, 0, s>>>((const __half*)tops, xf, wts, n, w, h, acc, best);
    else lsb_launched(), halo_top_kernel<float><<<g, b, 0, s>>>((const float*)tops, xf, wts, n, w, h, acc, best);
    return cudaGetLastError();
}
// fuse.rs:508: the weighted means
__global__ void halo_divide_kernel(float* __restrict__ acc, const float* __restrict__ best, size_t n2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n2; i += (size_t)gridDim.x * blockDim.x)
        for (int c = 0; c < 3; c++) acc[c * n2 + i] = __fdiv_rn(acc[c * n2 + i], best[i]);
}
cudaError_t halo_divide(float* acc, const float* best, int w, int h, cudaStream_t s) {
    const size_t n2 = (size_t)w * h;
    lsb_launched(), halo_divide_kernel<<<(int)std::min<size_t>((n2 + 255) / 256, 148 * 8), 256, 0, s>>>(acc, best, n2);
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
            if (rgb) rgb[((size_t)y * w + x) * 3 + c] = (uint16_t)__fadd_rn(__fmul_rn(v, 65535.f), 0.5f);
        }
        out[o] = v;
    }
}

// fuse.rs:336 `upsample_index`: the depth level's winner map, nearest, to full size (clamped at the edge)
__global__ void upsample_index_kernel(const uint16_t* __restrict__ win, int dwl, int dhl, int scale, int w, int h, float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    out[(size_t)y * w + x] = (float)win[(size_t)min(y / scale, dhl - 1) * dwl + min(x / scale, dwl - 1)];
}
cudaError_t upsample_index(const uint16_t* win, int dwl, int dhl, int scale, int w, int h, float* out, cudaStream_t s) {
    dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    lsb_launched(), upsample_index_kernel<<<g, b, 0, s>>>(win, dwl, dhl, scale, w, h, out);
    return cudaGetLastError();
}

cudaError_t collapse_level(const float* acc, const float* coarse, float* out, int w, int h, int cw, int ch, bool last,
                           uint16_t* rgb_out, cudaStream_t s) {
    dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    lsb_launched(), collapse_kernel<<<g, b, 0, s>>>(acc, coarse, out, w, h, cw, ch, last ? 1 : 0, rgb_out);
    return cudaGetLastError();
}

// ------------------------------------------------------------ winner shares
// fuse.rs:315 `winner_shares`: the plane's largest winning energy, then per frame the cells it
// wins above 1% of that.
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
// brightness.rs:67: each frame's partials summed in part order.
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
