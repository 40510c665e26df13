// Frame preparation on the device: what a decoded 16-bit frame goes through
// before it is registered and folded, done on its way into the frame store.
//
// - the dust map (dust.rs:487 DustMap::apply_rgb16): every spot filled by
//   pull-push (dust.rs:591) over a window around it in which every spot's
//   pixels are weighted out, or divided by its measured attenuation (flat);
// - the quarter turns and the draft block mean (lapstack-web decode.rs:68,
//   :92), in one gather;
// - a frame of another size brought to the run's (decode.rs:125, bilinear).
//
// The order and the rounding are the reference's: f32 values u16 / 65535 (a
// division), IEEE products, sums and quotients in the reference's order
// (explicit _rn intrinsics; the build also passes -fmad=false), and
// (clamp(v, 0, 1) * 65535 + 0.5) truncated on the way back; the turn and the
// block mean are integer work. The result is bit-identical to the reference
// order (the oracle's orc_dust.hpp restates it).
//
// Spots are independent: a spot's fill reads its window with every spot's
// pixels weighted out (weight 0: their values never enter the fill), and it
// writes its own mask pixels only. Only spots whose masks overlap depend on
// their order (the later one's value stays; in flat mode the gains compound),
// so the host sorts the spots into layers, each without overlapping masks,
// and the layers run in order. One CTA fills one (spot, channel) pair: its
// window's pull-push pyramid lives in global scratch (L2-resident for the
// usual spot sizes), level by level between block barriers.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "lapstack_b200.h"
#include "lsb_common.cuh"
#include "lsb_prep.h"

namespace lsb {

// pull-push levels of a window (dust.rs:596): halved until 1 x 1, at most 24
constexpr int PP_MAX_LEVELS = 24;
constexpr int PREP_THREADS = 512;

struct DSpot {
    int x, y, w, h;      // the spot's window of the frame (its mask's)
    int x0, y0, ww, wh;  // the fill's window (the spot and as much again around it)
    long long mask_off;  // into masks and gains: w*h
    long long wz_off;    // into wzero: ww*wh, 1 where any spot's mask pixel lies
    long long scr_off;   // into scratch: 3 channel blocks of scr_len floats
    long long scr_len;
};

__host__ __device__ inline int pp_half(int n) { return (n + 1) / 2; }

// the pull-push level dims and the nums/dens offsets of a window; returns the level count
__host__ __device__ inline int pp_levels(int w, int h, int lw[PP_MAX_LEVELS], int lh[PP_MAX_LEVELS], long long off[PP_MAX_LEVELS + 1]) {
    int n = 0;
    lw[0] = w;
    lh[0] = h;
    off[0] = 0;
    for (;;) {
        off[n + 1] = off[n] + (long long)lw[n] * lh[n];
        n++;
        if (!((lw[n - 1] > 1 || lh[n - 1] > 1) && n < PP_MAX_LEVELS)) break;
        lw[n] = pp_half(lw[n - 1]);
        lh[n] = pp_half(lh[n - 1]);
    }
    return n;
}

__device__ __forceinline__ float u16_val(uint16_t u) { return __fdiv_rn((float)u, 65535.f); }
__device__ __forceinline__ uint16_t u16_of_val(float v) {
    const float c = fminf(fmaxf(v, 0.f), 1.f);  // NaN -> 0, as the reference's cast of NaN
    return (uint16_t)fminf(__fadd_rn(__fmul_rn(c, 65535.f), 0.5f), 65535.f);
}

// pyramid.rs:86 REDUCE of a w x h plane into its half, through tmp (h x ow): horizontal taps at even
// columns, a = 0, a += k_t s_t in order; then vertically k0 r0 + k1 r1 + ... left to right
__device__ void pp_reduce(const float* src, int w, int h, float* tmp, float* dst) {
    const float k[5] = {0.0625f, 0.25f, 0.375f, 0.25f, 0.0625f};
    const int ow = pp_half(w), oh = pp_half(h);
    for (int i = threadIdx.x; i < h * ow; i += blockDim.x) {
        const int y = i / ow, x = i - y * ow, c = 2 * x;
        const float* s = src + (size_t)y * w;
        float a = 0.f;
        for (int t = 0; t < 5; t++) a = __fadd_rn(a, __fmul_rn(k[t], s[lsb_reflect(c + t - 2, w)]));
        tmp[i] = a;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < oh * ow; i += blockDim.x) {
        const int y = i / ow, x = i - y * ow, c = 2 * y;
        float a = __fmul_rn(k[0], tmp[(size_t)lsb_reflect(c - 2, h) * ow + x]);
        for (int t = 1; t < 5; t++) a = __fadd_rn(a, __fmul_rn(k[t], tmp[(size_t)lsb_reflect(c + t - 2, h) * ow + x]));
        dst[i] = a;
    }
    __syncthreads();
}

// pyramid.rs:128 expand_row at i of a line of n values `stride` apart
__device__ __forceinline__ float pp_expand_at(const float* c, int n, int i, int stride) {
    const int ci = i >> 1;
    if ((i & 1) == 0)
        return __fadd_rn(__fadd_rn(__fmul_rn(0.125f, c[(size_t)lsb_reflect(ci - 1, n) * stride]), __fmul_rn(0.75f, c[(size_t)lsb_reflect(ci, n) * stride])),
                         __fmul_rn(0.125f, c[(size_t)lsb_reflect(ci + 1, n) * stride]));
    return __fmul_rn(0.5f, __fadd_rn(c[(size_t)lsb_reflect(ci, n) * stride], c[(size_t)lsb_reflect(ci + 1, n) * stride]));
}

// the scratch of one (spot, channel): nums and dens pyramids, the separable passes' tmp, two f planes
__host__ __device__ inline long long pp_scratch_len(int ww, int wh) {
    int lw[PP_MAX_LEVELS], lh[PP_MAX_LEVELS];
    long long off[PP_MAX_LEVELS + 1];
    const int n = pp_levels(ww, wh, lw, lh, off);
    const long long a0 = (long long)ww * wh;
    return 2 * off[n] + (a0 + ww + wh) + 2 * a0;
}

// dust.rs:511-547 DustMode::Fill for the spots list[0 .. gridDim.x) of one layer, channel blockIdx.y:
// the window's values (u16 / 65535) weighted 0 at every spot's mask pixel, pull-push (dust.rs:591),
// and the spot's own mask pixels set from the result.
__global__ void __launch_bounds__(PREP_THREADS) dust_fill_kernel(const DSpot* __restrict__ spots, const int* __restrict__ list,
                                                                const uint8_t* __restrict__ masks, const uint8_t* __restrict__ wzero,
                                                                float* __restrict__ scratch, uint16_t* __restrict__ rgb, int W) {
    const DSpot S = spots[list[blockIdx.x]];
    const int c = blockIdx.y;
    int lw[PP_MAX_LEVELS], lh[PP_MAX_LEVELS];
    long long off[PP_MAX_LEVELS + 1];
    const int L = pp_levels(S.ww, S.wh, lw, lh, off);
    const long long a0 = (long long)S.ww * S.wh;
    float* nums = scratch + S.scr_off + (long long)c * S.scr_len;
    float* dens = nums + off[L];
    float* tmp = dens + off[L];
    float* fa = tmp + a0 + S.ww + S.wh;
    float* fb = fa + a0;
    const uint8_t* wz = wzero + S.wz_off;
    // level 0: nums = v * wt, dens = wt (dust.rs:592-593); a pixel of weight 0 gives 0 whatever its
    // value, so it is not read (another spot of the layer may be writing it)
    for (long long i = threadIdx.x; i < a0; i += blockDim.x) {
        const int y = (int)(i / S.ww), x = (int)(i - (long long)y * S.ww);
        const bool out = wz[i] != 0;
        nums[i] = out ? 0.f : u16_val(rgb[3 * ((size_t)(S.y0 + y) * W + S.x0 + x) + c]);
        dens[i] = out ? 0.f : 1.f;
    }
    __syncthreads();
    for (int l = 0; l + 1 < L; l++) {
        pp_reduce(nums + off[l], lw[l], lh[l], tmp, nums + off[l + 1]);
        pp_reduce(dens + off[l], lw[l], lh[l], tmp, dens + off[l + 1]);
    }
    // the top: n / d where there is weight (dust.rs:605)
    const int top = L - 1;
    float* f = fa;
    for (long long i = threadIdx.x; i < (long long)lw[top] * lh[top]; i += blockDim.x) {
        const float d = dens[off[top] + i];
        f[i] = d > 1e-9f ? __fdiv_rn(nums[off[top] + i], d) : 0.f;
    }
    __syncthreads();
    // down: EXPAND the coarser f (horizontal, then vertical), blended with n / d by wc = clamp(d, 0, 1)
    for (int l = top - 1; l >= 0; l--) {
        const int cw = lw[l + 1], ch = lh[l + 1], ow = lw[l], oh = lh[l];
        for (long long i = threadIdx.x; i < (long long)ch * ow; i += blockDim.x) {
            const int y = (int)(i / ow), x = (int)(i - (long long)y * ow);
            tmp[i] = pp_expand_at(f + (size_t)y * cw, cw, x, 1);
        }
        __syncthreads();
        float* g = (f == fa) ? fb : fa;
        for (long long i = threadIdx.x; i < (long long)oh * ow; i += blockDim.x) {
            const int y = (int)(i / ow), x = (int)(i - (long long)y * ow);
            const float u = pp_expand_at(tmp + x, ch, y, ow);
            const float n = nums[off[l] + i], d = dens[off[l] + i];
            const float wc = fminf(fmaxf(d, 0.f), 1.f);
            g[i] = d > 1e-9f ? __fadd_rn(__fmul_rn(wc, __fdiv_rn(n, d)), __fmul_rn(__fsub_rn(1.f, wc), u)) : u;
        }
        __syncthreads();
        f = g;
    }
    // the spot's own mask pixels take the fill
    const uint8_t* m = masks + S.mask_off;
    for (long long i = threadIdx.x; i < (long long)S.w * S.h; i += blockDim.x) {
        if (!m[i]) continue;
        const int sy = (int)(i / S.w), sx = (int)(i - (long long)sy * S.w);
        const int x = S.x + sx, y = S.y + sy;
        rgb[3 * ((size_t)y * W + x) + c] = u16_of_val(f[(size_t)(y - S.y0) * S.ww + (x - S.x0)]);
    }
}

// dust.rs:503-510 DustMode::Flat: every mask pixel times its attenuation
__global__ void dust_flat_kernel(const DSpot* __restrict__ spots, const int* __restrict__ list, const uint8_t* __restrict__ masks,
                                 const float* __restrict__ gains, uint16_t* __restrict__ rgb, int W) {
    const DSpot S = spots[list[blockIdx.x]];
    const int c = blockIdx.y;
    const uint8_t* m = masks + S.mask_off;
    const float* g = gains + S.mask_off;
    for (long long i = threadIdx.x; i < (long long)S.w * S.h; i += blockDim.x) {
        if (!m[i]) continue;
        const int sy = (int)(i / S.w), sx = (int)(i - (long long)sy * S.w);
        uint16_t& p = rgb[3 * ((size_t)(S.y + sy) * W + S.x + sx) + c];
        p = u16_of_val(__fmul_rn(u16_val(p), g[i]));
    }
}

// decode.rs:68 `rotate` then decode.rs:92 `reduce` in one gather: output pixel (ox, oy) of the turned,
// block-averaged frame sums the turned frame's k x k block (the ragged edge what is there) from the
// source pixels each turned pixel comes from, and rounds (s + n/2) / n
__global__ void turn_draft_kernel(const uint16_t* __restrict__ in, int w, int h, int q, int k, uint16_t* __restrict__ out, int ow, int oh) {
    const int ox = blockIdx.x * blockDim.x + threadIdx.x, oy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ox >= ow || oy >= oh) return;
    const int rw = (q & 1) ? h : w, rh = (q & 1) ? w : h;
    const int X0 = ox * k, X1 = min(X0 + k, rw), Y0 = oy * k, Y1 = min(Y0 + k, rh);
    unsigned long long s0 = 0, s1 = 0, s2 = 0;
    for (int Y = Y0; Y < Y1; Y++)
        for (int X = X0; X < X1; X++) {
            int sx, sy;
            switch (q) {
                case 0: sx = X, sy = Y; break;
                case 1: sx = Y, sy = h - 1 - X; break;
                case 2: sx = w - 1 - X, sy = h - 1 - Y; break;
                default: sx = w - 1 - Y, sy = X; break;
            }
            const uint16_t* p = in + 3 * ((size_t)sy * w + sx);
            s0 += p[0];
            s1 += p[1];
            s2 += p[2];
        }
    const unsigned long long n = (unsigned long long)(Y1 - Y0) * (X1 - X0);
    uint16_t* o = out + 3 * ((size_t)oy * ow + ox);
    o[0] = (uint16_t)((s0 + n / 2) / n);
    o[1] = (uint16_t)((s1 + n / 2) / n);
    o[2] = (uint16_t)((s2 + n / 2) / n);
}

// decode.rs:125 `resize`: bilinear in f64, centres kept, edge-clamped, + 0.5 truncated
__global__ void resize_u16_kernel(const uint16_t* __restrict__ in, int sw, int sh, double kx, double ky, uint16_t* __restrict__ out, int w, int h) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const double fy = fmin(fmax(__dsub_rn(__dmul_rn(__dadd_rn((double)y, 0.5), ky), 0.5), 0.0), (double)(sh - 1));
    const double fx = fmin(fmax(__dsub_rn(__dmul_rn(__dadd_rn((double)x, 0.5), kx), 0.5), 0.0), (double)(sw - 1));
    const int y0 = (int)floor(fy), x0 = (int)floor(fx);
    const double ty = __dsub_rn(fy, floor(fy)), tx = __dsub_rn(fx, floor(fx));
    const int y1 = min(y0 + 1, sh - 1), x1 = min(x0 + 1, sw - 1);
    const uint16_t *a = in + 3 * ((size_t)y0 * sw + x0), *b = in + 3 * ((size_t)y0 * sw + x1);
    const uint16_t *c = in + 3 * ((size_t)y1 * sw + x0), *d = in + 3 * ((size_t)y1 * sw + x1);
    uint16_t* o = out + 3 * ((size_t)y * w + x);
    for (int ch = 0; ch < 3; ch++) {
        const double top = __dadd_rn(__dmul_rn((double)a[ch], __dsub_rn(1.0, tx)), __dmul_rn((double)b[ch], tx));
        const double bot = __dadd_rn(__dmul_rn((double)c[ch], __dsub_rn(1.0, tx)), __dmul_rn((double)d[ch], tx));
        o[ch] = (uint16_t)__dadd_rn(__dadd_rn(__dmul_rn(top, __dsub_rn(1.0, ty)), __dmul_rn(bot, ty)), 0.5);
    }
}

// ------------------------------------------------------------------ host side
DustDev::~DustDev() {
    for (void* p : {(void*)spots, (void*)masks, (void*)wzero, (void*)gains, (void*)scratch, (void*)list})
        if (p) cudaFree(p);
}

// the largest pull-push scratch one map may ask for (every (spot, channel) pair holds its own)
constexpr size_t DUST_SCRATCH_MAX = (size_t)8 << 30;

static bool boxes_meet(const lsb_dust_spot& a, const lsb_dust_spot& b) {
    return a.x < b.x + b.w && b.x < a.x + a.w && a.y < b.y + b.h && b.y < a.y + a.h;
}
static bool masks_meet(const lsb_dust_spot& a, const lsb_dust_spot& b) {
    if (!boxes_meet(a, b)) return false;
    const uint32_t x0 = std::max(a.x, b.x), x1 = std::min(a.x + a.w, b.x + b.w), y0 = std::max(a.y, b.y), y1 = std::min(a.y + a.h, b.y + b.h);
    for (uint32_t y = y0; y < y1; y++)
        for (uint32_t x = x0; x < x1; x++)
            if (a.mask[(size_t)(y - a.y) * a.w + (x - a.x)] && b.mask[(size_t)(y - b.y) * b.w + (x - b.x)]) return true;
    return false;
}

template <class T>
static cudaError_t upload(T** dst, const std::vector<T>& v) {
    cudaError_t e = cudaMalloc(dst, sizeof(T) * std::max<size_t>(v.size(), 1));
    if (e == cudaSuccess && !v.empty()) e = cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
    return e;
}

std::string dust_create(const lsb_dust_map* m, DustDev** out) {
    *out = nullptr;
    if (!m) return "null dust map";
    if (m->w == 0 || m->h == 0 || m->w > 65535 || m->h > 65535) return "dust map: width and height must be 1 to 65535";
    if (m->mode > 1) return "dust map: mode must be 0 (fill) or 1 (flat)";
    if (m->n_spots > (1u << 20)) return "dust map: at most 2^20 spots";
    if (m->n_spots && !m->spots) return "dust map: null spots";
    const int W = (int)m->w, H = (int)m->h, n = (int)m->n_spots;
    for (int k = 0; k < n; k++) {
        const lsb_dust_spot& s = m->spots[k];
        if (s.w == 0 || s.h == 0 || s.x >= m->w || s.y >= m->h || s.w > m->w - s.x || s.h > m->h - s.y)
            return "dust map: spot " + std::to_string(k) + " is not inside the map";
        if (!s.mask) return "dust map: spot " + std::to_string(k) + " has no mask";
        if (m->mode == 1 && !s.gain) return "dust map: spot " + std::to_string(k) + " has no gains (flat mode)";
    }
    std::vector<DSpot> tab(n);
    std::vector<uint8_t> masks, wzero;
    std::vector<float> gains;
    std::vector<int> layer(n, 0);
    long long moff = 0, woff = 0, soff = 0;
    for (int k = 0; k < n; k++) {
        const lsb_dust_spot& s = m->spots[k];
        DSpot& d = tab[k];
        d.x = (int)s.x, d.y = (int)s.y, d.w = (int)s.w, d.h = (int)s.h;
        // dust.rs:514-517 the window: the spot and max(its longer side / 2, 6) around it, cut to the frame
        const int pad = std::max(std::max(d.w, d.h) / 2, 6);
        d.x0 = std::max(d.x - pad, 0);
        d.y0 = std::max(d.y - pad, 0);
        const int x1 = std::min(d.x + d.w + pad, W), y1 = std::min(d.y + d.h + pad, H);
        d.ww = x1 - d.x0;
        d.wh = y1 - d.y0;
        d.mask_off = moff;
        masks.insert(masks.end(), s.mask, s.mask + (size_t)s.w * s.h);
        if (m->mode == 1) gains.insert(gains.end(), s.gain, s.gain + (size_t)s.w * s.h);
        moff += (long long)s.w * s.h;
        if (m->mode == 0) {
            // dust.rs:524-533 every spot's mask pixels in the window weigh 0
            d.wz_off = woff;
            std::vector<uint8_t> wz((size_t)d.ww * d.wh, 0);
            const lsb_dust_spot win{(uint32_t)d.x0, (uint32_t)d.y0, (uint32_t)d.ww, (uint32_t)d.wh, nullptr, nullptr};
            for (int j = 0; j < n; j++) {
                const lsb_dust_spot& o = m->spots[j];
                if (!boxes_meet(o, win)) continue;
                for (uint32_t sy = 0; sy < o.h; sy++)
                    for (uint32_t sx = 0; sx < o.w; sx++) {
                        const int x = (int)(o.x + sx), y = (int)(o.y + sy);
                        if (o.mask[(size_t)sy * o.w + sx] && x >= d.x0 && x < x1 && y >= d.y0 && y < y1)
                            wz[(size_t)(y - d.y0) * d.ww + (x - d.x0)] = 1;
                    }
            }
            wzero.insert(wzero.end(), wz.begin(), wz.end());
            woff += (long long)d.ww * d.wh;
            d.scr_len = pp_scratch_len(d.ww, d.wh);
            d.scr_off = soff;
            soff += 3 * d.scr_len;
        } else {
            d.wz_off = d.scr_off = d.scr_len = 0;
        }
        // spots whose masks overlap keep their order: a later one runs in a later layer
        for (int j = 0; j < k; j++)
            if (masks_meet(m->spots[j], s)) layer[k] = std::max(layer[k], layer[j] + 1);
    }
    if ((size_t)soff * sizeof(float) > DUST_SCRATCH_MAX) return "dust map: the spots' fill windows need more than 8 GiB of scratch";
    const int nl = n ? *std::max_element(layer.begin(), layer.end()) + 1 : 0;
    std::vector<int> list;
    DustDev* d = new DustDev();
    d->W = W, d->H = H, d->mode = (int)m->mode, d->nspots = n;
    d->layer_off.push_back(0);
    for (int l = 0; l < nl; l++) {
        for (int k = 0; k < n; k++)
            if (layer[k] == l) list.push_back(k);
        d->layer_off.push_back((int)list.size());
    }
    d->scratch_bytes = (size_t)soff * sizeof(float);
    cudaError_t e = cudaMalloc(&d->spots, sizeof(DSpot) * std::max(n, 1));
    if (e == cudaSuccess && n) e = cudaMemcpy(d->spots, tab.data(), sizeof(DSpot) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = upload(&d->masks, masks);
    if (e == cudaSuccess) e = upload(&d->wzero, wzero);
    if (e == cudaSuccess) e = upload(&d->gains, gains);
    if (e == cudaSuccess) e = upload(&d->list, list);
    if (e == cudaSuccess) e = cudaMalloc(&d->scratch, std::max<size_t>(d->scratch_bytes, 4));
    if (e != cudaSuccess) {
        delete d;
        return std::string("dust map upload: ") + cudaGetErrorString(e);
    }
    *out = d;
    return std::string();
}

cudaError_t dust_apply_rgb16(const DustDev* d, uint16_t* rgb, cudaStream_t s) {
    for (size_t l = 0; l + 1 < d->layer_off.size(); l++) {
        const int k0 = d->layer_off[l], cnt = d->layer_off[l + 1] - k0;
        if (cnt <= 0) continue;
        const dim3 g(cnt, 3);
        lsb_launched();
        if (d->mode == 0) dust_fill_kernel<<<g, PREP_THREADS, 0, s>>>(d->spots, d->list + k0, d->masks, d->wzero, d->scratch, rgb, d->W);
        else dust_flat_kernel<<<g, 256, 0, s>>>(d->spots, d->list + k0, d->masks, d->gains, rgb, d->W);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void turn_draft_dims(int w, int h, int q, int draft, int* ow, int* oh) {
    const int rw = (q & 1) ? h : w, rh = (q & 1) ? w : h, k = 1 << draft;
    *ow = std::max((rw + k - 1) / k, 1);
    *oh = std::max((rh + k - 1) / k, 1);
}

cudaError_t turn_draft_rgb16(const uint16_t* in, int w, int h, int q, int draft, uint16_t* out, cudaStream_t s) {
    int ow, oh;
    turn_draft_dims(w, h, q & 3, draft, &ow, &oh);
    const dim3 b(32, 8), g((ow + 31) / 32, (oh + 7) / 8);
    lsb_launched();
    turn_draft_kernel<<<g, b, 0, s>>>(in, w, h, q & 3, 1 << draft, out, ow, oh);
    return cudaGetLastError();
}

cudaError_t resize_rgb16(const uint16_t* in, int sw, int sh, uint16_t* out, int w, int h, cudaStream_t s) {
    const dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    lsb_launched();
    resize_u16_kernel<<<g, b, 0, s>>>(in, sw, sh, (double)sw / (double)w, (double)sh / (double)h, out, w, h);
    return cudaGetLastError();
}

}  // namespace lsb
