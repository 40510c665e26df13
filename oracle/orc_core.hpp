// Oracle: a CPU restatement of lapstack-core's stacking-engine hot path.
//
// TEST INFRASTRUCTURE ONLY. This code is the checker the CUDA engine is
// compared against; it is never linked into or called by the engine. Only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm
// load it.
//
// Every function follows the reference's Rust CPU path operation for
// operation (same association order, no FMA contraction: build with
// -ffp-contract=off), templated on the scalar type: `float` is the
// reference FP32 path, `double` the FP64 oracle. Citations are
// crates/lapstack-core/src/<file>:<line> of ragtux/LAPSTACK.
//
// This file: shared helpers, pyramid.rs, fuse.rs.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <type_traits>
#include <vector>

namespace orc {

// A literal of the scalar type: the f32 literal for float (as Rust parses
// `0.299` into an f32), the f64 literal for double.
#define LIT(x) (std::is_same<T, float>::value ? (T)(x##f) : (T)(x))

// pyramid.rs:81 `half`
inline size_t half(size_t n) { return (n + 1) / 2; }

// pyramid.rs:51 `reflect`: reflect-101 (period 2(n-1)), looping for tiny n.
inline size_t reflect(long i, size_t n) {
    if (n == 1) return 0;
    long nn = (long)n;
    for (;;) {
        if (i < 0) i = -i;
        else if (i >= nn) i = 2 * (nn - 1) - i;
        else return (size_t)i;
    }
}

// pyramid.rs:20 `Img3`: three row-major planes.
template <class T>
struct Img3 {
    size_t w = 0, h = 0;
    std::vector<T> p[3];
    Img3() {}
    Img3(size_t w_, size_t h_) : w(w_), h(h_) {
        for (int c = 0; c < 3; c++) p[c].assign(w * h, T(0));
    }
};

// ----------------------------------------------------------------- pyramid.rs

// pyramid.rs:46 KERNEL = [1 4 6 4 1]/16
template <class T>
inline T kern(int t) {
    static const T k[5] = {T(1) / T(16), T(4) / T(16), T(6) / T(16), T(4) / T(16), T(1) / T(16)};
    return k[t];
}

// pyramid.rs:86 `reduce`: horizontal 5-tap at even columns, then vertical.
template <class T>
void reduce(const T* src, size_t w, size_t h, std::vector<T>& out, size_t& ow, size_t& oh) {
    ow = half(w);
    oh = half(h);
    std::vector<T> tmp(h * ow);
#pragma omp parallel for schedule(static) if (h * ow >= (1u << 15))
    for (long y = 0; y < (long)h; y++) {
        const T* s = src + (size_t)y * w;
        for (size_t i = 0; i < ow; i++) {
            long c = 2 * (long)i;
            T a = T(0);
            for (int t = 0; t < 5; t++) a += kern<T>(t) * s[reflect(c + t - 2, w)];
            tmp[(size_t)y * ow + i] = a;
        }
    }
    out.assign(oh * ow, T(0));
#pragma omp parallel for schedule(static) if (oh * ow >= (1u << 15))
    for (long y = 0; y < (long)oh; y++) {
        long c = 2 * y;
        const T* r[5];
        for (int t = 0; t < 5; t++) r[t] = &tmp[reflect(c + t - 2, h) * ow];
        for (size_t j = 0; j < ow; j++)
            out[(size_t)y * ow + j] = kern<T>(0) * r[0][j] + kern<T>(1) * r[1][j] + kern<T>(2) * r[2][j] +
                                      kern<T>(3) * r[3][j] + kern<T>(4) * r[4][j];
    }
}

// pyramid.rs:124-125 EVEN = 2*[K0 K2 K4], ODD = 2*K1
template <class T> inline T even_w(int t) { return t == 1 ? T(2) * kern<T>(2) : T(2) * kern<T>(0); }
template <class T> inline T odd_w() { return T(2) * kern<T>(1); }

// pyramid.rs:128 `expand_row`
template <class T>
inline T expand_at(const T* c, size_t cw, size_t i, size_t stride) {
    long ci = (long)(i / 2);
    if (i % 2 == 0)
        return even_w<T>(0) * c[reflect(ci - 1, cw) * stride] + even_w<T>(1) * c[reflect(ci, cw) * stride] +
               even_w<T>(2) * c[reflect(ci + 1, cw) * stride];
    return odd_w<T>() * (c[reflect(ci, cw) * stride] + c[reflect(ci + 1, cw) * stride]);
}

// pyramid.rs:143 `expand`: horizontal then vertical.
template <class T>
std::vector<T> expand(const T* coarse, size_t cw, size_t ch, size_t ow, size_t oh) {
    std::vector<T> tmp(ch * ow);
#pragma omp parallel for schedule(static) if (ch * ow >= (1u << 15))
    for (long y = 0; y < (long)ch; y++)
        for (size_t i = 0; i < ow; i++) tmp[(size_t)y * ow + i] = expand_at<T>(coarse + (size_t)y * cw, cw, i, 1);
    std::vector<T> out(oh * ow);
#pragma omp parallel for schedule(static) if (oh * ow >= (1u << 15))
    for (long i = 0; i < (long)oh; i++)
        for (size_t j = 0; j < ow; j++) out[(size_t)i * ow + j] = expand_at<T>(&tmp[j], ch, (size_t)i, ow);
    return out;
}

// pyramid.rs:170 `reduce3`
template <class T>
Img3<T> reduce3(const Img3<T>& im) {
    Img3<T> o;
    for (int c = 0; c < 3; c++) reduce<T>(im.p[c].data(), im.w, im.h, o.p[c], o.w, o.h);
    return o;
}

// pyramid.rs:177 `expand3`
template <class T>
Img3<T> expand3(const Img3<T>& im, size_t ow, size_t oh) {
    Img3<T> o;
    o.w = ow;
    o.h = oh;
    for (int c = 0; c < 3; c++) o.p[c] = expand<T>(im.p[c].data(), im.w, im.h, ow, oh);
    return o;
}

// pyramid.rs:191 `auto_levels`
inline size_t auto_levels(size_t w, size_t h, size_t min_top) {
    size_t n = 0, cw = w, ch = h;
    while ((cw > 1 || ch > 1) && std::min(half(cw), half(ch)) >= std::max<size_t>(min_top, 1)) {
        cw = half(cw);
        ch = half(ch);
        n++;
    }
    return std::max<size_t>(n, 1);
}

template <class T>
inline T stored(T v, int storage, const float scale[2]);

// pyramid.rs:203 `build`: [L_0 .. L_{N-1}, G_N]. With a 16-bit storage (the engine's, see `stored`)
// every level >= 1 is rounded as stored before anything reads it.
template <class T>
std::vector<Img3<T>> build(const Img3<T>& img, size_t levels, int storage = 0, const float* scale = nullptr) {
    std::vector<Img3<T>> out;
    Img3<T> g = img;
    for (size_t l = 0; l < levels; l++) {
        Img3<T> next = reduce3(g);
        if (storage != 0)
            for (int c = 0; c < 3; c++)
                for (auto& v : next.p[c]) v = stored(v, storage, scale);
        Img3<T> up = expand3(next, g.w, g.h);
        for (int c = 0; c < 3; c++)
            for (size_t i = 0; i < g.w * g.h; i++) g.p[c][i] -= up.p[c][i];
        out.push_back(std::move(g));
        g = std::move(next);
    }
    out.push_back(std::move(g));
    return out;
}

// pyramid.rs:219 `collapse`
template <class T>
Img3<T> collapse(std::vector<Img3<T>> pyr) {
    Img3<T> g = std::move(pyr.back());
    pyr.pop_back();
    while (!pyr.empty()) {
        Img3<T> l = std::move(pyr.back());
        pyr.pop_back();
        Img3<T> up = expand3(g, l.w, l.h);
        for (int c = 0; c < 3; c++)
            for (size_t i = 0; i < l.w * l.h; i++) l.p[c][i] += up.p[c][i];
        g = std::move(l);
    }
    return g;
}

// ------------------------------------------- the engine's 16-bit level storage
// Not the reference's: the rounding the CUDA engine applies when it stores Gaussian levels >= 1 in 16
// bits, so that its 16-bit path can be checked against the reference algorithm run with the same
// storage. STORE_UNORM16: a level of a frame whose largest gain is g (at least 1) is kept as
// u = (u16) clamp(v * (65535 / g) + 0.5, 0, 65535) and read back as u * (g / 65535), both factors
// rounded to f32 once; STORE_F16: IEEE half, round to nearest even.
enum Storage { STORE_F32 = 0, STORE_UNORM16 = 1, STORE_F16 = 2 };

// f32 -> f16 bits, round to nearest even (overflow to infinity, subnormal halves kept)
inline uint16_t f16_bits(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u, ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) return (uint16_t)(sign | 0x7c00u | (ax > 0x7f800000u ? 0x200u : 0u));  // inf, nan
    if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);  // rounds past the largest half
    if (ax >= 0x38800000u) {  // a normal half: drop 13 mantissa bits, nearest even
        uint32_t m = ax - 0x38000000u;  // rebias the exponent (127 -> 15) in place
        const uint32_t rest = m & 0x1fffu;
        m >>= 13;
        if (rest > 0x1000u || (rest == 0x1000u && (m & 1u))) m++;
        return (uint16_t)(sign | m);
    }
    // a subnormal half (or zero): the value in units of 2^-24, nearest even
    const int e = (int)(ax >> 23) - 127;  // the f32's exponent
    if (e < -25) return (uint16_t)sign;
    const uint32_t mant = (ax & 0x7fffffu) | 0x800000u;  // 24 significant bits, value = mant * 2^(e - 23)
    const int shift = -e - 1;  // units of 2^-24: mant * 2^(e + 1) = mant >> (-(e + 1))
    const uint32_t q = mant >> shift, rem = mant & ((1u << shift) - 1u), half = 1u << (shift - 1);
    return (uint16_t)(sign | (q + ((rem > half || (rem == half && (q & 1u))) ? 1u : 0u)));
}
inline float f16_value(uint16_t h) {
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    float v;
    if (e == 0) v = std::ldexp((float)m, -24);
    else if (e == 31) v = m ? std::numeric_limits<float>::quiet_NaN() : std::numeric_limits<float>::infinity();
    else v = std::ldexp((float)(m | 0x400u), (int)e - 25);
    return sign ? -v : v;
}
// a level value as the storage gives it back; scale = (65535 / g, g / 65535) of the frame
template <class T>
inline T stored(T v, int storage, const float scale[2]) {
    if (storage == STORE_UNORM16) {
        const float u = std::min(std::max((float)v * scale[0] + 0.5f, 0.f), 65535.f);
        return (T)((float)(uint16_t)u * scale[1]);
    }
    if (storage == STORE_F16) return (T)f16_value(f16_bits((float)v));
    return v;
}

// -------------------------------------------------------------------- fuse.rs

enum TopRule { TOP_DEV_ENTROPY = 0, TOP_DEVIATION = 1, TOP_AVERAGE = 2 };

// fuse.rs:70-107 `FuseParams` (levels 0 = auto)
struct FuseParams {
    size_t levels = 0;
    size_t energy_radius = 1;
    int top_rule = TOP_DEV_ENTROPY;
    size_t top_radius = 2;
    size_t entropy_bins = 256;
    bool use_chroma = false;
    size_t depth_level = 2;
    float halo = 0.0f;
};

// fuse.rs:112-117
constexpr float HALO_REF = 1e-4f;
constexpr float HALO_FLOOR = 1e-8f;
constexpr float HALO_MAX = 8.0f;
// fuse.rs:333
constexpr float DETAIL_FLOOR = 0.01f;

// fuse.rs:127 `halo_weight`
template <class T>
inline T halo_weight(T re, T p) {
    T v = p * std::log((re + (T)HALO_FLOOR) / (T)HALO_REF);
    v = std::min(std::max(v, T(-60)), T(60));
    return std::exp(v);
}

// fuse.rs:139 `binomial`
template <class T>
std::vector<T> binomial(size_t r) {
    size_t n = 2 * r + 1;
    std::vector<uint64_t> row(n, 1);
    for (size_t i = 1; i < n; i++)
        for (size_t j = i - 1; j >= 1; j--) row[j] += row[j - 1];
    uint64_t s = 0;
    for (auto v : row) s += v;
    std::vector<T> o(n);
    for (size_t i = 0; i < n; i++) o[i] = (T)row[i] / (T)s;
    return o;
}

// fuse.rs:160 (and depth.rs:163, align.rs:567): BT.601 luma, f32 literals
template <class T>
inline T luma_of(T r, T g, T b) {
    return LIT(0.299) * r + LIT(0.587) * g + LIT(0.114) * b;
}

// fuse.rs:152 `node_energy`
template <class T>
std::vector<T> node_energy(const Img3<T>& l, bool use_chroma) {
    size_t n = l.w * l.h;
    std::vector<T> e(n);
#pragma omp parallel for schedule(static) if (n >= (1u << 15))
    for (long i = 0; i < (long)n; i++) {
        T r = l.p[0][i], g = l.p[1][i], b = l.p[2][i];
        if (use_chroma) e[i] = r * r + g * g + b * b;
        else {
            T y = luma_of<T>(r, g, b);
            e[i] = y * y;
        }
    }
    return e;
}

// fuse.rs:168 `window_sum`: separable weights, reflect-101, horizontal first.
template <class T>
std::vector<T> window_sum(const T* src, size_t w, size_t h, const std::vector<T>& wt) {
    long r = (long)(wt.size() / 2);
    if (r == 0) return std::vector<T>(src, src + w * h);
    std::vector<T> tmp(w * h), out(w * h);
#pragma omp parallel for schedule(static) if (w * h >= (1u << 15))
    for (long y = 0; y < (long)h; y++) {
        const T* s = src + (size_t)y * w;
        for (size_t j = 0; j < w; j++) {
            T a = T(0);
            for (size_t t = 0; t < wt.size(); t++) a += wt[t] * s[reflect((long)j + (long)t - r, w)];
            tmp[(size_t)y * w + j] = a;
        }
    }
#pragma omp parallel for schedule(static) if (w * h >= (1u << 15))
    for (long y = 0; y < (long)h; y++) {
        T* row = &out[(size_t)y * w];
        for (size_t j = 0; j < w; j++) row[j] = T(0);
        for (size_t t = 0; t < wt.size(); t++) {
            const T* s = &tmp[reflect(y + (long)t - r, h) * w];
            for (size_t j = 0; j < w; j++) row[j] += wt[t] * s[j];
        }
    }
    return out;
}

// fuse.rs:200 `region_energy`
template <class T>
std::vector<T> region_energy(const Img3<T>& l, size_t radius, bool use_chroma) {
    std::vector<T> e = node_energy(l, use_chroma);
    return window_sum<T>(e.data(), l.w, l.h, binomial<T>(radius));
}

// The f32 natural log of the probabilities k/n an entropy window can hold:
// p.ln() with p = k as f32 * (1/n). glibc's logf is the platform libm the
// reference's f32::ln resolves to on Linux.
template <class T>
inline T ln_of(T p) {
    return std::log(p);
}

// fuse.rs:207 `deviation_entropy`
template <class T>
void deviation_entropy(const T* y, size_t w, size_t h, size_t radius, size_t bins_in, std::vector<T>& dev,
                       std::vector<T>& ent) {
    size_t n = (2 * radius + 1) * (2 * radius + 1);
    T inv_n = T(1) / (T)n;
    size_t bins = std::min<size_t>(std::max<size_t>(bins_in, 2), 65536);
    T qscale = (T)(bins - 1);
    dev.assign(w * h, T(0));
    ent.assign(w * h, T(0));
    long r = (long)radius;
#pragma omp parallel for schedule(static) if (w * h >= (1u << 12))
    for (long i = 0; i < (long)h; i++) {
        std::vector<uint32_t> hist(bins, 0);
        std::vector<size_t> touched;
        touched.reserve(n);
        for (size_t j = 0; j < w; j++) {
            T s = T(0), s2 = T(0);
            touched.clear();
            for (long dy = -r; dy <= r; dy++) {
                size_t yy = reflect(i + dy, h);
                for (long dx = -r; dx <= r; dx++) {
                    T v = y[yy * w + reflect((long)j + dx, w)];
                    s += v;
                    s2 += v * v;
                    T vc = std::min(std::max(v, T(0)), T(1));
                    size_t q = (size_t)(vc * qscale + LIT(0.5));
                    if (hist[q] == 0) touched.push_back(q);
                    hist[q] += 1;
                }
            }
            T mean = s * inv_n;
            dev[(size_t)i * w + j] = std::max(s2 * inv_n - mean * mean, T(0));
            T e = T(0);
            for (size_t q : touched) {
                T p = (T)hist[q] * inv_n;
                e -= p * ln_of<T>(p);
                hist[q] = 0;
            }
            ent[(size_t)i * w + j] = e;
        }
    }
}

// fuse.rs:248 `fuse_residuals`
template <class T>
Img3<T> fuse_residuals(const std::vector<Img3<T>>& tops, const FuseParams& params) {
    const Img3<T>& t0 = tops[0];
    size_t w = t0.w, h = t0.h, n = tops.size(), sz = w * h;
    Img3<T> out(w, h);
    if (n == 1 || params.top_rule == TOP_AVERAGE) {
        T inv = T(1) / (T)n;
        for (auto& t : tops)
            for (int c = 0; c < 3; c++)
                for (size_t i = 0; i < sz; i++) out.p[c][i] += t.p[c][i] * inv;
        return out;
    }
    std::vector<std::vector<T>> D(n), E(n);
    for (size_t k = 0; k < n; k++) {
        std::vector<T> y(sz);
        for (size_t i = 0; i < sz; i++) y[i] = luma_of<T>(tops[k].p[0][i], tops[k].p[1][i], tops[k].p[2][i]);
        deviation_entropy<T>(y.data(), w, h, params.top_radius, params.entropy_bins, D[k], E[k]);
    }
    bool use_entropy = params.top_rule == TOP_DEV_ENTROPY;
    std::vector<char> keep(n);
    for (size_t i = 0; i < sz; i++) {
        size_t kept = 0;
        for (size_t a = 0; a < n; a++) {
            T da = D[a][i], ea = E[a][i];
            bool dominated = false;
            for (size_t b = 0; b < n; b++) {
                if (a == b) continue;
                T db = D[b][i], eb = E[b][i];
                bool d = use_entropy ? (db >= da && eb >= ea && (db > da || eb > ea)) : (db > da || (db == da && b < a));
                if (d) {
                    dominated = true;
                    break;
                }
            }
            keep[a] = !dominated;
            kept += !dominated;
        }
        T inv = T(1) / (T)std::max<size_t>(kept, 1);
        for (size_t a = 0; a < n; a++)
            if (keep[a])
                for (int c = 0; c < 3; c++) out.p[c][i] += tops[a].p[c][i] * inv;
    }
    return out;
}

// fuse.rs:315 `winner_shares`
template <class W>
std::vector<float> winner_shares(const W* win, const float* best, size_t cells, size_t frames) {
    float mx = 0.0f;
    for (size_t i = 0; i < cells; i++) mx = std::max(mx, best[i]);
    float floor_ = DETAIL_FLOOR * mx;
    std::vector<size_t> counts(frames, 0);
    size_t total = 0;
    for (size_t i = 0; i < cells; i++) {
        if (best[i] > floor_ && floor_ > 0.0f) {
            size_t k = (size_t)std::round((float)win[i]);
            if (k < frames) {
                counts[k]++;
                total++;
            }
        }
    }
    std::vector<float> o(frames);
    for (size_t k = 0; k < frames; k++) o[k] = total > 0 ? (float)counts[k] / (float)total : 0.0f;
    return o;
}

// fuse.rs:336 `upsample_index`
template <class W>
std::vector<float> upsample_index(const W* win, size_t dw, size_t dh, size_t w, size_t h, size_t level) {
    size_t scale = (size_t)1 << level;
    std::vector<float> d(w * h);
    for (size_t y = 0; y < h; y++) {
        size_t sy = std::min(y / scale, dh - 1);
        for (size_t x = 0; x < w; x++) d[y * w + x] = (float)win[sy * dw + std::min(x / scale, dw - 1)];
    }
    return d;
}

// fuse.rs:349 `Fuser`: the incremental N-frame accumulator.
template <class T>
struct Fuser {
    size_t w, h, levels, depth_level;
    FuseParams params;
    std::vector<Img3<T>> acc;
    std::vector<std::vector<T>> best;
    std::vector<uint16_t> winner;
    std::vector<Img3<T>> tops;
    bool halo_on = false;
    size_t halo_guide = 0;
    T halo_p = T(0);
    size_t count = 0;
    int storage = 0;  // the engine's level storage to emulate (STORE_*; 0 = the reference's f32)

    Fuser(size_t w_, size_t h_, const FuseParams& p) : w(w_), h(h_), params(p) {
        levels = std::max<size_t>(p.levels ? p.levels : auto_levels(w, h, 32), 1);
        depth_level = std::min(p.depth_level, levels - 1);
        if (p.halo > 0.0f) {  // fuse.rs:120 `halo_guide`
            halo_on = true;
            halo_guide = std::min(p.depth_level, levels - 1);
            halo_p = (T)std::min(p.halo, HALO_MAX);
        }
    }
    size_t select_levels() const { return halo_on ? halo_guide + 1 : levels; }

    // fuse.rs:401 `push`; `max_gain`: the frame's largest brightness gain (the 16-bit storage's scale)
    void push(const Img3<T>& frame, float max_gain = 1.0f) {
        const float g = std::max(1.0f, max_gain);
        const float scale[2] = {(float)(65535.0 / g), (float)(g / 65535.0)};
        std::vector<Img3<T>> pyr = build(frame, levels, storage, scale);
        size_t nsel = select_levels();
        uint16_t idx = (uint16_t)count;
        bool first = count == 0;
        std::vector<std::vector<T>> energies(nsel);
        for (size_t l = 0; l < nsel; l++) energies[l] = region_energy(pyr[l], params.energy_radius, params.use_chroma);
        if (first) {
            winner.assign(pyr[depth_level].w * pyr[depth_level].h, 0);
            best = energies;
        } else {
            for (size_t li = 0; li < nsel; li++) {
                const Img3<T>& l = pyr[li];
                const std::vector<T>& en = energies[li];
                std::vector<T>& bs = best[li];
                Img3<T>& a = acc[li];
                size_t n = l.w * l.h;
                for (size_t i = 0; i < n; i++) {
                    if (en[i] > bs[i]) {
                        bs[i] = en[i];
                        a.p[0][i] = l.p[0][i];
                        a.p[1][i] = l.p[1][i];
                        a.p[2][i] = l.p[2][i];
                        if (li == depth_level) winner[i] = idx;
                    }
                }
            }
        }
        if (halo_on) {
            std::vector<T> wgt(energies[halo_guide].size());
            for (size_t i = 0; i < wgt.size(); i++) wgt[i] = halo_weight<T>(energies[halo_guide][i], halo_p);
            size_t ww = pyr[halo_guide].w, wh = pyr[halo_guide].h;
            for (size_t li = halo_guide + 1; li <= levels; li++) {
                std::vector<T> nw;
                size_t nww, nwh;
                reduce<T>(wgt.data(), ww, wh, nw, nww, nwh);
                wgt.swap(nw);
                ww = nww;
                wh = nwh;
                if (first) {
                    for (int c = 0; c < 3; c++)
                        for (size_t i = 0; i < wgt.size(); i++) pyr[li].p[c][i] *= wgt[i];
                    best.push_back(wgt);
                } else {
                    for (size_t i = 0; i < wgt.size(); i++) best[li][i] += wgt[i];
                    for (int c = 0; c < 3; c++)
                        for (size_t i = 0; i < wgt.size(); i++) acc[li].p[c][i] += wgt[i] * pyr[li].p[c][i];
                }
            }
            if (first) acc = std::move(pyr);
        } else {
            Img3<T> top = std::move(pyr.back());
            pyr.pop_back();
            if (first) acc = std::move(pyr);
            tops.push_back(std::move(top));
        }
        count++;
    }

    // fuse.rs:489 `shares`
    std::vector<float> shares() const {
        if (count == 0 || depth_level >= select_levels()) return {};
        std::vector<float> b(best[depth_level].size());
        for (size_t i = 0; i < b.size(); i++) b[i] = (float)best[depth_level][i];
        return winner_shares(winner.data(), b.data(), b.size(), count);
    }

    // fuse.rs:499 `finish`: the fused image (clamped) and the upsampled winner map.
    void finish(Img3<T>& img, std::vector<float>& depth) {
        size_t dw = acc[depth_level].w, dh = acc[depth_level].h;
        std::vector<Img3<T>> pyr = std::move(acc);
        if (halo_on) {
            for (size_t li = halo_guide + 1; li <= levels; li++)
                for (int c = 0; c < 3; c++)
                    for (size_t i = 0; i < pyr[li].p[c].size(); i++) pyr[li].p[c][i] /= best[li][i];
        } else {
            pyr.push_back(fuse_residuals(tops, params));
        }
        img = collapse(std::move(pyr));
        for (int c = 0; c < 3; c++)
            for (auto& v : img.p[c]) v = std::min(std::max(v, T(0)), T(1));
        depth = upsample_index(winner.data(), dw, dh, w, h, depth_level);
    }
};

}  // namespace orc
