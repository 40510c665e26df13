// Oracle (test infrastructure only; see orc_core.hpp): a host twin of the
// engine's seeded synthetic stack generator, so that the CPU baseline can make
// its frames without loading the CUDA library. Same recipe and arithmetic as
// the engine's host path (tests/test_oracle_synth.py holds them equal byte for
// byte): a height field of 12 random Gaussians normalised to [0,1]; a texture
// of white noise blurred at sigma 1.5, scaled to mean 0.45, std 0.15 per
// channel; frame k focused at f_k = k/(n-1), blurred per pixel by sigma =
// blur_px * |z - f_k| (a blend of the texture pre-blurred at sigma 0, 0.5,
// 1, ...), magnified by 1 + mag_step*k about the centre (plus a seeded
// similarity warp when asked), with additive noise and u16 quantisation.
// Random numbers come from a counter-based hash (splitmix64 finaliser).
#pragma once
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>
#include <vector>

namespace orc {

struct SynthDesc {
    uint32_t w, h, n, warp;
    uint64_t seed;
    float mag_step, noise_std, blur_px, warp_scale, warp_rot_deg, warp_shift;
};

namespace synth {

inline uint64_t mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// uniform in [0, 1) from the top 24 bits of the hash of (seed, stream, index)
inline float uni(uint64_t seed, uint64_t stream, uint64_t idx) {
    const uint64_t hv = mix(seed ^ mix(stream * 0xD1B54A32D192ED03ull + idx));
    return (float)(hv >> 40) * (1.0f / 16777216.0f);
}
// approximately N(0, 1): four uniforms summed, centred and scaled (Irwin-Hall)
inline float normal(uint64_t seed, uint64_t stream, uint64_t idx) {
    float s = uni(seed, stream, 4 * idx) + uni(seed, stream, 4 * idx + 1) + uni(seed, stream, 4 * idx + 2) + uni(seed, stream, 4 * idx + 3);
    return (s - 2.0f) * 1.7320508f;
}
inline int mirror(int i, int n) {  // reflect-101
    if (n == 1) return 0;
    while (i < 0 || i >= n) i = i < 0 ? -i : 2 * (n - 1) - i;
    return i;
}

struct Plan {
    int w, h, n, levels;
    uint64_t seed;
    double cx[12], cy[12], k2[12], amp[12];
    float tex_scale;
    float taps[32][40];
    int radius[32];
    std::vector<double> scale, cosr, sinr, tx, ty;
    std::vector<float> focal;
};

inline void plan(const SynthDesc& d, Plan& p) {
    p.w = (int)d.w;
    p.h = (int)d.h;
    p.n = (int)d.n;
    p.seed = d.seed;
    p.levels = std::min(32, std::max(2, (int)ceilf(d.blur_px / 0.5f) + 1));
    for (int i = 0; i < 12; i++) {
        p.cx[i] = uni(d.seed, 1, 4 * i) * d.w;
        p.cy[i] = uni(d.seed, 1, 4 * i + 1) * d.h;
        const double sg = 40.0 + 160.0 * uni(d.seed, 1, 4 * i + 2);
        p.amp[i] = 0.2 + 0.8 * uni(d.seed, 1, 4 * i + 3);
        p.k2[i] = 1.0 / (2.0 * sg * sg);
    }
    // the texture: U(-1/2, 1/2) noise blurred at sigma 1.5 (radius 5), std brought to 0.15
    double g[6], s = 0.0, s2 = 0.0;
    for (int i = 0; i <= 5; i++) g[i] = exp(-(double)(i * i) / (2.0 * 1.5 * 1.5));
    for (int i = -5; i <= 5; i++) s += g[abs(i)];
    for (int i = -5; i <= 5; i++) s2 += (g[abs(i)] / s) * (g[abs(i)] / s);
    p.tex_scale = (float)(0.15 / (sqrt(1.0 / 12.0) * s2));
    for (int j = 0; j < p.levels; j++) {
        const double sg = j == 0 ? 1.5 : 0.5 * j;  // level 0 is the texture's own blur
        const int r = std::min(19, (int)ceil(3.0 * sg));
        p.radius[j] = r;
        double t = 0.0;
        for (int i = -r; i <= r; i++) t += exp(-(double)(i * i) / (2.0 * sg * sg));
        for (int i = 0; i <= r; i++) p.taps[j][i] = (float)(exp(-(double)(i * i) / (2.0 * sg * sg)) / t);
    }
    p.scale.assign(p.n, 1.0);
    p.cosr.assign(p.n, 1.0);
    p.sinr.assign(p.n, 0.0);
    p.tx.assign(p.n, 0.0);
    p.ty.assign(p.n, 0.0);
    p.focal.assign(p.n, 0.5f);
    for (int k = 0; k < p.n; k++) {
        double sc = 1.0 + (double)d.mag_step * k, rot = 0.0, ox = 0.0, oy = 0.0;
        if (d.warp && k > 0) {
            sc *= 1.0 + d.warp_scale * (2.0 * uni(d.seed, 2, 4 * k) - 1.0);
            rot = d.warp_rot_deg * (M_PI / 180.0) * (2.0 * uni(d.seed, 2, 4 * k + 1) - 1.0);
            ox = d.warp_shift * (2.0 * uni(d.seed, 2, 4 * k + 2) - 1.0);
            oy = d.warp_shift * (2.0 * uni(d.seed, 2, 4 * k + 3) - 1.0);
        }
        p.scale[k] = sc;
        p.cosr[k] = cos(rot);
        p.sinr[k] = sin(rot);
        p.tx[k] = ox;
        p.ty[k] = oy;
        if (p.n > 1) p.focal[k] = (float)k / (float)(p.n - 1);
    }
}

// one separable pass of level j's Gaussian along rows (axis 0) or columns (axis 1)
inline float pass(const Plan& p, const float* src, int j, int x, int y, int axis) {
    const int r = p.radius[j];
    float s = 0.f;
    for (int i = -r; i <= r; i++) {
        const int xx = axis == 0 ? mirror(x + i, p.w) : x, yy = axis == 1 ? mirror(y + i, p.h) : y;
        s += p.taps[j][i < 0 ? -i : i] * src[(size_t)yy * p.w + xx];
    }
    return s;
}

// frame k's blurred scene at an integer point, channel c: a blend of the two pre-blurred
// levels around sigma / 0.5
inline float scene(const Plan& p, const float* z, const float* B, float blur_px, int k, int c, int x, int y) {
    const size_t np = (size_t)p.w * p.h, o = (size_t)y * p.w + x;
    const float t = blur_px * fabsf(z[o] - p.focal[k]) / 0.5f;
    int j = (int)t;
    if (j > p.levels - 2) j = p.levels - 2;
    const float fr = fminf(t - (float)j, 1.0f);
    const float a = B[((size_t)j * 3 + c) * np + o], b = B[((size_t)(j + 1) * 3 + c) * np + o];
    return a + fr * (b - a);
}

inline uint16_t pixel(const Plan& p, const SynthDesc& d, const float* z, const float* B, int k, int c, int x, int y) {
    const double cx0 = p.w / 2.0, cy0 = p.h / 2.0;
    const double qx = x - cx0 - p.tx[k], qy = y - cy0 - p.ty[k];
    double px = (p.cosr[k] * qx + p.sinr[k] * qy) / p.scale[k] + cx0;
    double py = (-p.sinr[k] * qx + p.cosr[k] * qy) / p.scale[k] + cy0;
    px = fmin(fmax(px, 0.0), (double)(p.w - 1));
    py = fmin(fmax(py, 0.0), (double)(p.h - 1));
    const int ix = (int)px, iy = (int)py;
    const int ix1 = ix + 1 < p.w ? ix + 1 : ix, iy1 = iy + 1 < p.h ? iy + 1 : iy;
    const float fx = (float)(px - ix), fy = (float)(py - iy);
    const float v00 = scene(p, z, B, d.blur_px, k, c, ix, iy), v01 = scene(p, z, B, d.blur_px, k, c, ix1, iy);
    const float v10 = scene(p, z, B, d.blur_px, k, c, ix, iy1), v11 = scene(p, z, B, d.blur_px, k, c, ix1, iy1);
    float v = (v00 + fx * (v01 - v00)) * (1.f - fy) + (v10 + fx * (v11 - v10)) * fy;
    v += d.noise_std * normal(p.seed, 100 + (uint64_t)k * 3 + c, (uint64_t)y * p.w + x);
    v = fminf(fmaxf(v, 0.f), 1.f);
    return (uint16_t)(v * 65535.f + 0.5f);
}

}  // namespace synth

// frames k0 .. k0+count-1 of the n-frame stack, [count][h][w][3] u16, into out; truth (n*4, may be
// null): scale, rotation (rad), tx, ty of every frame
inline bool synth_stack(const SynthDesc& d, uint16_t* out, double* truth, uint32_t k0, uint32_t count) {
    using namespace synth;
    if (d.w == 0 || d.h == 0 || d.n == 0 || d.n > 1024 || k0 >= d.n || count == 0 || count > d.n - k0) return false;
    Plan p;
    plan(d, p);
    const size_t np = (size_t)p.w * p.h;
    std::vector<float> z(np), t(3 * np), tmp(3 * np), B((size_t)p.levels * 3 * np);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)np; i++) {
        const int x = (int)(i % p.w), y = (int)(i / p.w);
        double acc = 0.0;
        for (int b = 0; b < 12; b++) {
            const double dx = x - p.cx[b], dy = y - p.cy[b];
            acc += p.amp[b] * exp(-(dx * dx + dy * dy) * p.k2[b]);
        }
        z[i] = (float)acc;
    }
    const float lo = *std::min_element(z.begin(), z.end()), hi = *std::max_element(z.begin(), z.end());
    const float inv = hi > lo ? 1.f / (hi - lo) : 0.f;
    for (auto& v : z) v = (v - lo) * inv;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)(3 * np); i++) t[i] = uni(p.seed, 10 + i / np, i % np) - 0.5f;
    for (int j = 0; j < p.levels; j++) {
        const float* src = j == 0 ? t.data() : B.data();  // every level blurs the texture (level 0)
        const float sc = j == 0 ? p.tex_scale : 1.f, off = j == 0 ? 0.45f : 0.f;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)(3 * np); i++)
            tmp[i] = pass(p, src + (i / np) * np, j, (int)((i % np) % p.w), (int)((i % np) / p.w), 0);
        float* dst = B.data() + (size_t)j * 3 * np;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)(3 * np); i++)
            dst[i] = off + sc * pass(p, tmp.data() + (i / np) * np, j, (int)((i % np) % p.w), (int)((i % np) / p.w), 1);
    }
    const size_t total = np * count * 3;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)total; i++) {
        const size_t k = k0 + i / (3 * np), r = i % (3 * np), o = r / 3;
        out[i] = pixel(p, d, z.data(), B.data(), (int)k, (int)(r % 3), (int)(o % p.w), (int)(o / p.w));
    }
    if (truth)
        for (int k = 0; k < p.n; k++) {
            truth[4 * k] = p.scale[k];
            truth[4 * k + 1] = atan2(p.sinr[k], p.cosr[k]);
            truth[4 * k + 2] = p.tx[k];
            truth[4 * k + 3] = p.ty[k];
        }
    return true;
}

}  // namespace orc
