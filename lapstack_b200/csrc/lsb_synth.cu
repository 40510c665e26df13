// Seeded synthetic focus stacks (the benchmark inputs; no reference
// counterpart): a height field of 12 random Gaussians normalised to [0,1], a
// band-limited noise texture (white noise blurred at sigma 1.5, mean 0.45,
// std 0.15 per channel), and per frame k a focal plane f_k = k/(n-1), a
// per-pixel defocus blur of sigma = blur_px * |z - f_k|, a magnification of
// 1 + mag_step*k about the centre (plus, when asked, a seeded similarity
// warp), additive Gaussian noise and quantisation to u16.
//
// The spatially varying blur is a blend of the texture pre-blurred at sigma
// 0, 0.5, 1, ..., blur_px (linear in sigma between neighbours). Random numbers
// come from a counter-based hash, so a pixel's value does not depend on the
// thread that makes it. The same functions run on the host (OpenMP) and on
// the device.
#include <math.h>
#include <omp.h>

#include <algorithm>
#include <vector>

#include "lsb_common.cuh"
#include "lapstack_b200.h"

namespace lsb {

LSB_HD uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
LSB_HD float u01(uint64_t seed, uint64_t stream, uint64_t idx) {
    uint64_t h = mix64(seed ^ mix64(stream * 0xD1B54A32D192ED03ull + idx));
    return (float)(h >> 40) * (1.0f / 16777216.0f);
}
// An approximately standard normal value: the Irwin-Hall sum of four uniforms.
LSB_HD float gauss4(uint64_t seed, uint64_t stream, uint64_t idx) {
    float s = u01(seed, stream, 4 * idx) + u01(seed, stream, 4 * idx + 1) + u01(seed, stream, 4 * idx + 2) + u01(seed, stream, 4 * idx + 3);
    return (s - 2.0f) * 1.7320508f;
}

struct Blob {
    double cx, cy, inv2s2, amp;
};
struct SynthPlan {
    int w, h, n, nb;
    uint64_t seed;
    Blob blobs[12];
    float tex_scale;             // 0.15 / std of the blurred noise
    float gk[32][40];            // Gaussian kernels per level (radius <= 19)
    int grad[32];
    double xf[1024][4];          // per frame: scale, cos, sin, (tx, ty packed below)
    double tx[1024], ty[1024];
    float focal[1024];
};

static void plan_of(const lsb_synth_desc& d, SynthPlan& p) {
    p.w = (int)d.w;
    p.h = (int)d.h;
    p.n = (int)d.n;
    p.seed = d.seed;
    p.nb = (int)ceilf(d.blur_px / 0.5f) + 1;
    if (p.nb < 2) p.nb = 2;
    if (p.nb > 32) p.nb = 32;
    for (int i = 0; i < 12; i++) {
        double cx = u01(d.seed, 1, 4 * i) * d.w, cy = u01(d.seed, 1, 4 * i + 1) * d.h;
        double sg = 40.0 + 160.0 * u01(d.seed, 1, 4 * i + 2), a = 0.2 + 0.8 * u01(d.seed, 1, 4 * i + 3);
        p.blobs[i] = Blob{cx, cy, 1.0 / (2.0 * sg * sg), a};
    }
    // texture: white noise U(-.5, .5) blurred at sigma 1.5 (radius 5)
    double g[6], s = 0.0, s2 = 0.0;
    for (int i = 0; i <= 5; i++) g[i] = exp(-(double)(i * i) / (2.0 * 1.5 * 1.5));
    for (int i = -5; i <= 5; i++) s += g[abs(i)];
    for (int i = -5; i <= 5; i++) s2 += (g[abs(i)] / s) * (g[abs(i)] / s);
    p.tex_scale = (float)(0.15 / (sqrt(1.0 / 12.0) * s2));
    for (int j = 0; j < p.nb; j++) {
        double sg = j == 0 ? 1.5 : 0.5 * j;  // level 0 holds the texture blur itself
        int r = std::min(19, (int)ceil(3.0 * sg));
        p.grad[j] = r;
        double t = 0.0;
        for (int i = -r; i <= r; i++) t += exp(-(double)(i * i) / (2.0 * sg * sg));
        for (int i = 0; i <= r; i++) p.gk[j][i] = (float)(exp(-(double)(i * i) / (2.0 * sg * sg)) / t);
    }
    for (int k = 0; k < p.n && k < 1024; k++) {
        double sc = 1.0 + (double)d.mag_step * k, rot = 0.0, tx = 0.0, ty = 0.0;
        if (d.warp && k > 0) {
            sc *= 1.0 + d.warp_scale * (2.0 * u01(d.seed, 2, 4 * k) - 1.0);
            rot = d.warp_rot_deg * (M_PI / 180.0) * (2.0 * u01(d.seed, 2, 4 * k + 1) - 1.0);
            tx = d.warp_shift * (2.0 * u01(d.seed, 2, 4 * k + 2) - 1.0);
            ty = d.warp_shift * (2.0 * u01(d.seed, 2, 4 * k + 3) - 1.0);
        }
        p.xf[k][0] = sc;
        p.xf[k][1] = cos(rot);
        p.xf[k][2] = sin(rot);
        p.tx[k] = tx;
        p.ty[k] = ty;
        p.focal[k] = p.n > 1 ? (float)k / (float)(p.n - 1) : 0.5f;
    }
}

LSB_HD double zraw_at(const SynthPlan& p, int x, int y) {
    double z = 0.0;
    for (int i = 0; i < 12; i++) {
        double dx = x - p.blobs[i].cx, dy = y - p.blobs[i].cy;
        z += p.blobs[i].amp * exp(-(dx * dx + dy * dy) * p.blobs[i].inv2s2);
    }
    return z;
}

// one separable pass (axis 0: rows, 1: columns) of level j's Gaussian, reflect-101
LSB_HD float blur_at(const SynthPlan& p, const float* src, int j, int x, int y, int axis) {
    const int r = p.grad[j];
    float s = 0.f;
    for (int i = -r; i <= r; i++) {
        float wv = p.gk[j][i < 0 ? -i : i];
        int xx = axis == 0 ? lsb_reflect(x + i, p.w) : x, yy = axis == 1 ? lsb_reflect(y + i, p.h) : y;
        s += wv * src[(size_t)yy * p.w + xx];
    }
    return s;
}

// the blurred scene of frame k at an integer point, channel c
LSB_HD float scene_at(const SynthPlan& p, const float* z, const float* B, float blur_px, int k, int c, int x, int y) {
    const size_t plane = (size_t)p.w * p.h;
    float sg = blur_px * fabsf(z[(size_t)y * p.w + x] - p.focal[k]);
    float t = sg / 0.5f;
    int j = (int)t;
    if (j > p.nb - 2) j = p.nb - 2;
    float fr = fminf(t - (float)j, 1.0f);
    // level 0 is the texture itself (sigma 0)
    const float* b0 = B + ((size_t)j * 3 + c) * plane;
    const float* b1 = B + ((size_t)(j + 1) * 3 + c) * plane;
    size_t o = (size_t)y * p.w + x;
    return b0[o] + fr * (b1[o] - b0[o]);
}

LSB_HD uint16_t frame_px(const SynthPlan& p, const lsb_synth_desc& d, const float* z, const float* B, int k, int c, int x, int y) {
    const double cx0 = p.w / 2.0, cy0 = p.h / 2.0;
    double qx = x - cx0 - p.tx[k], qy = y - cy0 - p.ty[k];
    double sc = p.xf[k][0], co = p.xf[k][1], si = p.xf[k][2];
    double px = (co * qx + si * qy) / sc + cx0, py = (-si * qx + co * qy) / sc + cy0;
    px = fmin(fmax(px, 0.0), (double)(p.w - 1));
    py = fmin(fmax(py, 0.0), (double)(p.h - 1));
    int ix = (int)px, iy = (int)py;
    int ix1 = ix + 1 < p.w ? ix + 1 : ix, iy1 = iy + 1 < p.h ? iy + 1 : iy;
    float fx = (float)(px - ix), fy = (float)(py - iy);
    float v00 = scene_at(p, z, B, d.blur_px, k, c, ix, iy), v01 = scene_at(p, z, B, d.blur_px, k, c, ix1, iy);
    float v10 = scene_at(p, z, B, d.blur_px, k, c, ix, iy1), v11 = scene_at(p, z, B, d.blur_px, k, c, ix1, iy1);
    float v = (v00 + fx * (v01 - v00)) * (1.f - fy) + (v10 + fx * (v11 - v10)) * fy;
    v += d.noise_std * gauss4(p.seed, 100 + (uint64_t)k * 3 + c, (uint64_t)y * p.w + x);
    v = fminf(fmaxf(v, 0.f), 1.f);
    return (uint16_t)(v * 65535.f + 0.5f);
}

// ------------------------------------------------------------------ device
__global__ void zraw_kernel(const SynthPlan* p, float* z) {
    size_t n = (size_t)p->w * p->h;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        z[i] = (float)zraw_at(*p, (int)(i % p->w), (int)(i / p->w));
}
__global__ void minmax_kernel(const float* z, size_t n, unsigned* mm) {
    float lo = 3.4e38f, hi = 0.f;  // z >= 0
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        lo = fminf(lo, z[i]);
        hi = fmaxf(hi, z[i]);
    }
    atomicMin(&mm[0], __float_as_uint(lo));  // z >= 0: float order is uint order
    atomicMax(&mm[1], __float_as_uint(hi));
}
__global__ void znorm_kernel(float* z, size_t n, const unsigned* mm) {
    float lo = __uint_as_float(mm[0]), hi = __uint_as_float(mm[1]);
    float inv = hi > lo ? 1.f / (hi - lo) : 0.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) z[i] = (z[i] - lo) * inv;
}
__global__ void noise_kernel(const SynthPlan* p, float* t) {
    size_t n = (size_t)p->w * p->h;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 3 * n; i += (size_t)gridDim.x * blockDim.x)
        t[i] = u01(p->seed, 10 + i / n, i % n) - 0.5f;
}
__global__ void blur_kernel(const SynthPlan* p, const float* src, float* dst, int j, int axis, float scale, float offset) {
    size_t n = (size_t)p->w * p->h;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 3 * n; i += (size_t)gridDim.x * blockDim.x) {
        size_t c = i / n, o = i % n;
        dst[i] = offset + scale * blur_at(*p, src + c * n, j, (int)(o % p->w), (int)(o / p->w), axis);
    }
}
__global__ void frames_kernel(const SynthPlan* p, lsb_synth_desc d, const float* z, const float* B, uint16_t* out) {
    size_t n = (size_t)p->w * p->h;
    size_t tot = n * p->n * 3;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
        size_t k = i / (3 * n), r = i % (3 * n), o = r / 3;
        int c = (int)(r % 3);
        out[i] = frame_px(*p, d, z, B, (int)k, c, (int)(o % p->w), (int)(o / p->w));
    }
}

static int gsz(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 32); }

}  // namespace lsb

using namespace lsb;

extern "C" {

// Truth of the applied per-frame transforms: [scale, rot (rad), tx (px), ty (px)] each.
static void fill_truth(const SynthPlan& p, double* truth) {
    if (!truth) return;
    for (int k = 0; k < p.n; k++) {
        truth[4 * k] = p.xf[k][0];
        truth[4 * k + 1] = atan2(p.xf[k][2], p.xf[k][1]);
        truth[4 * k + 2] = p.tx[k];
        truth[4 * k + 3] = p.ty[k];
    }
}

const char* lsb_synth_stack_host(const lsb_synth_desc* d, uint16_t* out, double* truth) {
    if (!d || !out || d->w == 0 || d->h == 0 || d->n == 0 || d->n > 1024) return "synth: bad description";
    SynthPlan* pp = new SynthPlan();
    SynthPlan& p = *pp;
    plan_of(*d, p);
    size_t n = (size_t)p.w * p.h;
    std::vector<float> z(n), t(3 * n), tmp(3 * n), B((size_t)p.nb * 3 * n);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) z[i] = (float)zraw_at(p, (int)(i % p.w), (int)(i / p.w));
    float lo = *std::min_element(z.begin(), z.end()), hi = *std::max_element(z.begin(), z.end());
    float inv = hi > lo ? 1.f / (hi - lo) : 0.f;
    for (auto& v : z) v = (v - lo) * inv;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)(3 * n); i++) t[i] = u01(p.seed, 10 + i / n, i % n) - 0.5f;
    for (int j = 0; j < p.nb; j++) {
        const float* src = j == 0 ? t.data() : B.data();  // levels >= 1 blur the texture (level 0)
        float sc = j == 0 ? p.tex_scale : 1.f, off = j == 0 ? 0.45f : 0.f;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)(3 * n); i++) tmp[i] = blur_at(p, src + (i / n) * n, j, (int)((i % n) % p.w), (int)((i % n) / p.w), 0);
        float* dst = B.data() + (size_t)j * 3 * n;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)(3 * n); i++)
            dst[i] = off + sc * blur_at(p, tmp.data() + (i / n) * n, j, (int)((i % n) % p.w), (int)((i % n) / p.w), 1);
    }
    size_t tot = n * p.n * 3;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)tot; i++) {
        size_t k = i / (3 * n), r = i % (3 * n), o = r / 3;
        out[i] = frame_px(p, *d, z.data(), B.data(), (int)k, (int)(r % 3), (int)(o % p.w), (int)(o / p.w));
    }
    fill_truth(p, truth);
    delete pp;
    return nullptr;
}

const char* lsb_synth_stack_device(const lsb_synth_desc* d, uint16_t* out_dev, double* truth, void* stream) {
    if (!d || !out_dev || d->w == 0 || d->h == 0 || d->n == 0 || d->n > 1024) return "synth: bad description";
    cudaStream_t s = (cudaStream_t)stream;
    SynthPlan* hp = new SynthPlan();
    plan_of(*d, *hp);
    size_t n = (size_t)hp->w * hp->h;
    SynthPlan* dp = nullptr;
    float *z = nullptr, *t = nullptr, *B = nullptr;
    unsigned* mm = nullptr;
    const char* err = nullptr;
    if (cudaMalloc(&dp, sizeof(SynthPlan)) != cudaSuccess || cudaMalloc(&z, n * 4) != cudaSuccess ||
        cudaMalloc(&t, 3 * n * 4) != cudaSuccess || cudaMalloc(&B, (size_t)hp->nb * 3 * n * 4) != cudaSuccess ||
        cudaMalloc(&mm, 8) != cudaSuccess) {
        err = "synth: device allocation failed";
    } else {
        cudaMemcpyAsync(dp, hp, sizeof(SynthPlan), cudaMemcpyHostToDevice, s);
        unsigned init[2] = {0x7f7fffffu, 0u};
        cudaMemcpyAsync(mm, init, 8, cudaMemcpyHostToDevice, s);
        lsb_launched(), zraw_kernel<<<gsz(n), 256, 0, s>>>(dp, z);
        lsb_launched(), minmax_kernel<<<gsz(n), 256, 0, s>>>(z, n, mm);
        lsb_launched(), znorm_kernel<<<gsz(n), 256, 0, s>>>(z, n, mm);
        lsb_launched(), noise_kernel<<<gsz(3 * n), 256, 0, s>>>(dp, t);
        for (int j = 0; j < hp->nb; j++) {
            const float* src = j == 0 ? t : B;
            float* tmp = j == 0 ? B + 3 * n : t;  // scratch: level 1's slot (not yet written) / the spent noise
            float sc = j == 0 ? hp->tex_scale : 1.f, off = j == 0 ? 0.45f : 0.f;
            lsb_launched(), blur_kernel<<<gsz(3 * n), 256, 0, s>>>(dp, src, tmp, j, 0, 1.f, 0.f);
            lsb_launched(), blur_kernel<<<gsz(3 * n), 256, 0, s>>>(dp, tmp, B + (size_t)j * 3 * n, j, 1, sc, off);
        }
        lsb_launched(), frames_kernel<<<gsz(n * hp->n * 3), 256, 0, s>>>(dp, *d, z, B, out_dev);
        if (cudaStreamSynchronize(s) != cudaSuccess) err = "synth: device generation failed";
    }
    cudaFree(dp);
    cudaFree(z);
    cudaFree(t);
    cudaFree(B);
    cudaFree(mm);
    fill_truth(*hp, truth);
    delete hp;
    return err;
}

}  // extern "C"
