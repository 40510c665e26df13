// Interpolation kernels of the warp (crates/lapstack-core/src/align.rs:
// 413-474, Interp ids in Interp::ALL order) and the level-0 pixel loader
// shared by the fold and the registration kernels. f64 weights rounded to
// f32 as align.rs:508 does, f32 tap sums in the reference's order.
#pragma once
#include "lsb_common.cuh"
#include "lsb_internal.h"

namespace lsb {

// -------------------------------------------------------------- level-0 warp
// align.rs:416 `spline4` in f64 (taps at -1..+2), rounded to f32 as warp_with does.
__device__ __forceinline__ void spline4_d(double t, float w[4]) {
    double w0 = __dmul_rn(__dsub_rn(__dmul_rn(__dadd_rn(__dmul_rn(-1.0 / 3.0, t), 0.8), t), 0.46666667), t);
    double w1 = __dadd_rn(__dmul_rn(__dsub_rn(__dmul_rn(__dsub_rn(t, 1.8), t), 0.2), t), 1.0);
    double w2 = __dmul_rn(__dadd_rn(__dmul_rn(__dsub_rn(1.2, t), t), 0.8), t);
    double w3 = __dmul_rn(__dsub_rn(__dmul_rn(__dsub_rn(__dmul_rn(1.0 / 3.0, t), 0.2), t), 0.13333334), t);
    w[0] = (float)w0;
    w[1] = (float)w1;
    w[2] = (float)w2;
    w[3] = (float)w3;
}

// align.rs:427 `keys`, :433 `spline36`, :449 `lanczos3`, :463 `taps_of`
__device__ __forceinline__ double keys_d(double d) {
    if (d < 1.0) return __dadd_rn(__dmul_rn(__dmul_rn(__dsub_rn(__dmul_rn(1.5, d), 2.5), d), d), 1.0);
    if (d < 2.0) return __dadd_rn(__dmul_rn(__dsub_rn(__dmul_rn(__dadd_rn(__dmul_rn(-0.5, d), 2.5), d), 4.0), d), 2.0);
    return 0.0;
}
__device__ __forceinline__ double spline36_d(double d) {
    if (d < 1.0)
        return __dadd_rn(__dmul_rn(__dsub_rn(__dmul_rn(__dsub_rn(__dmul_rn(13.0 / 11.0, d), 453.0 / 209.0), d), 3.0 / 209.0), d), 1.0);
    if (d < 2.0) {
        double u = __dsub_rn(d, 1.0);
        return __dmul_rn(__dsub_rn(__dmul_rn(__dadd_rn(__dmul_rn(-6.0 / 11.0, u), 270.0 / 209.0), u), 156.0 / 209.0), u);
    }
    if (d < 3.0) {
        double u = __dsub_rn(d, 2.0);
        return __dmul_rn(__dadd_rn(__dmul_rn(__dsub_rn(__dmul_rn(1.0 / 11.0, u), 45.0 / 209.0), u), 26.0 / 209.0), u);
    }
    return 0.0;
}
__device__ __forceinline__ double lanczos3_d(double d) {
    if (d < 1e-9) return 1.0;
    if (d < 3.0) {
        double a = __dmul_rn(3.141592653589793, d), b = __ddiv_rn(a, 3.0);
        return __dmul_rn(__ddiv_rn(sin(a), a), __ddiv_rn(sin(b), b));
    }
    return 0.0;
}
// The interpolation weights of kind k at fraction t; returns the tap count.
__device__ __forceinline__ int interp_w(int k, double t, float w[6]) {
    if (k == 0) {
        w[0] = t < 0.5 ? 1.f : 0.f;
        w[1] = t < 0.5 ? 0.f : 1.f;
        return 2;
    }
    if (k == 1) {
        w[0] = (float)__dsub_rn(1.0, t);
        w[1] = (float)t;
        return 2;
    }
    if (k == 3) {
        spline4_d(t, w);
        return 4;
    }
    int n = k == 2 ? 4 : 6;
    double wd[6], sum = 0.0;
    for (int i = 0; i < n; i++) {
        double d = fabs(__dsub_rn(t, __dsub_rn(__dadd_rn((double)i, 1.0), (double)(n / 2))));
        wd[i] = k == 2 ? keys_d(d) : (k == 4 ? spline36_d(d) : lanczos3_d(d));
        sum = __dadd_rn(sum, wd[i]);
    }
    for (int i = 0; i < n; i++) w[i] = (float)__ddiv_rn(wd[i], sum);
    return n;
}

// The level-0 value of pixel (x, y), all three channels: the u16 sample
// times 1/65535, warped by the frame's inverse homography (align.rs:489
// `warp_with`: f64 source point, f32 taps and sums, edge-clamped; the pixel
// as shot where the source point leaves the frame, stack.rs:668-679), then
// the brightness gains (brightness.rs:124).
__device__ __forceinline__ void load_px_core(const uint16_t* __restrict__ f, const double* inv, int warp, int affine, int interp,
                                             int W, int H, int x, int y, float v[3]) {
    if (warp) {
        double sx, sy, xd = (double)x, yd = (double)y;
        const double* m = inv;
        if (affine) {
            sx = __dadd_rn(__dadd_rn(__dmul_rn(m[1], yd), m[2]), __dmul_rn(m[0], xd));
            sy = __dadd_rn(__dadd_rn(__dmul_rn(m[4], yd), m[5]), __dmul_rn(m[3], xd));
        } else {
            double d = __dadd_rn(__dadd_rn(__dmul_rn(m[6], xd), __dmul_rn(m[7], yd)), m[8]);
            sx = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[0], xd), __dmul_rn(m[1], yd)), m[2]), d);
            sy = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[3], xd), __dmul_rn(m[4], yd)), m[5]), d);
        }
        bool valid = sx >= 0.0 && sx <= (double)(W - 1) && sy >= 0.0 && sy <= (double)(H - 1);
        if (valid) {
            double fx = floor(sx), fy = floor(sy);
            int ix = (int)fx, iy = (int)fy;
            float wx[6], wy[6];
            int n = interp_w(interp, __dsub_rn(sx, fx), wx);
            interp_w(interp, __dsub_rn(sy, fy), wy);
            int start = 1 - n / 2;
            float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f;
            for (int j = 0; j < n; j++) {
                int yy = min(max(iy + start + j, 0), H - 1);
                float r0 = 0.f, r1 = 0.f, r2 = 0.f;
                for (int i = 0; i < n; i++) {
                    int xx = min(max(ix + start + i, 0), W - 1);
                    const uint16_t* p = f + ((size_t)yy * W + xx) * 3;
                    r0 = __fadd_rn(r0, __fmul_rn(wx[i], __fmul_rn((float)p[0], LSB_INV16)));
                    r1 = __fadd_rn(r1, __fmul_rn(wx[i], __fmul_rn((float)p[1], LSB_INV16)));
                    r2 = __fadd_rn(r2, __fmul_rn(wx[i], __fmul_rn((float)p[2], LSB_INV16)));
                }
                acc0 = __fadd_rn(acc0, __fmul_rn(wy[j], r0));
                acc1 = __fadd_rn(acc1, __fmul_rn(wy[j], r1));
                acc2 = __fadd_rn(acc2, __fmul_rn(wy[j], r2));
            }
            v[0] = acc0;
            v[1] = acc1;
            v[2] = acc2;
        } else {
            const uint16_t* p = f + ((size_t)y * W + x) * 3;
            for (int c = 0; c < 3; c++) v[c] = __fmul_rn((float)p[c], LSB_INV16);
        }
    } else {
        const uint16_t* p = f + ((size_t)y * W + x) * 3;
        for (int c = 0; c < 3; c++) v[c] = __fmul_rn((float)p[c], LSB_INV16);
    }
}
__device__ __forceinline__ void load_u16_px(const uint16_t* __restrict__ f, const FrameXform& xf, int interp, int W, int H, int x,
                                            int y, float v[3]) {
    load_px_core(f, xf.inv, xf.warp, xf.affine, interp, W, H, x, y, v);
    for (int c = 0; c < 3; c++)
        if (xf.gain_on & (1 << c)) v[c] = __fmul_rn(v[c], xf.gain[c]);
}

}  // namespace lsb
