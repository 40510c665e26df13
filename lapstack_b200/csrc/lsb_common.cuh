// Shared device helpers of the lapstack-b200 engine (sm_100a).
//
// Arithmetic that must be bit-identical to the reference's FP32 CPU path
// (crates/lapstack-core/src/pyramid.rs, fuse.rs) is written with explicit
// __fmul_rn / __fadd_rn / __fsub_rn so that no a*b+c is contracted into an
// FMA whatever the compiler flags: the reference's rustc build never fuses.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#define LSB_HD __host__ __device__ __forceinline__

// Every kernel launch of the engine counts itself (lsb_launch_count in the C ABI).
void lsb_launched();
// Graph replays count the kernels they hold; a capture takes back the counts its launches added.
void lsb_launched_add(long long k);
uint64_t lsb_launched_now();

// Reflect-101 into [0, n) (pyramid.rs:51 `reflect`): period 2(n-1); n == 1 maps to 0.
LSB_HD int lsb_reflect(int i, int n) {
    if (n == 1) return 0;
    if (i >= 0 && i < n) return i;
    int p = 2 * (n - 1);
    i %= p;
    if (i < 0) i += p;
    return i < n ? i : p - i;
}

// BT.601 luma with the reference's f32 literals and left-to-right order
// (fuse.rs:160, depth.rs:163, align.rs:567).
__device__ __forceinline__ float lsb_luma(float r, float g, float b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(0.299f, r), __fmul_rn(0.587f, g)), __fmul_rn(0.114f, b));
}

// u16 -> [0,1] as v * (1/65535) in f32 (io.rs:89-94).
#define LSB_INV16 (1.0f / 65535.0f)

// pyramid.rs:46 KERNEL and pyramid.rs:124-125 EVEN / ODD.
#define LSB_K0 (1.0f / 16.0f)
#define LSB_K1 (4.0f / 16.0f)
#define LSB_K2 (6.0f / 16.0f)
#define LSB_E0 (2.0f * LSB_K0)
#define LSB_E1 (2.0f * LSB_K2)
#define LSB_OD (2.0f * LSB_K1)

// a5 = ((((k0*s0 + k1*s1) + k2*s2) + k1*s3) + k0*s4), the order of pyramid.rs:95/111.
__device__ __forceinline__ float lsb_tap5(float s0, float s1, float s2, float s3, float s4) {
    float a = __fmul_rn(LSB_K0, s0);
    a = __fadd_rn(a, __fmul_rn(LSB_K1, s1));
    a = __fadd_rn(a, __fmul_rn(LSB_K2, s2));
    a = __fadd_rn(a, __fmul_rn(LSB_K1, s3));
    return __fadd_rn(a, __fmul_rn(LSB_K0, s4));
}
// EXPAND taps (pyramid.rs:128-166): even = E0*a + E1*b + E0*c, odd = OD*(a + b).
__device__ __forceinline__ float lsb_exp_even(float a, float b, float c) {
    return __fadd_rn(__fadd_rn(__fmul_rn(LSB_E0, a), __fmul_rn(LSB_E1, b)), __fmul_rn(LSB_E0, c));
}
__device__ __forceinline__ float lsb_exp_odd(float a, float b) { return __fmul_rn(LSB_OD, __fadd_rn(a, b)); }

// 16-bit fixed point over [0, 1/inv]: the Gaussian levels are convex
// combinations of 16-bit inputs, so UNORM16 keeps them at the inputs' own
// quantisation step (IEEE half would round them to 11 bits).
struct unorm16 {
    uint16_t v;
};

// Load / store a pyramid sample in its storage type; `sc` = (scale, 1/scale)
// of the fixed-point format (unused by the floating-point ones).
template <class S>
struct Store;
template <>
struct Store<float> {
    static __device__ __forceinline__ float ld(const float* p, float2) { return *p; }
    static __device__ __forceinline__ void st(float* p, float v, float2) { *p = v; }
    static __device__ __forceinline__ float as_stored(float v, float2) { return v; }
};
template <>
struct Store<__half> {
    static __device__ __forceinline__ float ld(const __half* p, float2) { return __half2float(*p); }
    static __device__ __forceinline__ void st(__half* p, float v, float2) { *p = __float2half_rn(v); }
    static __device__ __forceinline__ float as_stored(float v, float2) { return __half2float(__float2half_rn(v)); }
};
template <>
struct Store<unorm16> {
    static __device__ __forceinline__ uint16_t enc(float v, float2 sc) {
        return (uint16_t)fminf(fmaxf(__fadd_rn(__fmul_rn(v, sc.x), 0.5f), 0.f), 65535.f);
    }
    static __device__ __forceinline__ float dec(uint16_t u, float2 sc) { return __fmul_rn((float)u, sc.y); }
    static __device__ __forceinline__ float ld(const unorm16* p, float2 sc) { return dec(p->v, sc); }
    static __device__ __forceinline__ void st(unorm16* p, float v, float2 sc) { p->v = enc(v, sc); }
    static __device__ __forceinline__ float as_stored(float v, float2 sc) { return dec(enc(v, sc), sc); }
};

template <class S>
__device__ __forceinline__ float lsb_ld(const S* p);
template <>
__device__ __forceinline__ float lsb_ld<float>(const float* p) { return *p; }
template <>
__device__ __forceinline__ float lsb_ld<__half>(const __half* p) { return __half2float(*p); }
template <class S>
__device__ __forceinline__ void lsb_st(S* p, float v);
template <>
__device__ __forceinline__ void lsb_st<float>(float* p, float v) { *p = v; }
template <>
__device__ __forceinline__ void lsb_st<__half>(__half* p, float v) { *p = __float2half_rn(v); }

// depth.rs:201 `upsample_bilinear` along one axis: the grid coordinate of output pixel x
// ((x + 0.5) / k - 0.5, clamped), its two grid neighbours and the weight of the second.
__device__ __forceinline__ void bil_axis(int x, float inv, int dn, int& x0, int& x1, float& t) {
    const float f = fminf(fmaxf(__fsub_rn(__fmul_rn(__fadd_rn((float)x, 0.5f), inv), 0.5f), 0.f), (float)(dn - 1));
    x0 = (int)f;
    x1 = min(x0 + 1, dn - 1);
    t = __fsub_rn(f, (float)x0);
}
// ... and the bilinear value of a grid plane g (dw wide) there, in the reference's order
__device__ __forceinline__ float bil(const float* g, int dw, int x0, int x1, int y0, int y1, float tx, float ty) {
    const float* r0 = g + (size_t)y0 * dw;
    const float* r1 = g + (size_t)y1 * dw;
    const float top = __fadd_rn(r0[x0], __fmul_rn(__fsub_rn(r0[x1], r0[x0]), tx));
    const float bot = __fadd_rn(r1[x0], __fmul_rn(__fsub_rn(r1[x1], r1[x0]), tx));
    return __fadd_rn(top, __fmul_rn(__fsub_rn(bot, top), ty));
}
// Error flag bits a kernel may raise in the engine's device status word.
enum { LSB_ERR_BOUNDS = 1, LSB_ERR_TIMEOUT = 2, LSB_ERR_SHAPE = 4 };
