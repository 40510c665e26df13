// The learned warm start of the WLS depth solve (no counterpart in the
// reference): a 4-level U-Net, 32 base channels, BF16 weights and
// activations with FP32 accumulation, that maps the quarter-resolution
// (guide luma, raw DfF depth, confidence) to the WLS solution. Its output is
// the x0 of MG-PCG, which then runs to the same relative residual as the
// plain solve, so the network changes only how fast the solve gets there.
//
// Layout: activations NHWC bf16 with channels a multiple of 32; weights
// [tap][cout][cin] bf16 for the forward conv (FP32 masters, Adam moments).
// conv3x3_kernel is an implicit GEMM on the tensor cores (mma.sync
// m16n8k16 bf16 -> f32): a CTA owns 8x16 output pixels x NT output
// channels; per 32-channel input chunk it stages the 10x18 input halo and the
// 9 x NT x 32 weights in shared memory (rows padded to 40 bf16 so the
// fragment loads hit 32 distinct banks). The same kernel computes dX in the
// backward pass with the flipped, transposed weights. The input loader reads
// a layer's input straight from where it lives: the previous activation, a
// 2x2 average pool of a finer one (encoder), a nearest 2x upsample of a
// coarser one (decoder), and the channel concat of an upsampled tensor with
// a skip tensor, so no pooled, upsampled or concatenated copy is written.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "lapstack_b200.h"
#include "lsb_common.cuh"

namespace lsb {

constexpr int UN_CH = 32;        // input-chunk channels
constexpr int UN_TH = 8, UN_TW = 16;  // output tile (pixels)
constexpr int UN_HP = UN_TH + 2, UN_WP = UN_TW + 2;
constexpr int UN_LD = UN_CH + 8;  // padded row (bf16)
constexpr int UN_THREADS = 128;

enum { SRC_SAME = 0, SRC_UP = 1, SRC_POOL = 2 };

struct ConvArgs {
    const __nv_bfloat16* src1;
    const __nv_bfloat16* src2;
    int c1, c1s, mode1;  // channels of source 1 read, its channel stride, its mode
    int c2s, mode2;      // source 2 (channels c1..cin-1), its channel stride
    int cin, cout;
    const __nv_bfloat16* w;  // [9][cout][cin]
    const float* bias;       // [cout] or null
    int relu;
    __nv_bfloat16* out;      // [B][H][W][cout] bf16, or null
    float* out_f32;          // [B][H][W][cout] f32, or null
    float* out_c0;           // [B][H][W] channel 0 only (f32), or null
    int B, H, W;             // output grid
};

__device__ __forceinline__ uint32_t bf2_as_u32(__nv_bfloat162 v) { return *reinterpret_cast<uint32_t*>(&v); }

// 8 consecutive channels (16 bytes) of one input pixel, through the source's mode.
__device__ __forceinline__ uint4 load8(const __nv_bfloat16* src, int cs, int mode, int b, int y, int x, int H, int W, int c) {
    if (mode == SRC_SAME) {
        return *reinterpret_cast<const uint4*>(src + (((size_t)b * H + y) * W + x) * cs + c);
    }
    if (mode == SRC_UP) {
        const int h2 = H >> 1, w2 = W >> 1;
        return *reinterpret_cast<const uint4*>(src + (((size_t)b * h2 + (y >> 1)) * w2 + (x >> 1)) * cs + c);
    }
    // SRC_POOL: the mean of the 2x2 block of the finer source
    const int H2 = H * 2, W2 = W * 2;
    float acc[8];
#pragma unroll
    for (int i = 0; i < 8; i++) acc[i] = 0.f;
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
#pragma unroll
        for (int dx = 0; dx < 2; dx++) {
            uint4 v = *reinterpret_cast<const uint4*>(src + (((size_t)b * H2 + 2 * y + dy) * W2 + 2 * x + dx) * cs + c);
            const __nv_bfloat162* p = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                float2 f = __bfloat1622float2(p[i]);
                acc[2 * i] += f.x;
                acc[2 * i + 1] += f.y;
            }
        }
    uint4 o;
    __nv_bfloat162* q = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
    for (int i = 0; i < 4; i++) q[i] = __floats2bfloat162_rn(acc[2 * i] * 0.25f, acc[2 * i + 1] * 0.25f);
    return o;
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// out[p][n] = sum_{tap, ci} X[p + off(tap)][ci] * w[tap][n][ci] (+ bias, ReLU), zero padding.
template <int NT>
__global__ void __launch_bounds__(UN_THREADS) conv3x3_kernel(const ConvArgs a) {
    extern __shared__ __align__(16) unsigned char un_smem[];
    __nv_bfloat16* xs = reinterpret_cast<__nv_bfloat16*>(un_smem);  // [UN_HP*UN_WP][UN_LD]
    __nv_bfloat16* ws = xs + UN_HP * UN_WP * UN_LD;                  // [9][NT][UN_LD]
    const int tiles_x = (a.W + UN_TW - 1) / UN_TW;
    const int x0 = (blockIdx.x % tiles_x) * UN_TW, y0 = (blockIdx.x / tiles_x) * UN_TH;
    const int n0 = blockIdx.y * NT, b = blockIdx.z;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    constexpr int NJ = NT / 8;
    float acc[2][NJ][4];
#pragma unroll
    for (int m = 0; m < 2; m++)
#pragma unroll
        for (int j = 0; j < NJ; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[m][j][q] = 0.f;

    for (int c0 = 0; c0 < a.cin; c0 += UN_CH) {
        const bool first = c0 < a.c1;
        const __nv_bfloat16* src = first ? a.src1 : a.src2;
        const int cs = first ? a.c1s : a.c2s, mode = first ? a.mode1 : a.mode2, cb = first ? c0 : c0 - a.c1;
        // stage the input halo: UN_HP*UN_WP pixels x 4 vectors of 8 channels
        for (int i = tid; i < UN_HP * UN_WP * 4; i += UN_THREADS) {
            const int pix = i >> 2, v = i & 3;
            const int yy = y0 - 1 + pix / UN_WP, xx = x0 - 1 + pix % UN_WP;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (yy >= 0 && yy < a.H && xx >= 0 && xx < a.W) val = load8(src, cs, mode, b, yy, xx, a.H, a.W, cb + 8 * v);
            *reinterpret_cast<uint4*>(xs + pix * UN_LD + 8 * v) = val;
        }
        // stage the weights of this chunk: 9 x NT rows of 32 channels
        for (int i = tid; i < 9 * NT * 4; i += UN_THREADS) {
            const int row = i >> 2, v = i & 3;
            const int tap = row / NT, n = row % NT;
            const uint4 val = *reinterpret_cast<const uint4*>(a.w + ((size_t)tap * a.cout + n0 + n) * a.cin + c0 + 8 * v);
            *reinterpret_cast<uint4*>(ws + row * UN_LD + 8 * v) = val;
        }
        __syncthreads();
#pragma unroll 1
        for (int tap = 0; tap < 9; tap++) {
            const int ky = tap / 3, kx = tap % 3;
#pragma unroll
            for (int kk = 0; kk < UN_CH; kk += 16) {
                uint32_t af[2][4];
#pragma unroll
                for (int m = 0; m < 2; m++) {
                    const int r = 2 * warp + m;  // tile row of this m16 block
                    const __nv_bfloat16* p0 = xs + ((r + ky) * UN_WP + g + kx) * UN_LD + kk + 2 * t;
                    const __nv_bfloat16* p1 = p0 + 8 * UN_LD;
                    af[m][0] = *reinterpret_cast<const uint32_t*>(p0);
                    af[m][1] = *reinterpret_cast<const uint32_t*>(p1);
                    af[m][2] = *reinterpret_cast<const uint32_t*>(p0 + 8);
                    af[m][3] = *reinterpret_cast<const uint32_t*>(p1 + 8);
                }
#pragma unroll
                for (int j = 0; j < NJ; j++) {
                    const __nv_bfloat16* q = ws + (tap * NT + 8 * j + g) * UN_LD + kk + 2 * t;
                    const uint32_t b0 = *reinterpret_cast<const uint32_t*>(q);
                    const uint32_t b1 = *reinterpret_cast<const uint32_t*>(q + 8);
                    mma_bf16(acc[0][j], af[0][0], af[0][1], af[0][2], af[0][3], b0, b1);
                    mma_bf16(acc[1][j], af[1][0], af[1][1], af[1][2], af[1][3], b0, b1);
                }
            }
        }
        __syncthreads();
    }
    // epilogue: c0,c1 -> (pixel g, channels 2t, 2t+1); c2,c3 -> pixel g+8
#pragma unroll
    for (int m = 0; m < 2; m++) {
        const int y = y0 + 2 * warp + m;
        if (y >= a.H) continue;
#pragma unroll
        for (int half = 0; half < 2; half++) {
            const int x = x0 + g + 8 * half;
            if (x >= a.W) continue;
            const size_t pix = ((size_t)b * a.H + y) * a.W + x;
#pragma unroll
            for (int j = 0; j < NJ; j++) {
                const int n = n0 + 8 * j + 2 * t;
                float v0 = acc[m][j][2 * half], v1 = acc[m][j][2 * half + 1];
                if (a.bias) {
                    v0 += a.bias[n];
                    v1 += a.bias[n + 1];
                }
                if (a.relu) {
                    v0 = fmaxf(v0, 0.f);
                    v1 = fmaxf(v1, 0.f);
                }
                if (a.out) *reinterpret_cast<__nv_bfloat162*>(a.out + pix * a.cout + n) = __floats2bfloat162_rn(v0, v1);
                if (a.out_f32) *reinterpret_cast<float2*>(a.out_f32 + pix * a.cout + n) = make_float2(v0, v1);
                if (a.out_c0 && n == 0) a.out_c0[pix] = v0;
            }
        }
    }
}

// ------------------------------------------------- the same conv on tcgen05
// conv3x3_tc_kernel: the implicit GEMM on the 5th-generation tensor cores. A CTA of 4 warps owns a
// 16 x 8 tile of output pixels (M = 128, one TMEM lane per pixel) and N = cout output channels (one
// fp32 TMEM column each). Per 32-channel input chunk every thread stages the 18 x 10 input halo and
// the chunk's 9 x N x 32 weights in shared memory in the canonical no-swizzle K-major layout of the
// UMMA operand descriptors (8 rows of 16 bytes per core matrix): the halo as [k8][pixel][8 channels],
// so that the tap (ky, kx) of the A operand is the same layout started (ky * 10 + kx) pixels later
// (rows of 8 pixels 10 pixels apart: SBO = 160 B, the next 8 channels LBO = 180 pixels further);
// the weights as [tap][k8][n][8]. One thread issues the 9 taps x 2 K-steps of tcgen05.mma
// (kind::f16, BF16 x BF16 -> FP32 in TMEM) and commits them to an mbarrier that every thread waits
// on (bounded) before the staging of the next chunk; the epilogue reads the accumulator with
// tcgen05.ld (warp w: lanes 32w..32w+31), adds the bias, applies ReLU and stores NHWC.
constexpr int TC_TH = 16, TC_TW = 8;
constexpr int TC_HP = TC_TH + 2, TC_WP = TC_TW + 2, TC_PIX = TC_HP * TC_WP;  // 18 x 10 halo
// try_wait polls per wait: far beyond a chunk's MMAs (microseconds); a CTA that meets a set error word
// (an earlier wait ran out) does nothing
constexpr unsigned TC_SPIN_LIMIT = 1u << 20;

__host__ __device__ constexpr size_t tc_a_bytes() { return (size_t)4 * TC_PIX * 16; }
__host__ __device__ constexpr size_t tc_b_bytes(int n) { return (size_t)9 * 4 * n * 16; }
// A, B, the mbarrier and the TMEM address slot
__host__ __device__ constexpr size_t tc_smem_bytes(int n) { return tc_a_bytes() + tc_b_bytes(n) + 16; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// the UMMA shared-memory descriptor, no swizzle (layout type 0), version 1; addresses and offsets in bytes
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
           (1ull << 46);
}
// the instruction descriptor of kind::f16: D f32, A and B bf16, both K-major, M = 128, N
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

template <int N>
__global__ void __launch_bounds__(UN_THREADS) conv3x3_tc_kernel(const ConvArgs a, int* status) {
    extern __shared__ __align__(128) unsigned char tc_smem[];
    unsigned char* As = tc_smem;
    unsigned char* Bs = tc_smem + tc_a_bytes();
    uint64_t* mbar = reinterpret_cast<uint64_t*>(Bs + tc_b_bytes(N));
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
    const int tiles_x = (a.W + TC_TW - 1) / TC_TW;
    const int x0 = (blockIdx.x % tiles_x) * TC_TW, y0 = (blockIdx.x / tiles_x) * TC_TH;
    const int n0 = blockIdx.y * N, b = blockIdx.z;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr uint32_t COLS = N < 32 ? 32 : N;
    if (*(volatile int*)status) return;  // an earlier CTA's wait ran out: nothing is allocated yet
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tslot;
    const uint32_t a_base = smem_u32(As), b_base = smem_u32(Bs);
    constexpr uint32_t IDESC = umma_idesc_bf16(N);
    bool ok = true;
    int chunk = 0;
    for (int c0 = 0; c0 < a.cin; c0 += UN_CH, chunk++) {
        const bool first = c0 < a.c1;
        const __nv_bfloat16* src = first ? a.src1 : a.src2;
        const int cs = first ? a.c1s : a.c2s, mode = first ? a.mode1 : a.mode2, cb = first ? c0 : c0 - a.c1;
        // the halo: [k8][pixel][8 channels], zero outside the image
        for (int i = tid; i < TC_PIX * 4; i += UN_THREADS) {
            const int pix = i >> 2, v = i & 3;
            const int yy = y0 - 1 + pix / TC_WP, xx = x0 - 1 + pix % TC_WP;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (yy >= 0 && yy < a.H && xx >= 0 && xx < a.W) val = load8(src, cs, mode, b, yy, xx, a.H, a.W, cb + 8 * v);
            *reinterpret_cast<uint4*>(As + ((size_t)v * TC_PIX + pix) * 16) = val;
        }
        // the weights: [tap][k8][n][8]
        for (int i = tid; i < 9 * N * 4; i += UN_THREADS) {
            const int v = i & 3, row = i >> 2, tap = row / N, n = row % N;
            const uint4 val = *reinterpret_cast<const uint4*>(a.w + ((size_t)tap * a.cout + n0 + n) * a.cin + c0 + 8 * v);
            *reinterpret_cast<uint4*>(Bs + (((size_t)tap * 4 + v) * N + n) * 16) = val;
        }
        // the generic-proxy stores, visible to the tensor cores' async proxy
        asm volatile("fence.proxy.async.shared::cta;");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll 1
            for (int tap = 0; tap < 9; tap++) {
                const int ky = tap / 3, kx = tap % 3;
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const uint64_t da = umma_desc(a_base + (uint32_t)((2 * j * TC_PIX + ky * TC_WP + kx) * 16), TC_PIX * 16, TC_WP * 16);
                    const uint64_t db = umma_desc(b_base + (uint32_t)(((tap * 4 + 2 * j) * N) * 16), N * 16, 8 * 16);
                    const uint32_t acc = (chunk > 0 || tap > 0 || j > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                        "l"(da), "l"(db), "r"(IDESC), "r"(acc));
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar)) : "memory");
        }
        // every thread: the chunk's MMAs are done (their shared-memory reads too) before the next staging
        uint32_t done = 0;
        for (unsigned it = 0; it < TC_SPIN_LIMIT && !done; it++)
            asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                         : "=r"(done)
                         : "r"(smem_u32(mbar)), "r"((uint32_t)(chunk & 1)));
        if (!done) {
            ok = false;
            break;
        }
    }
    if (!ok) {
        // the wait ran out: flag it, give the MMAs in flight a second bounded wait, free the TMEM, return
        if (tid == 0) atomicOr(status, 0x100);
        uint32_t done = 0;
        for (unsigned it = 0; it < TC_SPIN_LIMIT && !done; it++)
            asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                         : "=r"(done)
                         : "r"(smem_u32(mbar)), "r"((uint32_t)(chunk & 1)));
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;");
        // epilogue: pixel m = 32 warp + lane = (row m / 8, column m % 8); 8 channels per load
        const int m = 32 * warp + lane, y = y0 + m / TC_TW, x = x0 + m % TC_TW;
        const bool in = y < a.H && x < a.W;
        const size_t pix = ((size_t)b * a.H + y) * a.W + x;
#pragma unroll 1
        for (int c = 0; c < N; c += 8) {
            uint32_t r[8];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                         : "r"(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c));
            asm volatile("tcgen05.wait::ld.sync.aligned;");
            if (!in) continue;
            float v[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                v[q] = __uint_as_float(r[q]);
                if (a.bias) v[q] += a.bias[n0 + c + q];
                if (a.relu) v[q] = fmaxf(v[q], 0.f);
            }
            const int n = n0 + c;
            if (a.out) {
                uint4 o;
                __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
                for (int q = 0; q < 4; q++) h[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
                *reinterpret_cast<uint4*>(a.out + pix * a.cout + n) = o;
            }
            if (a.out_f32) {
                float4* o = reinterpret_cast<float4*>(a.out_f32 + pix * a.cout + n);
                o[0] = make_float4(v[0], v[1], v[2], v[3]);
                o[1] = make_float4(v[4], v[5], v[6], v[7]);
            }
            if (a.out_c0 && n == 0) a.out_c0[pix] = v[0];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(COLS));
}

// ------------------------------------------------------------ backward parts
// dZ = dY * (Y > 0) rounded to bf16 (the operand of the dX conv and dW)
__global__ void relu_grad_kernel(const float* __restrict__ dy, const __nv_bfloat16* __restrict__ y, __nv_bfloat16* __restrict__ dz,
                                 size_t n, int relu) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = relu && !(__bfloat162float(y[i]) > 0.f) ? 0.f : dy[i];
        dz[i] = __float2bfloat16_rn(v);
    }
}
// the output layer: only channel 0 carries a gradient
__global__ void out_grad_kernel(const float* __restrict__ dy0, __nv_bfloat16* __restrict__ dz, size_t npx, int c) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < npx * c; i += (size_t)gridDim.x * blockDim.x)
        dz[i] = __float2bfloat16_rn(i % c == 0 ? dy0[i / c] : 0.f);
}

// dX (at the layer's grid, cin channels) into the gradient of a source:
// SAME adds, UP sums the 4 children into the coarse pixel, POOL spreads 1/4.
__global__ void route_kernel(const float* __restrict__ dx, int cin, int coff, int cn, float* __restrict__ gsrc, int cs, int mode,
                             int B, int H, int W) {
    // one thread per (source pixel, channel)
    const int Hs = mode == SRC_SAME ? H : (mode == SRC_UP ? H / 2 : 2 * H), Ws = mode == SRC_SAME ? W : (mode == SRC_UP ? W / 2 : 2 * W);
    const size_t total = (size_t)B * Hs * Ws * cn;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % cn);
        const size_t p = i / cn;
        const int x = (int)(p % Ws), y = (int)((p / Ws) % Hs), b = (int)(p / ((size_t)Ws * Hs));
        float v;
        if (mode == SRC_SAME) {
            v = dx[(((size_t)b * H + y) * W + x) * cin + coff + c];
        } else if (mode == SRC_UP) {
            v = 0.f;
            for (int dy = 0; dy < 2; dy++)
                for (int dxx = 0; dxx < 2; dxx++) v += dx[(((size_t)b * H + 2 * y + dy) * W + 2 * x + dxx) * cin + coff + c];
        } else {
            v = 0.25f * dx[(((size_t)b * H + y / 2) * W + x / 2) * cin + coff + c];
        }
        gsrc[p * cs + c] += v;
    }
}

// dW[tap][co][ci] and db[co] on the CUDA cores: a CTA owns 32 couts x 32
// cins for a slice of the output tiles, keeps its 9 x 32 x 32 sums in
// registers (thread: one (co, ci) pair x ... ) and adds them once.
constexpr int DW_TILES_PER_CTA = 16;
__global__ void __launch_bounds__(256) conv_dw_kernel(const ConvArgs a, const __nv_bfloat16* __restrict__ dz, float* __restrict__ dw,
                                                      float* __restrict__ db) {
    __shared__ float xs[UN_HP * UN_WP][UN_CH + 1];
    __shared__ float zs[UN_TH * UN_TW][UN_CH + 1];
    const int co0 = blockIdx.y * 32, c0 = (blockIdx.z % (a.cin / UN_CH)) * UN_CH;
    const int tid = threadIdx.x;
    const int tiles_x = (a.W + UN_TW - 1) / UN_TW, tiles_y = (a.H + UN_TH - 1) / UN_TH;
    const int ntiles = tiles_x * tiles_y * a.B;
    // thread -> (co, 4 consecutive ci): 32 x 8 = 256 threads, 9 taps x 4 ci sums each
    const int co = tid >> 3, ci4 = (tid & 7) * 4;
    float s[9][4];
#pragma unroll
    for (int q = 0; q < 9; q++)
#pragma unroll
        for (int r = 0; r < 4; r++) s[q][r] = 0.f;
    float sb = 0.f;
    const bool first = c0 < a.c1;
    const __nv_bfloat16* src = first ? a.src1 : a.src2;
    const int cs = first ? a.c1s : a.c2s, mode = first ? a.mode1 : a.mode2, cb = first ? c0 : c0 - a.c1;
    const int t_lo = blockIdx.x * DW_TILES_PER_CTA, t_hi = min(ntiles, t_lo + DW_TILES_PER_CTA);
    for (int tile = t_lo; tile < t_hi; tile++) {
        const int b = tile / (tiles_x * tiles_y), tr = tile % (tiles_x * tiles_y);
        const int x0 = (tr % tiles_x) * UN_TW, y0 = (tr / tiles_x) * UN_TH;
        for (int i = tid; i < UN_HP * UN_WP * 4; i += 256) {
            const int pix = i >> 2, v = i & 3;
            const int yy = y0 - 1 + pix / UN_WP, xx = x0 - 1 + pix % UN_WP;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (yy >= 0 && yy < a.H && xx >= 0 && xx < a.W) val = load8(src, cs, mode, b, yy, xx, a.H, a.W, cb + 8 * v);
            const __nv_bfloat162* p = reinterpret_cast<const __nv_bfloat162*>(&val);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const float2 f = __bfloat1622float2(p[e]);
                xs[pix][8 * v + 2 * e] = f.x;
                xs[pix][8 * v + 2 * e + 1] = f.y;
            }
        }
        for (int i = tid; i < UN_TH * UN_TW * 32; i += 256) {
            const int pix = i >> 5, c = i & 31;
            const int yy = y0 + pix / UN_TW, xx = x0 + pix % UN_TW;
            float v = 0.f;
            if (yy < a.H && xx < a.W) v = __bfloat162float(dz[(((size_t)b * a.H + yy) * a.W + xx) * a.cout + co0 + c]);
            zs[pix][c] = v;
        }
        __syncthreads();
        for (int p = 0; p < UN_TH * UN_TW; p++) {
            const float z = zs[p][co];
            const int py = p / UN_TW, px = p % UN_TW;
            sb += z;
#pragma unroll
            for (int tap = 0; tap < 9; tap++) {
                const float* xr = &xs[(py + tap / 3) * UN_WP + px + tap % 3][ci4];
#pragma unroll
                for (int r = 0; r < 4; r++) s[tap][r] += z * xr[r];
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int tap = 0; tap < 9; tap++)
#pragma unroll
        for (int r = 0; r < 4; r++) atomicAdd(&dw[((size_t)tap * a.cout + co0 + co) * a.cin + c0 + ci4 + r], s[tap][r]);
    if (db && c0 == 0 && (tid & 7) == 0) atomicAdd(&db[co0 + co], sb);
}

// Adam on the FP32 masters, then the bf16 forward copy and the flipped,
// transposed copy the dX conv reads: wt[8 - tap][ci][co] = w[tap][co][ci].
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ gw, float* __restrict__ m, float* __restrict__ v, size_t n,
                            float lr, float b1, float b2, float c1, float c2, float eps, const unsigned char* __restrict__ mask) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (mask && !mask[i]) continue;
        const float gr = gw[i];
        const float mi = b1 * m[i] + (1.f - b1) * gr, vi = b2 * v[i] + (1.f - b2) * gr * gr;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}
__global__ void cast_weights_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, __nv_bfloat16* __restrict__ wt,
                                    int cout, int cin) {
    const size_t n = (size_t)9 * cout * cin;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int ci = (int)(i % cin), co = (int)((i / cin) % cout), tap = (int)(i / ((size_t)cin * cout));
        const __nv_bfloat16 v = __float2bfloat16_rn(w[i]);
        wb[i] = v;
        wt[((size_t)(8 - tap) * cin + ci) * cout + co] = v;
    }
}

// ------------------------------------------------------------ input / output
// The network's input from the depth grid's planes (dw x dh): 2x2 means
// (clamped at the edge) onto a grid padded to a multiple of 8, channels
// (guide, d / dmax, conf), the rest zero; d_in keeps d / dmax in f32.
__global__ void unet_input_kernel(const float* __restrict__ guide, const float* __restrict__ d, const float* __restrict__ conf, int dw,
                                  int dh, float inv_dmax, int H, int W, int b, __nv_bfloat16* __restrict__ in, float* __restrict__ d_in) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    float s[3] = {0.f, 0.f, 0.f};
    for (int dy = 0; dy < 2; dy++)
        for (int dx = 0; dx < 2; dx++) {
            const int sx = min(2 * x + dx, dw - 1), sy = min(2 * y + dy, dh - 1);
            const size_t k = (size_t)sy * dw + sx;
            s[0] += guide[k];
            s[1] += d[k] * inv_dmax;
            s[2] += conf[k];
        }
    const size_t p = ((size_t)b * H + y) * W + x;
    __nv_bfloat16* o = in + p * UN_CH;
    o[0] = __float2bfloat16_rn(0.25f * s[0]);
    o[1] = __float2bfloat16_rn(0.25f * s[1]);
    o[2] = __float2bfloat16_rn(fminf(0.25f * s[2], 4.f));
    for (int c = 3; c < UN_CH; c++) o[c] = __float2bfloat16_rn(0.f);
    d_in[p] = 0.25f * s[1];
}
// y = d_in + out0 on the network grid; bilinear back to the depth grid, times dmax
__global__ void unet_output_kernel(const float* __restrict__ d_in, const float* __restrict__ out0, int H, int W, int b, int dw, int dh,
                                   float dmax, float* __restrict__ x0) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= dw || y >= dh) return;
    const float fx = fminf(fmaxf((x + 0.5f) * 0.5f - 0.5f, 0.f), (float)(W - 1));
    const float fy = fminf(fmaxf((y + 0.5f) * 0.5f - 0.5f, 0.f), (float)(H - 1));
    const int xa = (int)fx, ya = (int)fy, xb = min(xa + 1, W - 1), yb = min(ya + 1, H - 1);
    const float tx = fx - xa, ty = fy - ya;
    const size_t base = (size_t)b * H * W;
    auto Y = [&](int yy, int xx) { const size_t k = base + (size_t)yy * W + xx; return d_in[k] + out0[k]; };
    const float v = (1.f - ty) * ((1.f - tx) * Y(ya, xa) + tx * Y(ya, xb)) + ty * ((1.f - tx) * Y(yb, xa) + tx * Y(yb, xb));
    x0[(size_t)y * dw + x] = fminf(fmaxf(v, 0.f), 1.f) * dmax;
}
// MSE on the network grid: loss partials and dL/dout0 = 2 (d_in + out0 - t) / n
__global__ void mse_kernel(const float* __restrict__ d_in, const float* __restrict__ out0, const float* __restrict__ tgt, size_t n,
                           float* __restrict__ dout0, double* __restrict__ loss) {
    double s = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float e = d_in[i] + out0[i] - tgt[i];
        dout0[i] = 2.f * e / (float)n;
        s += (double)e * e;
    }
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0] / (double)n);
}

// ------------------------------------------------------------------- network
struct Layer {
    int src1, mode1, c1, src2, mode2, c2, cout, level, relu;
    size_t woff, boff;  // offsets in the parameter arrays
};
// tensor t (0 = input, i + 1 = output of layer i): level, channels
static const int N_LAYERS = 15;
static std::vector<Layer> unet_layers() {
    std::vector<Layer> L;
    auto add = [&](int s1, int m1, int c1, int s2, int m2, int c2, int co, int lv, int relu) {
        L.push_back(Layer{s1, m1, c1, s2, m2, c2, co, lv, relu, 0, 0});
    };
    add(0, SRC_SAME, 32, -1, 0, 0, 32, 0, 1);      // 0  E0a  (input: 3 channels of 32)
    add(1, SRC_SAME, 32, -1, 0, 0, 32, 0, 1);      // 1  E0b  skip0
    add(2, SRC_POOL, 32, -1, 0, 0, 64, 1, 1);      // 2  E1a
    add(3, SRC_SAME, 64, -1, 0, 0, 64, 1, 1);      // 3  E1b  skip1
    add(4, SRC_POOL, 64, -1, 0, 0, 128, 2, 1);     // 4  E2a
    add(5, SRC_SAME, 128, -1, 0, 0, 128, 2, 1);    // 5  E2b  skip2
    add(6, SRC_POOL, 128, -1, 0, 0, 256, 3, 1);    // 6  B3a
    add(7, SRC_SAME, 256, -1, 0, 0, 256, 3, 1);    // 7  B3b
    add(8, SRC_UP, 256, 6, SRC_SAME, 128, 128, 2, 1);  // 8  D2a = up(B3b) ++ skip2
    add(9, SRC_SAME, 128, -1, 0, 0, 128, 2, 1);    // 9  D2b
    add(10, SRC_UP, 128, 4, SRC_SAME, 64, 64, 1, 1);   // 10 D1a = up(D2b) ++ skip1
    add(11, SRC_SAME, 64, -1, 0, 0, 64, 1, 1);     // 11 D1b
    add(12, SRC_UP, 64, 2, SRC_SAME, 32, 32, 0, 1);    // 12 D0a = up(D1b) ++ skip0
    add(13, SRC_SAME, 32, -1, 0, 0, 32, 0, 1);     // 13 D0b
    add(14, SRC_SAME, 32, -1, 0, 0, 32, 0, 0);     // 14 OUT  (channel 0 only; linear)
    size_t wo = 0, bo = 0;
    for (auto& l : L) {
        l.woff = wo;
        l.boff = bo;
        wo += (size_t)9 * l.cout * (l.c1 + l.c2);
        bo += l.cout;
    }
    return L;
}

}  // namespace lsb

using namespace lsb;

struct lsb_unet {
    int device = 0;
    cudaStream_t s = nullptr;
    std::vector<Layer> layers;
    size_t nw = 0, nb = 0;  // parameter counts
    // FP32 masters, grads, Adam moments (weights then biases, one array each)
    float *w = nullptr, *gw = nullptr, *mw = nullptr, *vw = nullptr;
    float *b = nullptr, *gb = nullptr, *mb = nullptr, *vb = nullptr;
    unsigned char* wmask = nullptr;  // trainable weights (the output layer keeps channels 1.. at zero)
    unsigned char* bmask = nullptr;
    __nv_bfloat16 *wb = nullptr, *wt = nullptr;
    int step = 0;
    // activations for the current shape
    int B = 0, H = 0, W = 0;
    std::vector<__nv_bfloat16*> act;  // bf16 [B][h_l][w_l][c]
    std::vector<float*> grad;         // f32, same shapes
    float *out0 = nullptr, *dout0 = nullptr, *d_in = nullptr, *dxbuf = nullptr, *x0 = nullptr;
    __nv_bfloat16* dz = nullptr;
    double* loss = nullptr;
    double* loss_host = nullptr;
    std::vector<void*> shape_allocs;
    int* status = nullptr;  // device error word of the tcgen05 convolution (a bounded wait ran out)
    bool tc = true;         // the 3x3 convolutions on tcgen05 (false: mma.sync, for comparison)
    cudaEvent_t fev[2] = {nullptr, nullptr};  // around the last forward pass's layers on s
    float fwd_ms = 0.f;
};

static char* un_err(const std::string& s) {
    char* p = (char*)malloc(s.size() + 1);
    memcpy(p, s.c_str(), s.size() + 1);
    return p;
}
#define UTRY(x)                                                                                 \
    do {                                                                                        \
        cudaError_t _e = (x);                                                                   \
        if (_e != cudaSuccess) return un_err(std::string("unet: ") + cudaGetErrorString(_e)); \
    } while (0)

static int ugrid(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 8); }

static size_t act_channels(const lsb_unet* u, int t) { return t == 0 ? 32 : u->layers[t - 1].cout; }
static int act_level(const lsb_unet* u, int t) { return t == 0 ? 0 : u->layers[t - 1].level; }

static void free_shape(lsb_unet* u) {
    for (void* p : u->shape_allocs) cudaFree(p);
    u->shape_allocs.clear();
    u->act.clear();
    u->grad.clear();
    u->B = u->H = u->W = 0;
}

static cudaError_t ensure_shape(lsb_unet* u, int B, int H, int W, bool train) {
    if (u->B == B && u->H == H && u->W == W && (!train || !u->grad.empty())) return cudaSuccess;
    free_shape(u);
    auto get = [&](size_t bytes, void** p) {
        cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
        if (e == cudaSuccess) u->shape_allocs.push_back(*p);
        return e;
    };
    size_t maxc = 0;
    for (int t = 0; t <= N_LAYERS; t++) {
        const int lv = act_level(u, t);
        const size_t px = (size_t)B * (H >> lv) * (W >> lv), c = act_channels(u, t);
        void* p;
        cudaError_t e = get(px * c * sizeof(__nv_bfloat16), &p);
        if (e != cudaSuccess) return e;
        u->act.push_back((__nv_bfloat16*)p);
        if (train) {
            e = get(px * c * sizeof(float), &p);
            if (e != cudaSuccess) return e;
            u->grad.push_back((float*)p);
        }
        maxc = std::max(maxc, px * c);
    }
    for (auto& l : u->layers) maxc = std::max(maxc, (size_t)B * (H >> l.level) * (W >> l.level) * (l.c1 + l.c2));
    const size_t px0 = (size_t)B * H * W;
    void* p;
    cudaError_t e;
    if ((e = get(px0 * sizeof(float), &p)) != cudaSuccess) return e;
    u->out0 = (float*)p;
    if ((e = get(px0 * sizeof(float), &p)) != cudaSuccess) return e;
    u->d_in = (float*)p;
    if (train) {
        if ((e = get(px0 * sizeof(float), &p)) != cudaSuccess) return e;
        u->dout0 = (float*)p;
        if ((e = get(maxc * sizeof(float), &p)) != cudaSuccess) return e;
        u->dxbuf = (float*)p;
        if ((e = get(maxc * sizeof(__nv_bfloat16), &p)) != cudaSuccess) return e;
        u->dz = (__nv_bfloat16*)p;
    }
    u->B = B;
    u->H = H;
    u->W = W;
    return cudaSuccess;
}

template <int N>
static cudaError_t conv_tc_launch(const ConvArgs& a, int* status, cudaStream_t s) {
    const size_t smem = tc_smem_bytes(N);
    cudaError_t e = cudaFuncSetAttribute(conv3x3_tc_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid(((a.W + TC_TW - 1) / TC_TW) * ((a.H + TC_TH - 1) / TC_TH), a.cout / N, a.B);
    lsb_launched(), conv3x3_tc_kernel<N><<<grid, UN_THREADS, smem, s>>>(a, status);
    return cudaGetLastError();
}

static cudaError_t conv_launch(const ConvArgs& a, cudaStream_t s, int* status = nullptr, bool tc = false) {
    // tcgen05: every layer's cin is a multiple of 32 and its cout 32, 64, 128 or 256 (one CTA takes them all)
    if (tc && status && a.cin % UN_CH == 0) {
        switch (a.cout) {
            case 32: return conv_tc_launch<32>(a, status, s);
            case 64: return conv_tc_launch<64>(a, status, s);
            case 128: return conv_tc_launch<128>(a, status, s);
            case 256: return conv_tc_launch<256>(a, status, s);
            default: break;
        }
    }
    const int NT = a.cout % 64 == 0 ? 64 : 32;
    const size_t smem = (size_t)(UN_HP * UN_WP + 9 * NT) * UN_LD * sizeof(__nv_bfloat16);
    const dim3 grid(((a.W + UN_TW - 1) / UN_TW) * ((a.H + UN_TH - 1) / UN_TH), a.cout / NT, a.B);
    if (NT == 64) {
        cudaFuncSetAttribute(conv3x3_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        lsb_launched(), conv3x3_kernel<64><<<grid, UN_THREADS, smem, s>>>(a);
    } else {
        cudaFuncSetAttribute(conv3x3_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        lsb_launched(), conv3x3_kernel<32><<<grid, UN_THREADS, smem, s>>>(a);
    }
    return cudaGetLastError();
}

static ConvArgs layer_args(const lsb_unet* u, int i) {
    const Layer& l = u->layers[i];
    ConvArgs a{};
    a.src1 = u->act[l.src1];
    a.c1 = l.c1;
    a.c1s = (int)act_channels(u, l.src1);
    a.mode1 = l.mode1;
    a.src2 = l.src2 >= 0 ? u->act[l.src2] : nullptr;
    a.c2s = l.src2 >= 0 ? (int)act_channels(u, l.src2) : 0;
    a.mode2 = l.mode2;
    a.cin = l.c1 + l.c2;
    a.cout = l.cout;
    a.w = u->wb + l.woff;
    a.bias = u->b + l.boff;
    a.relu = l.relu;
    a.B = u->B;
    a.H = u->H >> l.level;
    a.W = u->W >> l.level;
    return a;
}

static cudaError_t unet_forward(lsb_unet* u) {
    for (int i = 0; i < N_LAYERS; i++) {
        ConvArgs a = layer_args(u, i);
        const bool last = i == N_LAYERS - 1;
        a.out = last ? nullptr : u->act[i + 1];
        a.out_c0 = last ? u->out0 : nullptr;
        if (last) a.out = u->act[i + 1];
        cudaError_t e = conv_launch(a, u->s, u->status, u->tc);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

static cudaError_t cast_all(lsb_unet* u) {
    for (auto& l : u->layers) {
        lsb_launched(), cast_weights_kernel<<<ugrid((size_t)9 * l.cout * (l.c1 + l.c2)), 256, 0, u->s>>>(u->w + l.woff, u->wb + l.woff,
                                                                                                      u->wt + l.woff, l.cout, l.c1 + l.c2);
    }
    return cudaGetLastError();
}

extern "C" char* lsb_unet_create(int32_t device, uint64_t seed, lsb_unet** out) {
    *out = nullptr;
    lsb_unet* u = new lsb_unet();
    u->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete u;
        return un_err(std::string("unet: ") + cudaGetErrorString(e));
    }
    u->layers = unet_layers();
    for (auto& l : u->layers) {
        u->nw = l.woff + (size_t)9 * l.cout * (l.c1 + l.c2);
        u->nb = l.boff + l.cout;
    }
    std::vector<float> w(u->nw, 0.f), b(u->nb, 0.f);
    std::vector<unsigned char> wm(u->nw, 1), bm(u->nb, 1);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    for (size_t li = 0; li < u->layers.size(); li++) {
        const Layer& l = u->layers[li];
        const int cin = l.c1 + l.c2;
        const int fan_in = 9 * (li == 0 ? 3 : cin);
        const float sd = li + 1 == u->layers.size() ? 1e-3f : std::sqrt(2.f / fan_in);
        for (int tap = 0; tap < 9; tap++)
            for (int co = 0; co < l.cout; co++)
                for (int ci = 0; ci < cin; ci++) {
                    const size_t k = l.woff + ((size_t)tap * l.cout + co) * cin + ci;
                    const bool live = (li != 0 || ci < 3) && (li + 1 != u->layers.size() || co == 0);
                    w[k] = live ? sd * nd(rng) : 0.f;
                    wm[k] = live;
                }
        for (int co = 0; co < l.cout; co++) bm[l.boff + co] = li + 1 != u->layers.size() || co == 0;
    }
    auto alloc = [&](void** p, size_t bytes) -> bool {
        if (cudaMalloc(p, bytes) != cudaSuccess) return false;
        return cudaMemset(*p, 0, bytes) == cudaSuccess;
    };
    bool ok = alloc((void**)&u->w, u->nw * 4) && alloc((void**)&u->gw, u->nw * 4) && alloc((void**)&u->mw, u->nw * 4) &&
              alloc((void**)&u->vw, u->nw * 4) && alloc((void**)&u->b, u->nb * 4) && alloc((void**)&u->gb, u->nb * 4) &&
              alloc((void**)&u->mb, u->nb * 4) && alloc((void**)&u->vb, u->nb * 4) && alloc((void**)&u->wmask, u->nw) &&
              alloc((void**)&u->bmask, u->nb) && alloc((void**)&u->wb, u->nw * 2) && alloc((void**)&u->wt, u->nw * 2) &&
              alloc((void**)&u->loss, 8) && alloc((void**)&u->status, 4) &&
              cudaHostAlloc((void**)&u->loss_host, 8, cudaHostAllocDefault) == cudaSuccess &&
              cudaStreamCreateWithFlags(&u->s, cudaStreamNonBlocking) == cudaSuccess;
    if (!ok) {
        lsb_unet_destroy(u);
        return un_err("unet: device allocation failed");
    }
    cudaMemcpy(u->w, w.data(), u->nw * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(u->b, b.data(), u->nb * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(u->wmask, wm.data(), u->nw, cudaMemcpyHostToDevice);
    cudaMemcpy(u->bmask, bm.data(), u->nb, cudaMemcpyHostToDevice);
    e = cast_all(u);
    if (e == cudaSuccess) e = cudaStreamSynchronize(u->s);
    if (e != cudaSuccess) {
        lsb_unet_destroy(u);
        return un_err(std::string("unet: ") + cudaGetErrorString(e));
    }
    *out = u;
    return nullptr;
}

extern "C" void lsb_unet_destroy(lsb_unet* u) {
    if (!u) return;
    if (u->s) cudaStreamSynchronize(u->s);
    free_shape(u);
    for (void* p : {(void*)u->w, (void*)u->gw, (void*)u->mw, (void*)u->vw, (void*)u->b, (void*)u->gb, (void*)u->mb, (void*)u->vb,
                    (void*)u->wmask, (void*)u->bmask, (void*)u->wb, (void*)u->wt, (void*)u->loss, (void*)u->status})
        if (p) cudaFree(p);
    if (u->loss_host) cudaFreeHost(u->loss_host);
    for (cudaEvent_t v : u->fev)
        if (v) cudaEventDestroy(v);
    if (u->s) cudaStreamDestroy(u->s);
    delete u;
}

// The device error word: a tcgen05 convolution whose bounded wait ran out (its output is not written).
static char* conv_status(lsb_unet* u) {
    int st = 0;
    UTRY(cudaMemcpy(&st, u->status, sizeof st, cudaMemcpyDeviceToHost));
    if (st) {
        cudaMemset(u->status, 0, sizeof st);
        return un_err("unet: a tensor-core convolution's wait for its MMAs ran out");
    }
    return nullptr;
}

extern "C" char* lsb_unet_set_conv(lsb_unet* u, uint32_t path) {
    if (!u) return un_err("unet: null network");
    if (path > 1) return un_err("unet: conv path must be 0 (tcgen05) or 1 (mma.sync)");
    u->tc = path == 0;
    return nullptr;
}

extern "C" void lsb_unet_sizes(const lsb_unet* u, uint64_t* n_weights, uint64_t* n_biases) {
    *n_weights = u->nw;
    *n_biases = u->nb;
}

extern "C" char* lsb_unet_get_params(lsb_unet* u, float* w, float* b, float* gw, float* gb) {
    UTRY(cudaStreamSynchronize(u->s));
    if (w) UTRY(cudaMemcpy(w, u->w, u->nw * 4, cudaMemcpyDeviceToHost));
    if (b) UTRY(cudaMemcpy(b, u->b, u->nb * 4, cudaMemcpyDeviceToHost));
    if (gw) UTRY(cudaMemcpy(gw, u->gw, u->nw * 4, cudaMemcpyDeviceToHost));
    if (gb) UTRY(cudaMemcpy(gb, u->gb, u->nb * 4, cudaMemcpyDeviceToHost));
    return nullptr;
}

extern "C" char* lsb_unet_set_params(lsb_unet* u, const float* w, const float* b) {
    UTRY(cudaStreamSynchronize(u->s));
    UTRY(cudaMemcpy(u->w, w, u->nw * 4, cudaMemcpyHostToDevice));
    UTRY(cudaMemcpy(u->b, b, u->nb * 4, cudaMemcpyHostToDevice));
    UTRY(cast_all(u));
    UTRY(cudaStreamSynchronize(u->s));
    return nullptr;
}

// in: device [B][H][W][32] bf16 (lsb_unet_prepare's layout), d_in: device [B][H][W] f32
static char* stage_batch(lsb_unet* u, const void* in, const float* d_in, int B, int H, int W, bool train) {
    if (H % 8 || W % 8 || H < 8 || W < 8) return un_err("unet: the grid must be a multiple of 8 on both sides");
    UTRY(ensure_shape(u, B, H, W, train));
    UTRY(cudaMemcpyAsync(u->act[0], in, (size_t)B * H * W * UN_CH * 2, cudaMemcpyDeviceToDevice, u->s));
    UTRY(cudaMemcpyAsync(u->d_in, d_in, (size_t)B * H * W * 4, cudaMemcpyDeviceToDevice, u->s));
    return nullptr;
}

extern "C" char* lsb_unet_forward(lsb_unet* u, const void* in_dev, const float* d_in_dev, uint32_t B, uint32_t H, uint32_t W,
                                  float* out0_dev) {
    if (char* er = stage_batch(u, in_dev, d_in_dev, (int)B, (int)H, (int)W, false)) return er;
    for (cudaEvent_t& v : u->fev)
        if (!v) UTRY(cudaEventCreate(&v));
    UTRY(cudaEventRecord(u->fev[0], u->s));
    UTRY(unet_forward(u));
    UTRY(cudaEventRecord(u->fev[1], u->s));
    if (out0_dev) UTRY(cudaMemcpyAsync(out0_dev, u->out0, (size_t)B * H * W * 4, cudaMemcpyDeviceToDevice, u->s));
    UTRY(cudaStreamSynchronize(u->s));
    UTRY(cudaEventElapsedTime(&u->fwd_ms, u->fev[0], u->fev[1]));
    return conv_status(u);
}

extern "C" char* lsb_unet_forward_ms(lsb_unet* u, float* ms) {
    if (!u || !ms) return un_err("unet: null argument");
    *ms = u->fwd_ms;
    return nullptr;
}

static cudaError_t unet_backward(lsb_unet* u) {
    const size_t px0 = (size_t)u->B * u->H * u->W;
    cudaMemsetAsync(u->gw, 0, u->nw * 4, u->s);
    cudaMemsetAsync(u->gb, 0, u->nb * 4, u->s);
    for (int t = 0; t <= N_LAYERS; t++) {
        const int lv = act_level(u, t);
        cudaMemsetAsync(u->grad[t], 0, (size_t)u->B * (u->H >> lv) * (u->W >> lv) * act_channels(u, t) * 4, u->s);
    }
    for (int i = N_LAYERS - 1; i >= 0; i--) {
        const Layer& l = u->layers[i];
        ConvArgs a = layer_args(u, i);
        const size_t npx = (size_t)a.B * a.H * a.W;
        if (i == N_LAYERS - 1)
            lsb_launched(), out_grad_kernel<<<ugrid(npx * l.cout), 256, 0, u->s>>>(u->dout0, u->dz, npx, l.cout);
        else
            lsb_launched(), relu_grad_kernel<<<ugrid(npx * l.cout), 256, 0, u->s>>>(u->grad[i + 1], u->act[i + 1], u->dz, npx * l.cout, l.relu);
        const int cin = l.c1 + l.c2;
        const int ntiles = ((a.W + UN_TW - 1) / UN_TW) * ((a.H + UN_TH - 1) / UN_TH) * a.B;
        const dim3 gdw((ntiles + DW_TILES_PER_CTA - 1) / DW_TILES_PER_CTA, l.cout / 32, cin / UN_CH);
        lsb_launched(), conv_dw_kernel<<<gdw, 256, 0, u->s>>>(a, u->dz, u->gw + l.woff, u->gb + l.boff);
        if (i == 0) continue;  // no gradient for the input
        ConvArgs d{};
        d.src1 = u->dz;
        d.c1 = l.cout;
        d.c1s = l.cout;
        d.mode1 = SRC_SAME;
        d.cin = l.cout;
        d.cout = cin;
        d.w = u->wt + l.woff;
        d.out_f32 = u->dxbuf;
        d.B = a.B;
        d.H = a.H;
        d.W = a.W;
        cudaError_t e = conv_launch(d, u->s, u->status, u->tc);
        if (e != cudaSuccess) return e;
        const size_t s1px = (size_t)a.B * (u->H >> act_level(u, l.src1)) * (u->W >> act_level(u, l.src1));
        lsb_launched(), route_kernel<<<ugrid(s1px * l.c1), 256, 0, u->s>>>(u->dxbuf, cin, 0, l.c1, u->grad[l.src1],
                                                                           (int)act_channels(u, l.src1), l.mode1, a.B, a.H, a.W);
        if (l.src2 >= 0) {
            const size_t s2px = (size_t)a.B * (u->H >> act_level(u, l.src2)) * (u->W >> act_level(u, l.src2));
            lsb_launched(), route_kernel<<<ugrid(s2px * l.c2), 256, 0, u->s>>>(u->dxbuf, cin, l.c1, l.c2, u->grad[l.src2],
                                                                               (int)act_channels(u, l.src2), l.mode2, a.B, a.H, a.W);
        }
    }
    (void)px0;
    return cudaGetLastError();
}

// One step on a batch: forward, MSE against target (d / dmax on the network
// grid), backward; Adam when lr > 0. loss_out gets the batch's MSE.
extern "C" char* lsb_unet_train_step(lsb_unet* u, const void* in_dev, const float* d_in_dev, const float* target_dev, uint32_t B,
                                     uint32_t H, uint32_t W, float lr, double* loss_out) {
    if (char* er = stage_batch(u, in_dev, d_in_dev, (int)B, (int)H, (int)W, true)) return er;
    UTRY(unet_forward(u));
    const size_t n = (size_t)B * H * W;
    UTRY(cudaMemsetAsync(u->loss, 0, 8, u->s));
    lsb_launched(), mse_kernel<<<ugrid(n), 256, 0, u->s>>>(u->d_in, u->out0, target_dev, n, u->dout0, u->loss);
    UTRY(unet_backward(u));
    if (lr > 0.f) {
        u->step++;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)u->step), c2 = 1.f - std::pow(b2, (float)u->step);
        lsb_launched(), adam_kernel<<<ugrid(u->nw), 256, 0, u->s>>>(u->w, u->gw, u->mw, u->vw, u->nw, lr, b1, b2, c1, c2, 1e-8f, u->wmask);
        lsb_launched(), adam_kernel<<<ugrid(u->nb), 256, 0, u->s>>>(u->b, u->gb, u->mb, u->vb, u->nb, lr, b1, b2, c1, c2, 1e-8f, u->bmask);
        UTRY(cast_all(u));
    }
    UTRY(cudaMemcpyAsync(u->loss_host, u->loss, 8, cudaMemcpyDeviceToHost, u->s));
    UTRY(cudaStreamSynchronize(u->s));
    if (loss_out) *loss_out = *u->loss_host;
    return conv_status(u);
}

// The network input of one depth grid (device planes dw x dh): in [H][W][32]
// bf16 and d_in [H][W] f32 at batch index b, H = round_up(ceil(dh/2), 8), W likewise.
extern "C" void lsb_unet_grid(uint32_t dw, uint32_t dh, uint32_t* H, uint32_t* W) {
    *W = ((dw + 1) / 2 + 7) / 8 * 8;
    *H = ((dh + 1) / 2 + 7) / 8 * 8;
}
extern "C" char* lsb_unet_prepare(const float* guide, const float* d, const float* conf, uint32_t dw, uint32_t dh, float dmax,
                                  void* in_dev, float* d_in_dev, uint32_t b, void* stream) {
    uint32_t H, W;
    lsb_unet_grid(dw, dh, &H, &W);
    const dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
    lsb_launched(), unet_input_kernel<<<grd, blk, 0, (cudaStream_t)stream>>>(guide, d, conf, (int)dw, (int)dh, 1.f / std::max(dmax, 1e-6f),
                                                                             (int)H, (int)W, (int)b, (__nv_bfloat16*)in_dev, d_in_dev);
    UTRY(cudaGetLastError());
    return nullptr;
}

namespace lsb {
// The warm start for a depth grid: prepare, forward, back to the grid.
cudaError_t unet_warm_start(lsb_unet* u, const float* guide, const float* d, const float* conf, int dw, int dh, float dmax, float* x0,
                            cudaStream_t st) {
    uint32_t H, W;
    lsb_unet_grid((uint32_t)dw, (uint32_t)dh, &H, &W);
    cudaError_t e = ensure_shape(u, 1, (int)H, (int)W, false);
    if (e != cudaSuccess) return e;
    // the network runs on the caller's stream
    cudaStream_t keep = u->s;
    u->s = st;
    const dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
    lsb_launched(), unet_input_kernel<<<grd, blk, 0, st>>>(guide, d, conf, dw, dh, 1.f / std::max(dmax, 1e-6f), (int)H, (int)W, 0,
                                                           u->act[0], u->d_in);
    e = unet_forward(u);
    if (e == cudaSuccess) {
        const dim3 g2((dw + 31) / 32, (dh + 7) / 8);
        lsb_launched(), unet_output_kernel<<<g2, blk, 0, st>>>(u->d_in, u->out0, (int)H, (int)W, 0, dw, dh, dmax, x0);
        e = cudaGetLastError();
    }
    u->s = keep;
    return e;
}
}  // namespace lsb
