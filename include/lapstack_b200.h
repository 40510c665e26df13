/* lapstack-b200: the stacking-engine hot path of ragtux/LAPSTACK
 * (crates/lapstack-core) as a B200-native CUDA library behind a C ABI.
 *
 * Conventions follow the reference's one C ABI, crates/lapstack-raw/src/
 * ffi.rs:66-152: an ABI-version function, plain #[repr(C)]-style structs,
 * functions that return NULL on success or a heap error string (free it
 * with lsb_free_str), explicit free functions, no unwinding across the
 * boundary. A handle is used from one thread at a time; an engine owns one
 * CUDA stream and every stack made from it runs on that stream.
 *
 * What each entry point replaces in the reference (crates/lapstack-core/src):
 *   lsb_engine_create      gpu.rs:308 `available` + the NVRTC/context set-up of
 *                          gpu.rs:312-324 (GpuFuser::new, GpuFrames::new)
 *   lsb_stack_begin        stack.rs:740 `fuse_range` creating the fuser
 *                          (AnyFuser, stack.rs:123-201) and stack.rs:481
 *                          AlignedFrames::open for one stack
 *   lsb_stack_push_u16     stack.rs:785-821 one frame of the fold loop:
 *                          FrameSource::get_gpu (stack.rs:623) + GpuFrames::
 *                          process (gpu.rs:751) + GpuFuser::push_device
 *                          (gpu.rs:451), from the decoded 16-bit frame
 *   lsb_stack_push_f32     AnyFuser::push(&Img3) (stack.rs:152, gpu.rs:435)
 *   lsb_stack_shares       AnyFuser::shares (stack.rs:167, gpu.rs:505)
 *   lsb_stack_finish       AnyFuser::finish (stack.rs:178, gpu.rs:517) +
 *                          fuse_and_depth (stack.rs:833) with
 *                          gpu::depth_from_slices (gpu.rs:1327) + the
 *                          common-area crop rectangle (align.rs:344)
 *   lsb_depth_from_slices  gpu::depth_from_slices (gpu.rs:1327)
 *   lsb_wls_solve          depth::wls_solve (depth.rs:1081) / DWls (gpu.rs:1154)
 *   lsb_align_pair         align::multiscale_align (align.rs:896) /
 *                          GpuFrames::search (gpu.rs:692)
 *   lsb_warp_cost          align::warp_cost (align.rs:581) / the warp_cost
 *                          kernel (gpu.rs:148)
 */
#ifndef LAPSTACK_B200_H
#define LAPSTACK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LSB_ABI_VERSION 1u

/* lsb_config.flags: fold level 0 with the REDUCE and select kernels on every tile instead of the
   fused level-0 kernel on the interior tiles (the same results; for cross-checks and timing) */
#define LSB_FLAG_TWO_KERNEL_FOLD0 1
/* lsb_config.flags: with frames already in device memory, fold an aligned stack chunk by chunk beside
   its registration chain instead of after it (the same results; pushed frames always fold beside it) */
#define LSB_FLAG_FOLD_BESIDE_CHAIN 2
/* lsb_config.flags: aggregate the focus slices with direct window sums of 2R+1 taps instead of moving
   sums at radii 3 and 8 (the same results whenever the f64 sums are exact; for cross-checks and timing) */
#define LSB_FLAG_DIRECT_WINDOW_SUMS 4

typedef struct lsb_engine lsb_engine;
typedef struct lsb_stack lsb_stack;

typedef void (*lsb_log_fn)(const char* line, void* user);

typedef struct {
    int32_t device;        /* CUDA device ordinal */
    int32_t storage;       /* Gaussian levels >= 1 and focus slices: 0 FP32 (bit-exact with the reference
                              FP32 path); 1 16-bit: UNORM16 levels, FP16 slices; 2 FP16 levels and slices */
    int32_t grid_limit;    /* CTAs of the persistent kernels and of the device registration search;
                              0 = 2 x the SM count */
    int32_t flags;         /* LSB_FLAG_* bits; 0 for the defaults */
    lsb_log_fn log;        /* optional progress lines (stack.rs:1014 `log`) */
    void* user;
} lsb_config;

/* fuse.rs:70-107 FuseParams */
typedef struct {
    uint32_t levels;        /* band-pass levels; 0 = auto (residual short side >= 32) */
    uint32_t energy_radius; /* 0..2 (1 = 3x3 binomial) */
    uint32_t top_rule;      /* 0 dev-entropy, 1 deviation, 2 average */
    uint32_t top_radius;    /* 0..4 */
    uint32_t entropy_bins;
    uint32_t use_chroma;
    uint32_t depth_level;
    float halo;             /* halo control hardness; 0 = off */
} lsb_fuse_params;

/* align.rs:52-70 AlignParams (enabled = 0: stack.rs's no-align path) */
typedef struct {
    uint32_t enabled;
    uint32_t shift, scale, rotation;
    uint32_t model;   /* 0 similarity, 1 affine, 2 projective */
    uint32_t coarsen; /* skip the N finest registration levels */
    uint32_t interp;  /* align.rs Interp id: 0 nearest .. 3 spline4x4 .. 5 lanczos3 */
    uint32_t host_search; /* 0: each frame's whole Nelder-Mead search in one cooperative launch;
                             1: the host drives it, one launch and read-back per simplex step */
} lsb_align_params;

/* depth.rs:69-109 DepthParams (enabled = 0: report the fuse winner map) */
typedef struct {
    uint32_t enabled;
    uint32_t scale;     /* working grid 1/2^scale */
    uint32_t focus;     /* 0 ring difference filter, 1 sum-modified Laplacian */
    uint32_t r_in, r_out, sml_step;
    uint32_t agg_radius;
    float agg_eps;
    float lambda, sigma_c;
    uint32_t cg_iters;
    uint32_t median;
    uint32_t upsample;  /* 0 bilinear, 1 guided */
    uint32_t up_radius;
    float up_eps;
    float gate, robust;
    uint32_t edge_mode; /* 0 exp(-|dI|/sigma_c) (reference); 1 exp(-dI^2/(2 sigma_c^2)) */
    uint32_t vcycle_mode; /* 0 FP32 V-cycle (reference); 1 BF16 smoother + restriction */
} lsb_depth_params;

/* Results of lsb_stack_finish; buffers owned by the library until lsb_result_free. */
typedef struct {
    uint32_t w, h, n_frames, levels, dw, dh;
    uint16_t* image_u16; /* w*h*3 interleaved, io.rs:287 quantisation */
    float* image_f32;    /* 3*w*h planar, clamped to [0,1] */
    float* winner;       /* w*h, fuse winner map at depth_level, upsampled (fuse.rs:336) */
    float* depth;        /* w*h fractional frame index, or NULL without the depth pass */
    float* conf;         /* w*h */
    float* floor_cells;  /* dw*dh per-cell noise floor (depth.rs:151 DepthMap::floor) */
    double* sims;        /* n*8 align.rs:200 Sim vectors */
    float* gains;        /* n*3 */
    float* shares;       /* n, fuse.rs:315 winner_shares */
    uint32_t crop[4];    /* x, y, w, h of the common area (align.rs:344) */
    float floor_value, p90, wls_rel;
    uint32_t wls_iters, wls_iters_first, align_evals;
    double wls_rel64;
    double ms[12];       /* device ms per stage: align, gains, fold, residual+collapse, focus agg, wls, upsample,
                            total, fold level 0, then its two parts: [9] the select kernel (with the fused
                            level-0 kernel: the REDUCE and select of the border tiles after it) and [10] the
                            REDUCE kernel (or the fused kernel), then the WLS solves (warm start included) */
} lsb_result;

/* wav.rs:52-80 WavParams: the weighted average's settings (defaults 2, 3, 0.5, 1). */
typedef struct {
    float power;     /* the contrast above the floor raised to this */
    uint32_t smooth; /* box radius of the contrast, then of the weights, on the working grid (0: none) */
    float gate;      /* a contrast counts above (1 + gate) x the cell's noise floor */
    uint32_t edge;   /* 1: the weights smoothed by the guided filter with the fused luma as guide */
} lsb_wav_params;

/* dust.rs:85 Spot: a window (x, y, w, h) of the frame, its mask (w*h bytes, nonzero = dust) and, for
   flat mode, its attenuation (w*h floats, >= 1; may be NULL in fill mode). */
typedef struct {
    uint32_t x, y, w, h;
    const uint8_t* mask;
    const float* gain;
} lsb_dust_spot;

/* dust.rs:105 DustMap: the frame size it was made at, dust.rs:42 DustMode (0 fill: pull-push from the
   surroundings; 1 flat: times the attenuation) and the spots, taken out in order. */
typedef struct {
    uint32_t w, h;
    uint32_t mode;
    uint32_t n_spots;
    const lsb_dust_spot* spots;
} lsb_dust_map;

/* What every decoded frame goes through before it is registered and folded (stack.rs:52-58 Params::dust,
   rotate, reduce; lapstack-web lib.rs:766-784 on 16-bit frames): the dust map (NULL: none; frames of its
   size only), quarter turns clockwise (0..3), the draft block mean by 2^draft (0..8); then a frame of
   another size than the stack's is resampled to it (decode.rs:125). */
typedef struct {
    const lsb_dust_map* dust;
    uint32_t rotate;
    uint32_t draft;
} lsb_frame_prep;

/* Seeded synthetic stack description (no reference counterpart; the benchmark inputs). */
typedef struct {
    uint32_t w, h, n;
    uint32_t warp;          /* 1: a seeded similarity warp per frame */
    uint64_t seed;
    float mag_step;         /* frame k magnified by 1 + mag_step*k */
    float noise_std;
    float blur_px;          /* defocus sigma = blur_px * |z - f_k| */
    float warp_scale;       /* scale 1 + U(-a, a) */
    float warp_rot_deg;     /* rotation U(-a, a) degrees */
    float warp_shift;       /* translation U(-a, a) px */
} lsb_synth_desc;

/* The ABI version (LSB_ABI_VERSION), as crates/lapstack-raw/src/ffi.rs:69 lapstack_raw_abi. */
uint32_t lsb_abi(void);
/* Frees an error string any entry point returned (ffi.rs:148 lapstack_raw_free_str). */
void lsb_free_str(char* s);
/* Kernel launches the library has issued since it was loaded (no counterpart in the reference). */
uint64_t lsb_launch_count(void);

/* gpu.rs:308 `available` and the per-device context set-up (gpu.rs:312-324): one engine per device,
   its streams and its small persistent buffers. */
char* lsb_engine_create(const lsb_config* cfg, lsb_engine** out);
void lsb_engine_destroy(lsb_engine* e);
/* The engine's CUDA stream (cudaStream_t), for callers that share it (no counterpart in the reference). */
void* lsb_engine_stream(lsb_engine* e);

/* Checks settings without a device or an engine: NULL, or the error lsb_stack_begin would return
   for them (any pointer may be NULL; align and depth settings count only when enabled). The
   reference needs no counterpart: its options are typed enums, while a C caller passes codes. */
char* lsb_check_params(const lsb_fuse_params* fuse, const lsb_align_params* align, const lsb_depth_params* depth);

/* stack.rs:740 `fuse_range` creating its fuser (AnyFuser, stack.rs:123; GpuFuser::new, gpu.rs:359), with
   the stack's registration and depth passes (align / depth NULL or not enabled: off) and the
   brightness and crop switches of stack.rs:106-120 `Params`. */
char* lsb_stack_begin(lsb_engine* e, uint32_t w, uint32_t h, uint32_t n_frames, const lsb_fuse_params* fuse,
                      const lsb_align_params* align, const lsb_depth_params* depth, int32_t brightness, int32_t crop,
                      lsb_stack** out);
/* stack.rs:785-821 per frame: FrameSource::get_gpu, GpuFrames::process (gpu.rs:751) and
   GpuFuser::push_device (gpu.rs:451). One decoded frame: interleaved RGB u16, rows stride_px pixels apart (host or device pointer).
   The copy is asynchronous for page-locked memory: keep it unchanged until finish/run returns.
   The frame is registered on the device behind the next frame's copy; finish/run then warps,
   gains, REDUCEs and folds each pushed frame as soon as its transform is known. */
char* lsb_stack_push_u16(lsb_stack* s, const uint16_t* rgb, size_t stride_px);
/* gpu.rs:432 GpuFuser::push (stack.rs:152 AnyFuser::push): one frame as three planar f32 planes in
   [0,1] (host or device pointers); the frame is folded as given. */
char* lsb_stack_push_f32(lsb_stack* s, const float* const planes[3]);
/* The frame preparation of every frame pushed from now on (stack.rs:291-305 LazyFrames' dust, rotate and
   reduce; lapstack-web lib.rs:766-784), on the device as each frame lands: set it before the first push
   (the map is copied; p NULL clears it). The stack's w x h is the size the frames are brought to. */
char* lsb_stack_set_prep(lsb_stack* s, const lsb_frame_prep* p);
/* A decoded 16-bit frame of any size w x h (interleaved, host or device pointer), prepared as set
   (lsb_stack_set_prep) and brought to the stack's size (lapstack-web lib.rs:784 decode_for_run). With a
   preparation set, lsb_stack_push_u16 is this call with the stack's own size. */
char* lsb_stack_push_u16_sized(lsb_stack* s, const uint16_t* rgb, uint32_t w, uint32_t h);
/* The same preparation on one frame, on its own (host or device pointers; synchronous): in is w x h,
   out receives run_w x run_h (both 0: the prepared size, written to out_wh[0..1] in any case; out may be
   NULL to ask the size only). */
char* lsb_prep_frame_u16(lsb_engine* e, const lsb_frame_prep* p, const uint16_t* in, uint32_t w, uint32_t h, uint32_t run_w,
                         uint32_t run_h, uint16_t* out, uint32_t* out_wh);
/* The device buffer frames are pushed into ([n][h][w][3] u16), and a way to declare
   frames written there directly (count = frames now present). No counterpart in the reference. */
char* lsb_stack_frames_device(lsb_stack* s, uint16_t** frames_dev);
char* lsb_stack_set_count(lsb_stack* s, uint32_t count);
/* fuse.rs:315 shares of the frames pushed so far (runs the fold when needed); out_n holds n floats. */
char* lsb_stack_shares(lsb_stack* s, float* out_n);
/* stack.rs:181 AnyFuser::finish (gpu.rs:517), stack.rs:833 `fuse_and_depth` and align.rs:344
   `common_area`. Align, fold, depth: the whole pipeline over the frames pushed; may be called again.
   On an error *out is left empty (every pointer NULL, nothing to free). */
char* lsb_stack_finish(lsb_stack* s, lsb_result* out);
/* stack.rs:857 `weighted` / wav.rs:92 `weighted_average`: every frame of the last finish (or run),
   as folded (aligned, gains applied), averaged with weights that follow its contrast above the depth
   pass's per-cell noise floor; out receives 3*w*h planar f32 in [0,1] (host pointer). Needs a run
   with the depth pass. The stack's fold and depth results stay as they were. */
char* lsb_stack_weighted_average(lsb_stack* s, const lsb_wav_params* p, float* out);
/* stack.rs:76 `slab_ranges`: the slabs of a count-frame stack, size frames each (clamped to
   [1, count]), consecutive slabs overlapping by overlap (at most size - 1), the last cut short at the
   last frame. Writes the first max_slabs (lo, hi) pairs (inclusive frame indices) into lohi (may be
   NULL) and returns how many slabs there are (0 for an empty stack). Needs no device. */
uint32_t lsb_slab_ranges(uint32_t count, uint32_t size, uint32_t overlap, uint32_t* lohi, uint32_t max_slabs);
/* stack.rs:740 `fuse_range` with stack.rs:872 `fuse_slabs`'s cut and resize: frames lo..hi (inclusive)
   of the last finish (or run), as folded (aligned, gains applied), fused on their own with the stack's
   fusion settings, as a fresh fuser of those frames would fuse them; the stack's own results stay as
   they were. rect = {x, y, w, h} (NULL: the whole frame) cuts the fused image (pyramid.rs:31
   Img3::crop); out_w x out_h (both 0: rect's size) resamples the cut through prep.rs:46 `resize` with
   interpolation `interp` (align.rs:148 code; stack.rs:889 uses 3, Spline4x4). out receives
   3*ow*oh planar f32 (host pointer). */
char* lsb_stack_fuse_range(lsb_stack* s, uint32_t lo, uint32_t hi, const uint32_t* rect, uint32_t out_w, uint32_t out_h,
                           uint32_t interp, float* out);
/* prep.rs:46 `resize` / :63 `resize_plane` (stack.rs:951 `restretched`): `planes` host planes of
   pw x ph resampled to w x h through the scaling warp with pixel centres kept (output pixel o reads
   source (o + 1/2) / k - 1/2 on each axis), taps clamped at the edge; equal sizes copy. */
char* lsb_resize(lsb_engine* e, const float* src, uint32_t planes, uint32_t pw, uint32_t ph, uint32_t w, uint32_t h, uint32_t interp,
                 float* out);
/* lsb_stack_finish without copying results back (device-resident benchmarking; no counterpart). */
char* lsb_stack_run(lsb_stack* s, double* ms_out12);
/* Explicit frees, as ffi.rs:129 lapstack_raw_free_image. */
void lsb_stack_destroy(lsb_stack* s);
void lsb_result_free(lsb_result* r);

/* gpu.rs:1327 depth_from_slices: slices [n][dh][dw] f32, fused [3][h][w] f32 (host pointers).
   On an error *out is left empty. */
char* lsb_depth_from_slices(lsb_engine* e, const float* slices, uint32_t n, const float* fused, uint32_t w, uint32_t h,
                            const lsb_depth_params* p, lsb_result* out);
/* depth.rs:1081 wls_solve on the device (host pointers, w*h each). ms: device time from the edge
   weights to the converged solution (FGS guess and MG-PCG), the solver's planes allocated first. */
char* lsb_wls_solve(lsb_engine* e, const float* d, const float* conf, const float* guide, uint32_t w, uint32_t h, float lambda,
                    float sigma_c, uint32_t max_iters, uint32_t edge_mode, uint32_t vcycle_mode, float* u, float* rel,
                    uint32_t* iters, double* ms);
/* align.rs:896 multiscale_align of luma planes tg onto rf (host pointers, w*h f32). */
char* lsb_align_pair(lsb_engine* e, const float* rf, const float* tg, uint32_t w, uint32_t h, const double* init8,
                     const uint8_t* free8, uint32_t coarsen, double* out8, uint32_t* evals);
/* align.rs:581 warp_cost of tgt (tw x th) warped by sim onto rf (aw x ah), host pointers. */
char* lsb_warp_cost(lsb_engine* e, const float* rf, uint32_t aw, uint32_t ah, const float* tgt, uint32_t tw, uint32_t th,
                    const double* sim8, double* cost);

/* lsb_warp_cost without any allocation (no counterpart in the reference). For a
 * host that runs the Nelder-Mead search itself and keeps its level planes in
 * device memory it manages -- an allocator arena, a pool it sized up front,
 * or a process where a new device allocation mid-search would stall or fail
 * (a cudaMalloc synchronises the device and may not be available at all to a
 * caller that only ever borrows memory). rf_dev (aw x ah) and tgt_dev
 * (tw x th) are device f32 planes; sims8 holds n_sims (1..9) Sim vectors;
 * costs (host, n_sims) receives the align.rs:581 costs. Planes follow the
 * limits of the other entry points (sides at most 65535, 3 w h below 2^31).
 * The scratch is a fixed 64,152-byte (62.6 KiB) array in the library's device
 * image, per GPU; its address is looked up on the first call on each device.
 * Every call is synchronous: it reads the costs back and waits for `stream`,
 * so it cannot run inside a stream capture. Calls that overlap on the GPU
 * (other threads, other streams) race on that scratch.
 * Returns NULL or a static error string (do not free it). */
const char* lsb_warp_cost_noalloc(const float* rf_dev, uint32_t aw, uint32_t ah, const float* tgt_dev, uint32_t tw,
                                  uint32_t th, const double* sims8, uint32_t n_sims, double* costs, void* stream);

/* Synthetic stacks (no counterpart in the reference; the benchmark inputs): [n][h][w][3] u16 into host memory (OpenMP) or device memory. truth (n*4, may be NULL):
   per frame scale, rotation (rad), tx, ty (px) applied. */
const char* lsb_synth_stack_host(const lsb_synth_desc* d, uint16_t* out, double* truth);
const char* lsb_synth_stack_device(const lsb_synth_desc* d, uint16_t* out_dev, double* truth, void* stream);

/* The learned warm start of the WLS solve (no counterpart in the reference):
 * a 4-level U-Net, 32 base channels, BF16 weights and activations with FP32
 * accumulation, mapping the quarter-resolution (guide luma, raw depth / dmax,
 * confidence) to the WLS solution / dmax. Weights: [tap][cout][cin] per layer,
 * 15 layers; the input layer reads 3 live channels of 32, the output layer
 * writes channel 0 of 32. Trained by its own forward/backward/Adam kernels. */
typedef struct lsb_unet lsb_unet;
char* lsb_unet_create(int32_t device, uint64_t seed, lsb_unet** out);
void lsb_unet_destroy(lsb_unet* u);
void lsb_unet_sizes(const lsb_unet* u, uint64_t* n_weights, uint64_t* n_biases);
/* host copies of the FP32 master weights/biases and of the last step's gradients (any may be NULL) */
char* lsb_unet_get_params(lsb_unet* u, float* w, float* b, float* gw, float* gb);
char* lsb_unet_set_params(lsb_unet* u, const float* w, const float* b);
/* The 3x3 convolutions' tensor-core path: 0 (the default) tcgen05 MMAs with TMEM accumulators, 1 the
   mma.sync path (the same products, another summation order; kept for comparison). */
char* lsb_unet_set_conv(lsb_unet* u, uint32_t path);
/* network grid of a dw x dh depth grid: ceil(d/2) rounded up to a multiple of 8 */
void lsb_unet_grid(uint32_t dw, uint32_t dh, uint32_t* H, uint32_t* W);
/* device planes (dw x dh) -> batch entry b of in_dev [B][H][W][32] bf16 and d_in_dev [B][H][W] f32 (= d / dmax) */
char* lsb_unet_prepare(const float* guide, const float* d, const float* conf, uint32_t dw, uint32_t dh, float dmax, void* in_dev,
                       float* d_in_dev, uint32_t b, void* stream);
/* out0_dev [B][H][W]: the network's correction; the prediction is d_in + out0 */
char* lsb_unet_forward(lsb_unet* u, const void* in_dev, const float* d_in_dev, uint32_t B, uint32_t H, uint32_t W, float* out0_dev);
/* the last forward pass's device time: CUDA events around its layers on the network's stream (the
   input copies excluded) */
char* lsb_unet_forward_ms(lsb_unet* u, float* ms);
/* forward, MSE of d_in + out0 against target_dev [B][H][W], backward, and Adam when lr > 0 */
char* lsb_unet_train_step(lsb_unet* u, const void* in_dev, const float* d_in_dev, const float* target_dev, uint32_t B, uint32_t H,
                          uint32_t W, float lr, double* loss_out);
/* The autotuner (no counterpart in the reference): the persistent kernels' grid
 * sizes (the fold's select kernel, the depth aggregation) timed on this stack's
 * frames (two full runs per candidate), the fastest kept by the engine for every
 * later run. The grid size changes no result. */
typedef struct {
    uint32_t candidates[3];
    double fold_ms[3], aggregate_ms[3];
    uint32_t grid_select, grid_aggregate;
} lsb_tuning;
char* lsb_stack_autotune(lsb_stack* s, lsb_tuning* out);
/* Several stacks of uneven sizes and frame counts, one result each (the batch
 * entry point of the boundary; stack.rs runs one stack per call). Stacks of one
 * engine run back to back on its streams; stacks of different engines on one
 * device run side by side, one host thread per engine (so a log callback may be
 * called from several threads). Engines made with a share of the SMs each
 * (lsb_config.grid_limit, which bounds the registration search's CTAs too) fill
 * the GPU together. Stacks of different engines with depth on must share the
 * focus measure and its radii. On an error every result is freed and the
 * message names the stack. */
char* lsb_batch_run(lsb_stack* const* stacks, uint32_t n_stacks, lsb_result* outs);
/* Use the network's prediction as the x0 of this stack's WLS solves (NULL: the
 * reference's FGS start). The stack does not own the network. */
char* lsb_stack_set_warm_start(lsb_stack* s, lsb_unet* u);
/* Device planes of the last run's depth grid (dw x dh, valid until the next
 * run; no counterpart in the reference): the guide luma, the median-filtered raw depth, the normalised
 * confidence and the WLS solution -- the network's inputs and target. */
char* lsb_stack_depth_planes(lsb_stack* s, const float** guide, const float** d, const float** conf, const float** u,
                             uint32_t* dw, uint32_t* dh);

#ifdef __cplusplus
}
#endif
#endif
