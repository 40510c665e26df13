// The C ABI of include/lapstack_b200.h: engine, stack and the standalone
// depth / WLS / registration entry points. A stack runs the reference's
// pipeline order (stack.rs:1011 `run_with` for in-memory frames): register
// every frame to the previous aligned one, equalise brightness, fold all
// frames level by level, fuse the residuals, collapse, take the shares, then
// the depth pass on the focus slices the fold took.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <map>
#include <future>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "lapstack_b200.h"
#include "lsb_align.h"
#include "lsb_depth.h"
#include "lsb_internal.h"
#include "lsb_prep.h"

using namespace lsb;

static std::atomic<unsigned long long> g_launches{0};
void lsb_launched() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void lsb_launched_add(long long k) { g_launches.fetch_add((uint64_t)k, std::memory_order_relaxed); }
uint64_t lsb_launched_now() { return g_launches.load(std::memory_order_relaxed); }
extern "C" uint64_t lsb_launch_count(void) { return g_launches.load(); }

static char* dup_err(const std::string& s) {
    char* p = (char*)malloc(s.size() + 1);
    memcpy(p, s.c_str(), s.size() + 1);
    return p;
}
static std::string fmt(const char* f, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}
#define TRY(expr)                                                                                  \
    do {                                                                                           \
        cudaError_t _e = (expr);                                                                   \
        if (_e != cudaSuccess) return dup_err(fmt("%s: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__, __LINE__)); \
    } while (0)

struct DevPool {
    std::vector<void*> ptrs;
    template <class T>
    cudaError_t get(T** p, size_t n) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(q);
        *p = (T*)q;
        return e;
    }
    void release() {
        for (void* p : ptrs) cudaFree(p);
        ptrs.clear();
    }
    ~DevPool() { release(); }
};

// Blocks per frame of the brightness sums (brightness.rs:67): their f64 partials are summed in block order.
constexpr int BRIGHT_PARTS = 512;
// Frames per selection chunk when the fold runs on the side stream as the transforms land.
constexpr int SEL_CHUNK = 10;
// Frames of the last selection chunk (it folds after the last frame lands).
constexpr int SEL_TAIL = 4;

struct lsb_engine {
    lsb_config cfg;
    int device, sms, grid;
    int grid_select = 0, grid_agg = 0;  // autotuned persistent grids (0: grid)
    int coop = 0;  // cooperative launch: the registration search runs on the device
    cudaStream_t s;
    cudaStream_t cs = nullptr;  // host -> device frame copies, overlapped with the work on s
    cudaEvent_t s_mark = nullptr;  // recorded on s so that cs can wait for the work queued before it
    cudaStream_t bs = nullptr;  // registration targets (luma + pyramid of the next frame) beside the search on s
    cudaStream_t rs = nullptr;  // read-back of each frame's transform as its search ends
    cudaStream_t ws = nullptr;  // each aligned frame's warp and brightness sums, behind the registration chain
    DevPool pool;
    unsigned *hist, *sel;
    float* scal;  // [floor, p90, max, ...]
    AlignCtx actx;
    cudaEvent_t ev[12];
    void log(const std::string& line) {
        if (cfg.log) cfg.log(line.c_str(), cfg.user);
    }
};

struct lsb_stack {
    lsb_engine* e;
    uint32_t w, h, n, count;
    lsb_fuse_params fp;
    lsb_align_params ap;
    lsb_depth_params dp;
    bool brightness, crop, f32src;
    int storage;  // lsb::Storage of the Gaussian levels >= 1 and the slices
    int levels, depth_level;
    std::vector<int> lw, lh;  // level dims 0..levels
    DevPool pool;
    uint16_t* frames = nullptr;
    float* frames_f32 = nullptr;
    void* warped = nullptr;  // aligned frames, written once before the fold (f32 planar or u16 interleaved)
    std::vector<void*> g;      // G storage per level 1..levels (index l)
    std::vector<float*> acc, best;
    std::vector<float*> halo_w;  // halo control: each frame's weights at the guide level and the coarser ones
    uint16_t* winner = nullptr;
    void* slices = nullptr;
    int dw = 0, dh = 0, bk = 1;
    FrameXform* xf_dev = nullptr;
    std::vector<FrameXform> xf;
    std::vector<double> sims;   // n*8
    std::vector<float> gains;   // n*3
    float* top = nullptr;       // fused residual [3][ht][wt]
    float *dev_s = nullptr, *ent_s = nullptr, *lnp = nullptr;
    float *img = nullptr, *img_tmp = nullptr;
    uint16_t* img_u16 = nullptr;
    unsigned* counts = nullptr;
    float* mx = nullptr;
    double *mpart = nullptr, *means = nullptr;
    int* status = nullptr;
    // registration scratch
    float *yt = nullptr, *yr = nullptr;
    std::vector<float*> pt, pr;
    BrightXform* bx_dev = nullptr;
    double* bpart = nullptr;
    // depth scratch
    float *yfull = nullptr, *guide = nullptr, *mi = nullptr, *vi = nullptr, *tmp = nullptr, *state = nullptr;
    float *draw = nullptr, *dmed = nullptr, *conf = nullptr, *mins = nullptr, *u = nullptr, *w2 = nullptr;
    float *t0 = nullptr, *t1 = nullptr, *t2 = nullptr, *abar = nullptr, *bbar = nullptr, *dfull = nullptr, *cfull = nullptr;
    bool folded = false;
    size_t align_evals = 0;
    float floor_v = 0.f, p90 = 0.f, rel = 0.f;
    double rel64 = 0.0;
    int iters = 0, iters_first = 0;
    uint32_t crop_rect[4] = {0, 0, 0, 0};  // the common area of the last run (x, y, w, h)
    float* gsel = nullptr;  // the frame groups' selection states of the small levels
    size_t gsel_floats = 0;
    double ms[12] = {0};
    // registration chained on the device: per-frame transforms, the last warp, evaluations
    double* sims_dev = nullptr;  // n*8
    double* warp_dev = nullptr;  // inverse [9], affine, identity
    unsigned long long* evals_dev = nullptr;
    int aligned_upto = 0;        // frames already registered (at push time)
    bool search_timed_out = false;  // the last chained registration gave up waiting
    std::vector<cudaEvent_t> copied;  // per frame: its host -> device copy is done
    // per frame: its search is done (on s), its transform is back in sims_pin (on rs)
    std::vector<cudaEvent_t> searched, sims_back;
    double* sims_pin = nullptr;        // page-locked mirror of sims_dev
    FrameXform* xf_pin = nullptr;      // page-locked: each frame's warp as the streamed warps read it
    BrightXform* bx_pin = nullptr;
    cudaEvent_t wdone = nullptr;       // the streamed warps and brightness sums are done (on ws)
    // two target buffers (luma + pyramid), filled on the side stream: frame i+1's while frame i searches
    float* yt2[2] = {nullptr, nullptr};
    std::vector<float*> pt2[2];
    cudaEvent_t tdone[2] = {nullptr, nullptr}, tfree[2] = {nullptr, nullptr};
    WlsSolver* ws = nullptr;  // planes of the depth grid's solve, kept across runs
    lsb_unet* net = nullptr;  // learned warm start of the solves (not owned)
    float* x0 = nullptr;      // its prediction on the depth grid
    float* winner_full = nullptr;  // the winner map at full size (finish)
    lsb_result* early = nullptr;   // finish: the result whose fused planes leave on rs while the depth runs
    cudaEvent_t fused_ev = nullptr;  // recorded on s once the fused planes and the winner map are written
    size_t x0_cells = 0;
    float* wav_w = nullptr;  // the weighted average's weight planes [n][dh][dw]
    int wav_frames = 0;
    std::vector<cudaEvent_t> chunk_ev;  // per selection chunk folded on ws: [start, after the fused kernel, end] of level 0
    int chunks = 0;                     // chunks the last streamed fold ran
    // a frame range fused on its own (stack.rs:740 `fuse_range`): its accumulators, residual and image, made
    // on first use so that the stack's own fold results stay as they were; its cut and resized output
    std::vector<float*> slab_acc, slab_best;
    float *slab_top = nullptr, *slab_img = nullptr, *slab_out = nullptr;
    size_t slab_out_floats = 0;
    // the frame preparation (lsb_stack_set_prep): the uploaded dust map, the turn and the draft level,
    // two staging buffers for frames as decoded (frame i uses i & 1) and one for a turned frame to resize
    bool prep_on = false;
    DustDev* dust = nullptr;
    int prep_rot = 0, prep_draft = 0;
    uint16_t* stage[2] = {nullptr, nullptr};
    size_t stage_px = 0;
    uint16_t* stage_mid = nullptr;
    size_t mid_px = 0;
    cudaEvent_t stage_free[2] = {nullptr, nullptr};
    ~lsb_stack() {
        delete dust;
        for (int b = 0; b < 2; b++) {
            if (stage[b]) cudaFree(stage[b]);
            if (stage_free[b]) cudaEventDestroy(stage_free[b]);
        }
        if (stage_mid) cudaFree(stage_mid);
        if (slab_out) cudaFree(slab_out);
        for (auto& v : chunk_ev) cudaEventDestroy(v);
        if (wav_w) cudaFree(wav_w);
        wls_destroy(ws);
        if (x0) cudaFree(x0);
        for (auto& v : copied) cudaEventDestroy(v);
        for (auto& v : searched) cudaEventDestroy(v);
        for (auto& v : sims_back) cudaEventDestroy(v);
        if (wdone) cudaEventDestroy(wdone);
        if (fused_ev) cudaEventDestroy(fused_ev);
        if (sims_pin) cudaFreeHost(sims_pin);
        if (xf_pin) cudaFreeHost(xf_pin);
        if (bx_pin) cudaFreeHost(bx_pin);
        for (int b = 0; b < 2; b++) {
            if (tdone[b]) cudaEventDestroy(tdone[b]);
            if (tfree[b]) cudaEventDestroy(tfree[b]);
        }
    }
};

namespace lsb {
cudaError_t unet_warm_start(lsb_unet* u, const float* guide, const float* d, const float* conf, int dw, int dh, float dmax, float* x0,
                            cudaStream_t st);
}

// The x0 of this run's solves: the network's prediction (learned warm start)
// or none (the reference's FGS start).
static cudaError_t warm_start(lsb_stack* s, int dw, int dh, int n, cudaStream_t st, bool* given) {
    *given = false;
    if (!s->net) return cudaSuccess;
    const size_t m = (size_t)dw * dh;
    if (s->x0_cells < m) {
        if (s->x0) cudaFree(s->x0);
        s->x0 = nullptr;
        s->x0_cells = 0;
        cudaError_t e = cudaMalloc(&s->x0, m * sizeof(float));
        if (e != cudaSuccess) return e;
        s->x0_cells = m;
    }
    cudaError_t e = lsb::unet_warm_start(s->net, s->guide, s->dmed, s->conf, dw, dh, (float)std::max(n - 1, 1), s->x0, st);
    if (e == cudaSuccess) *given = true;
    return e;
}

static bool chained(const lsb_stack* s);
static char* align_frame(lsb_stack* s, int i);

// The stack's WLS solver for a dw x dh grid and this run's guide: planes
// allocated on the first run, edge weights recomputed every run.
static WlsSolver* stack_solver(lsb_stack* s, int dw, int dh, const lsb_depth_params& dp, cudaStream_t st, cudaError_t* ce) {
    *ce = cudaSuccess;
    if (s->ws && (wls_width(s->ws) != dw || wls_height(s->ws) != dh)) {
        wls_destroy(s->ws);
        s->ws = nullptr;
    }
    if (!s->ws) {
        s->ws = wls_alloc(dw, dh, ce);
        if (*ce != cudaSuccess) {
            wls_destroy(s->ws);
            s->ws = nullptr;
            return nullptr;
        }
    }
    *ce = wls_prepare(s->ws, s->guide, dp.lambda, dp.sigma_c, (int)dp.edge_mode, st);
    return s->ws;
}

// Everything lsb_engine_create makes; on an error the caller frees what was made with lsb_engine_destroy.
static char* engine_init(lsb_engine* e) {
    int ndev = 0;
    cudaError_t r = cudaGetDeviceCount(&ndev);
    if (r != cudaSuccess || ndev == 0)
        return dup_err(fmt("lapstack-b200 needs a CUDA device: %s", r != cudaSuccess ? cudaGetErrorString(r) : "none found"));
    TRY(cudaSetDevice(e->device));
    cudaDeviceProp prop;
    TRY(cudaGetDeviceProperties(&prop, e->device));
    if (prop.major < 10)
        return dup_err(fmt("lapstack-b200 is built for sm_100a; device %d is sm_%d%d", e->device, prop.major, prop.minor));
    e->sms = prop.multiProcessorCount;
    e->grid = e->cfg.grid_limit > 0 ? e->cfg.grid_limit : 2 * e->sms;
    // The registration chain (on s, its targets on bs) sets the pace of an aligned stack: its blocks go
    // first when the per-frame warps, sums and fold chunks on ws wait for room on the SMs.
    int prio_low = 0, prio_high = 0;
    TRY(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    TRY(cudaStreamCreateWithPriority(&e->s, cudaStreamNonBlocking, prio_high));
    TRY(cudaStreamCreateWithFlags(&e->cs, cudaStreamNonBlocking));
    TRY(cudaEventCreateWithFlags(&e->s_mark, cudaEventDisableTiming));
    TRY(cudaStreamCreateWithPriority(&e->bs, cudaStreamNonBlocking, prio_high));
    TRY(cudaStreamCreateWithFlags(&e->rs, cudaStreamNonBlocking));
    TRY(cudaStreamCreateWithPriority(&e->ws, cudaStreamNonBlocking, prio_low));
    TRY(e->pool.get(&e->hist, 65536));
    TRY(e->pool.get(&e->sel, 4));
    TRY(e->pool.get(&e->scal, 16));
    e->actx.s = e->s;
    e->actx.max_blocks = e->cfg.grid_limit > 0 ? e->cfg.grid_limit : 0;
    TRY(e->pool.get(&e->actx.part, MAX_CAND * 296 * 3));
    TRY(e->pool.get(&e->actx.sums_dev, MAX_CAND * 3));
    TRY(cudaHostAlloc((void**)&e->actx.sums_host, sizeof(double) * MAX_CAND * 3, cudaHostAllocDefault));
    TRY(e->pool.get(&e->actx.nm_part, (size_t)2 * MAX_CAND * NM_MAX_BLOCKS * 3));
    TRY(e->pool.get(&e->actx.nm_ctl, 4));
    TRY(e->pool.get(&e->actx.nm_out, 8));
    {
        int coop = 0;
        TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, e->cfg.device));
        e->coop = coop;
    }
    for (auto& v : e->ev) TRY(cudaEventCreate(&v));
    return nullptr;
}

extern "C" {

uint32_t lsb_abi(void) { return LSB_ABI_VERSION; }
void lsb_free_str(char* s) { free(s); }

char* lsb_engine_create(const lsb_config* cfg, lsb_engine** out) {
    *out = nullptr;
    lsb_engine* e = new lsb_engine();  // value-initialised: every stream, event and pointer starts null
    e->cfg = cfg ? *cfg : lsb_config{0, 0, 0, 0, nullptr, nullptr};
    e->device = e->cfg.device;
    if (char* err = engine_init(e)) {
        lsb_engine_destroy(e);
        return err;
    }
    *out = e;
    return nullptr;
}

void lsb_engine_destroy(lsb_engine* e) {
    if (!e) return;
    if (e->s) cudaStreamSynchronize(e->s);
    for (auto& v : e->ev)
        if (v) cudaEventDestroy(v);
    if (e->actx.sums_host) cudaFreeHost(e->actx.sums_host);
    e->pool.release();
    if (e->cs) cudaStreamSynchronize(e->cs), cudaStreamDestroy(e->cs);
    if (e->s_mark) cudaEventDestroy(e->s_mark);
    if (e->bs) cudaStreamSynchronize(e->bs), cudaStreamDestroy(e->bs);
    if (e->rs) cudaStreamSynchronize(e->rs), cudaStreamDestroy(e->rs);
    if (e->ws) cudaStreamSynchronize(e->ws), cudaStreamDestroy(e->ws);
    if (e->s) cudaStreamDestroy(e->s);
    delete e;
}

void* lsb_engine_stream(lsb_engine* e) { return e ? (void*)e->s : nullptr; }

}  // extern "C"

static size_t gs_bytes(const lsb_stack* s) { return s->storage == STORE_F32 ? 4 : 2; }

// depth.rs:454 `rdf_taps` in depth.rs:417 `conv_sparse`'s per-pixel order
static std::vector<float> focus_taps(uint32_t r_in, uint32_t r_out) {
    std::vector<std::array<int, 2>> disk, ring;
    int ri2 = (int)(r_in * r_in), ro2 = (int)(r_out * r_out), r = (int)r_out;
    for (int dy = -r; dy <= r; dy++)
        for (int dx = -r; dx <= r; dx++) {
            int d2 = dx * dx + dy * dy;
            if (d2 <= ri2) disk.push_back({dy, dx});
            else if (d2 <= ro2) ring.push_back({dy, dx});
        }
    float wd = 1.0f / (float)disk.size(), wr = -1.0f / (float)std::max<size_t>(ring.size(), 1);
    std::vector<std::array<float, 3>> list;
    for (auto& p : disk) list.push_back({(float)p[0], (float)p[1], wd});
    for (auto& p : ring) list.push_back({(float)p[0], (float)p[1], wr});
    std::vector<float> dys, out;
    for (auto& t : list)
        if (std::find(dys.begin(), dys.end(), t[0]) == dys.end()) dys.push_back(t[0]);
    for (float dy : dys)
        for (auto& t : list)
            if (t[0] == dy) out.insert(out.end(), {t[0], t[1], t[2]});
    return out;
}

static char* stack_alloc(lsb_stack* s) {
    DevPool& P = s->pool;
    const size_t W = s->w, H = s->h, N = s->n;
    // fold inputs carry 64 bytes of tail padding: the async tile copies read whole words
    TRY(P.get(&s->frames, N * W * H * 3 + 32));
    s->g.assign(s->levels + 1, nullptr);
    s->acc.assign(s->levels, nullptr);
    s->best.assign(s->levels, nullptr);
    for (int l = 1; l <= s->levels; l++) {
        void* p = nullptr;
        TRY(cudaMalloc(&p, N * 3 * (size_t)s->lw[l] * s->lh[l] * gs_bytes(s) + 64));
        P.ptrs.push_back(p);
        s->g[l] = p;
    }
    for (int l = 0; l < s->levels; l++) {
        TRY(P.get(&s->acc[l], 3 * (size_t)s->lw[l] * s->lh[l]));
        TRY(P.get(&s->best[l], (size_t)s->lw[l] * s->lh[l]));
    }
    TRY(P.get(&s->winner, (size_t)s->lw[s->depth_level] * s->lh[s->depth_level]));
    const size_t nt = (size_t)s->lw[s->levels] * s->lh[s->levels];
    TRY(P.get(&s->top, 3 * nt));
    TRY(P.get(&s->dev_s, N * nt));
    TRY(P.get(&s->ent_s, N * nt));
    TRY(P.get(&s->lnp, 128));
    TRY(P.get(&s->img, 3 * W * H));
    TRY(P.get(&s->img_tmp, 3 * W * H));
    TRY(P.get(&s->img_u16, 3 * W * H));
    TRY(P.get(&s->counts, N));
    TRY(P.get(&s->mx, 4));
    TRY(P.get(&s->mpart, N * 64 * 3));
    TRY(P.get(&s->means, N * 3));
    TRY(P.get(&s->status, 4));
    s->gsel_floats = (size_t)16 << 20;  // 64 MB: the small levels' frame-group states
    TRY(P.get(&s->gsel, s->gsel_floats));
    TRY(P.get(&s->xf_dev, N));
    if (s->dp.enabled) {
        s->bk = 1 << s->dp.scale;
        s->dw = (int)((W + s->bk - 1) / s->bk);
        s->dh = (int)((H + s->bk - 1) / s->bk);
        const size_t m = (size_t)s->dw * s->dh;
        void* p = nullptr;
        TRY(cudaMalloc(&p, N * m * gs_bytes(s)));
        P.ptrs.push_back(p);
        s->slices = p;
        for (float** q : {&s->guide, &s->mi, &s->vi, &s->tmp, &s->draw, &s->dmed, &s->conf, &s->mins, &s->u, &s->w2, &s->t0,
                          &s->t1, &s->t2, &s->abar, &s->bbar})
            TRY(P.get(q, m));
        TRY(P.get(&s->state, 9 * m));
        TRY(P.get(&s->yfull, W * H));
        TRY(P.get(&s->dfull, W * H));
        TRY(P.get(&s->cfull, W * H));
    }
    if (s->ap.enabled && N > 1) {
        {
            void* p = nullptr;
            TRY(cudaMalloc(&p, N * W * H * (s->storage == STORE_F32 ? 3 * sizeof(float) : 3 * sizeof(uint16_t)) + 64));
            P.ptrs.push_back(p);
            s->warped = p;
        }
        TRY(P.get(&s->yt, W * H));
        TRY(P.get(&s->yr, W * H));
        std::vector<std::pair<int, int>> dims;
        gauss_dims((int)W, (int)H, dims);
        for (auto& d : dims) {
            float *a, *b;
            TRY(P.get(&a, (size_t)d.first * d.second));
            TRY(P.get(&b, (size_t)d.first * d.second));
            s->pt.push_back(a);
            s->pr.push_back(b);
        }
        TRY(P.get(&s->bx_dev, N));
        TRY(P.get(&s->bpart, N * BRIGHT_PARTS * 7));
        TRY(P.get(&s->sims_dev, (size_t)N * 8));
        s->yt2[0] = s->yt;
        s->pt2[0] = s->pt;
        TRY(P.get(&s->yt2[1], W * H));
        for (auto& d : dims) {
            float* a;
            TRY(P.get(&a, (size_t)d.first * d.second));
            s->pt2[1].push_back(a);
        }
        for (int b = 0; b < 2; b++) {
            TRY(cudaEventCreateWithFlags(&s->tdone[b], cudaEventDisableTiming));
            TRY(cudaEventCreateWithFlags(&s->tfree[b], cudaEventDisableTiming));
        }
        TRY(P.get(&s->warp_dev, 16));
        TRY(P.get(&s->evals_dev, 1));
        TRY(cudaHostAlloc((void**)&s->sims_pin, sizeof(double) * 8 * N, cudaHostAllocDefault));
        TRY(cudaHostAlloc((void**)&s->xf_pin, sizeof(FrameXform) * N, cudaHostAllocDefault));
        TRY(cudaHostAlloc((void**)&s->bx_pin, sizeof(BrightXform) * N, cudaHostAllocDefault));
        s->searched.assign(N, nullptr);
        s->sims_back.assign(N, nullptr);
        for (auto& v : s->searched) TRY(cudaEventCreateWithFlags(&v, cudaEventDisableTiming));
        for (auto& v : s->sims_back) TRY(cudaEventCreateWithFlags(&v, cudaEventDisableTiming));
        TRY(cudaEventCreateWithFlags(&s->wdone, cudaEventDisableTiming));
        s->chunk_ev.assign(3 * ((N + SEL_CHUNK - 1) / SEL_CHUNK + 1), nullptr);
        for (auto& v : s->chunk_ev) TRY(cudaEventCreate(&v));
    }
    s->copied.assign(N, nullptr);
    for (auto& v : s->copied) TRY(cudaEventCreateWithFlags(&v, cudaEventDisableTiming));
    return nullptr;
}

// The settings' ranges: the codes the reference's typed options can take (fuse.rs:59 TopRule,
// align.rs:95 AlignModel, align.rs:148 Interp, depth.rs:112 FocusMeasure, depth.rs:127 Upsample),
// which a C caller could otherwise pass out of range and have read as another option, and the
// radii this engine's kernels are built for. Align and depth settings count only when enabled.
static const char* params_error(const lsb_fuse_params* f, const lsb_align_params* a, const lsb_depth_params* d) {
    if (f) {
        if (f->energy_radius > 2) return "energy_radius must be 0..2";
        if (f->top_rule > 2) return "top_rule must be 0 (dev-entropy), 1 (deviation) or 2 (average)";
        if (f->top_radius > 4) return "top_radius must be 0..4";
    }
    if (a && a->enabled) {
        if (a->model > 2) return "align model must be 0 (similarity), 1 (affine) or 2 (projective)";
        if (a->interp > 5) return "interp must be 0..5 (nearest, bilinear, bicubic, spline4x4, spline6x6, lanczos3)";
    }
    if (d && d->enabled) {
        if (d->scale > 2) return "depth scale must be 0..2";
        if (d->focus > 1) return "focus must be 0 (ring difference) or 1 (sum-modified Laplacian)";
        if (d->focus == 0 && (d->r_out > 3 || d->r_out <= d->r_in)) return "rdf radii: r_in < r_out <= 3";
        if (d->focus == 1 && (d->sml_step < 1 || d->sml_step > 3)) return "sml step must be 1..3";
        // bounded first: the tile size below is computed in int
        if (d->agg_radius > 64 || aggregate_smem_bytes((int)d->agg_radius) > 227 * 1024) return "agg_radius too large";
        if (d->upsample > 1) return "upsample must be 0 (bilinear) or 1 (guided)";
        if (d->up_radius > (1u << 20)) return "up_radius must be at most 2^20";
        if (d->edge_mode > 1) return "edge_mode must be 0 or 1";
        if (d->vcycle_mode > 1) return "vcycle_mode must be 0 or 1";
    }
    return nullptr;
}

// Image sizes the kernels index safely: one grid row per image row in some launches (at most 65535),
// and plane offsets within a frame (3 w h) in 32-bit ints.
static const char* size_error(uint32_t w, uint32_t h) {
    if (w == 0 || h == 0) return "width and height must be at least 1";
    if (w > 65535 || h > 65535) return "width and height must be at most 65535";
    if ((uint64_t)w * h * 3 > 0x7fffffffull) return "at most 715 Mpx per frame (3 w h must fit 31 bits)";
    return nullptr;
}

extern "C" char* lsb_check_params(const lsb_fuse_params* fuse, const lsb_align_params* align, const lsb_depth_params* depth) {
    const char* bad = params_error(fuse, align, depth);
    return bad ? dup_err(bad) : nullptr;
}

extern "C" char* lsb_stack_begin(lsb_engine* e, uint32_t w, uint32_t h, uint32_t n_frames, const lsb_fuse_params* fuse,
                                 const lsb_align_params* align, const lsb_depth_params* depth, int32_t brightness, int32_t crop,
                                 lsb_stack** out) {
    *out = nullptr;
    if (!e) return dup_err("no engine");
    if (w == 0 || h == 0 || n_frames == 0) return dup_err("a stack needs a size and at least one frame");
    if (n_frames > 65535) return dup_err("at most 65535 frames (the winner map is u16)");
    if (const char* bad = size_error(w, h)) return dup_err(bad);
    lsb_stack* s = new lsb_stack();
    s->e = e;
    s->w = w;
    s->h = h;
    s->n = n_frames;
    s->count = 0;
    s->fp = fuse ? *fuse : lsb_fuse_params{0, 1, 0, 2, 256, 0, 2, 0.f};
    s->ap = align ? *align : lsb_align_params{0, 1, 1, 1, 0, 0, 3, 0};
    s->dp = depth ? *depth : lsb_depth_params{};
    s->brightness = brightness != 0;
    s->crop = crop != 0;
    s->storage = e->cfg.storage;
    if (s->storage < 0 || s->storage > 2) {
        delete s;
        return dup_err("storage must be 0 (FP32), 1 (UNORM16 levels, FP16 slices) or 2 (FP16)");
    }
    s->f32src = false;
    if (const char* bad = params_error(&s->fp, &s->ap, &s->dp)) {
        delete s;
        return dup_err(bad);
    }
    // pyramid.rs:191 auto_levels(w, h, 32); fuse.rs:372-373
    uint32_t levels = s->fp.levels;
    if (levels == 0) {
        size_t cw = w, ch = h, k = 0;
        while ((cw > 1 || ch > 1) && std::min((cw + 1) / 2, (ch + 1) / 2) >= 32) {
            cw = (cw + 1) / 2;
            ch = (ch + 1) / 2;
            k++;
        }
        levels = (uint32_t)std::max<size_t>(k, 1);
    }
    s->levels = (int)levels;
    s->depth_level = (int)std::min(s->fp.depth_level, levels - 1);
    s->lw.push_back((int)w);
    s->lh.push_back((int)h);
    for (int l = 1; l <= s->levels; l++) {
        s->lw.push_back((s->lw.back() + 1) / 2);
        s->lh.push_back((s->lh.back() + 1) / 2);
    }
    char* err = stack_alloc(s);
    if (err) {
        delete s;
        return err;
    }
    s->sims.assign((size_t)n_frames * 8, 0.0);
    for (uint32_t k = 0; k < n_frames; k++) {
        s->sims[8 * k + 2] = 1.0;
        s->sims[8 * k + 4] = 1.0;
    }
    s->gains.assign((size_t)n_frames * 3, 1.f);
    *out = s;
    return nullptr;
}

static bool is_device_ptr(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

extern "C" char* lsb_stack_push_u16_sized(lsb_stack* s, const uint16_t* rgb, uint32_t w, uint32_t h);
extern "C" char* lsb_stack_push_u16(lsb_stack* s, const uint16_t* rgb, size_t stride_px) {
    if (!s || !rgb) return dup_err("null argument");
    if (s->f32src) return dup_err("this stack takes f32 frames");
    if (s->count >= s->n) return dup_err(fmt("the stack holds %u frames", s->n));
    if (s->prep_on) {
        if (stride_px != 0 && stride_px != s->w) return dup_err("a prepared frame is pushed without a row stride");
        return lsb_stack_push_u16_sized(s, rgb, s->w, s->h);
    }
    if (stride_px == 0) stride_px = s->w;
    if (stride_px < s->w) return dup_err("stride_px < width");
    uint16_t* dst = s->frames + (size_t)s->count * s->w * s->h * 3;
    cudaMemcpyKind kind = is_device_ptr(rgb) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    // the copy runs on the engine's copy stream; the work on this frame waits for it
    lsb_engine* e = s->e;
    const int i = (int)s->count;
    if (i == 0) {  // the frame store is rewritten: wait for whatever still reads it on the work stream
        TRY(cudaEventRecord(e->s_mark, e->s));
        TRY(cudaStreamWaitEvent(e->cs, e->s_mark, 0));
    }
    if (stride_px == s->w) TRY(cudaMemcpyAsync(dst, rgb, sizeof(uint16_t) * 3 * (size_t)s->w * s->h, kind, e->cs));
    else TRY(cudaMemcpy2DAsync(dst, 6 * (size_t)s->w, rgb, 6 * stride_px, 6 * (size_t)s->w, s->h, kind, e->cs));
    TRY(cudaEventRecord(s->copied[i], e->cs));
    TRY(cudaStreamWaitEvent(e->s, s->copied[i], 0));
    s->count++;
    s->folded = false;
    // register this frame now, behind the copy of the next one (stack.rs:785-821 does it per frame too)
    if (s->ap.enabled && s->n > 1 && chained(s) && s->aligned_upto == i)
        if (char* er = align_frame(s, i)) return er;
    return nullptr;
}

// stack.rs:52-58 / 291-305 (LazyFrames' dust, rotate, reduce) as lapstack-web lib.rs:766-784 does them on
// 16-bit frames: the map is uploaded once, the rest is set per stack
extern "C" char* lsb_stack_set_prep(lsb_stack* s, const lsb_frame_prep* p) {
    if (!s) return dup_err("null stack");
    if (s->count > 0) return dup_err("set the frame preparation before the first push");
    if (s->f32src) return dup_err("this stack takes f32 frames");
    if (p && p->rotate > 3) return dup_err("prep: rotate must be 0..3 quarter turns");
    if (p && p->draft > 8) return dup_err("prep: draft must be 0..8");
    DustDev* d = nullptr;
    if (p && p->dust) {
        std::string why = dust_create(p->dust, &d);
        if (!why.empty()) return dup_err(why);
    }
    delete s->dust;
    s->dust = d;
    s->prep_on = p != nullptr;
    s->prep_rot = p ? (int)p->rotate : 0;
    s->prep_draft = p ? (int)p->draft : 0;
    for (int b = 0; b < 2; b++)
        if (!s->stage_free[b]) TRY(cudaEventCreateWithFlags(&s->stage_free[b], cudaEventDisableTiming));
    return nullptr;
}

// A buffer of at least px pixels (3 u16 each), grown once nothing on the copy stream still uses it.
static cudaError_t grow_u16(uint16_t** buf, size_t* have, size_t px, cudaStream_t cs) {
    if (*have >= px) return cudaSuccess;
    cudaError_t e = cudaStreamSynchronize(cs);
    if (e != cudaSuccess) return e;
    if (*buf) cudaFree(*buf);
    *buf = nullptr;
    *have = 0;
    e = cudaMalloc(buf, sizeof(uint16_t) * 3 * px);
    if (e == cudaSuccess) *have = px;
    return e;
}

// lapstack-web lib.rs:766-784 `decode` + `decode_for_run` on the device, on the copy stream: the frame as
// decoded into a staging buffer, the dust map (frames of its size only), the turn and draft block mean in
// one gather, and a frame of another size resampled to the stack's (decode.rs:125), into frame i's slot.
extern "C" char* lsb_stack_push_u16_sized(lsb_stack* s, const uint16_t* rgb, uint32_t w, uint32_t h) {
    if (!s || !rgb) return dup_err("null argument");
    if (s->f32src) return dup_err("this stack takes f32 frames");
    if (s->count >= s->n) return dup_err(fmt("the stack holds %u frames", s->n));
    if (const char* why = size_error(w, h)) return dup_err(fmt("frame: %s", why));
    if (!s->prep_on && w == s->w && h == s->h) return lsb_stack_push_u16(s, rgb, 0);
    if (!s->prep_on) {  // only a resize: a preparation without steps
        lsb_frame_prep none{nullptr, 0, 0};
        if (char* er = lsb_stack_set_prep(s, &none)) return er;
    }
    lsb_engine* e = s->e;
    const int i = (int)s->count, b = i & 1;
    cudaStream_t cs = e->cs;
    if (i == 0) {  // the frame store is rewritten: wait for whatever still reads it on the work stream
        TRY(cudaEventRecord(e->s_mark, e->s));
        TRY(cudaStreamWaitEvent(cs, e->s_mark, 0));
    }
    const size_t px = (size_t)w * h;
    if (s->stage_px < px) {
        // both staging buffers, grown together once the copy stream is idle
        TRY(cudaStreamSynchronize(cs));
        for (int k = 0; k < 2; k++) {
            size_t have = 0;
            TRY(grow_u16(&s->stage[k], &have, px, cs));
        }
        s->stage_px = px;
    }
    TRY(cudaStreamWaitEvent(cs, s->stage_free[b], 0));
    uint16_t* raw = s->stage[b];
    cudaMemcpyKind kind = is_device_ptr(rgb) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    TRY(cudaMemcpyAsync(raw, rgb, sizeof(uint16_t) * 3 * px, kind, cs));
    if (s->dust && (int)w == s->dust->W && (int)h == s->dust->H) TRY(dust_apply_rgb16(s->dust, raw, cs));
    int pw = (int)w, ph = (int)h;
    const uint16_t* cur = raw;
    uint16_t* dst = s->frames + (size_t)i * s->w * s->h * 3;
    const bool turn = s->prep_rot != 0 || s->prep_draft != 0;
    if (turn) turn_draft_dims((int)w, (int)h, s->prep_rot, s->prep_draft, &pw, &ph);
    const bool resize = pw != (int)s->w || ph != (int)s->h;
    if (turn) {
        uint16_t* o = dst;
        if (resize) {
            TRY(grow_u16(&s->stage_mid, &s->mid_px, (size_t)pw * ph, cs));
            o = s->stage_mid;
        }
        TRY(turn_draft_rgb16(raw, (int)w, (int)h, s->prep_rot, s->prep_draft, o, cs));
        cur = o;
    }
    if (resize) TRY(resize_rgb16(cur, pw, ph, dst, (int)s->w, (int)s->h, cs));
    else if (!turn) TRY(cudaMemcpyAsync(dst, raw, sizeof(uint16_t) * 3 * px, cudaMemcpyDeviceToDevice, cs));
    TRY(cudaEventRecord(s->stage_free[b], cs));
    TRY(cudaEventRecord(s->copied[i], cs));
    TRY(cudaStreamWaitEvent(e->s, s->copied[i], 0));
    s->count++;
    s->folded = false;
    if (s->ap.enabled && s->n > 1 && chained(s) && s->aligned_upto == i)
        if (char* er = align_frame(s, i)) return er;
    return nullptr;
}

// One frame through lsb_frame_prep on its own, synchronously on the engine's copy stream.
extern "C" char* lsb_prep_frame_u16(lsb_engine* e, const lsb_frame_prep* p, const uint16_t* in, uint32_t w, uint32_t h, uint32_t run_w,
                                    uint32_t run_h, uint16_t* out, uint32_t* out_wh) {
    if (!e || !p || !in || !out_wh) return dup_err("null argument");
    if (const char* why = size_error(w, h)) return dup_err(fmt("frame: %s", why));
    if (p->rotate > 3) return dup_err("prep: rotate must be 0..3 quarter turns");
    if (p->draft > 8) return dup_err("prep: draft must be 0..8");
    if ((run_w == 0) != (run_h == 0)) return dup_err("prep: give both run dimensions or neither");
    int pw = (int)w, ph = (int)h;
    turn_draft_dims((int)w, (int)h, (int)p->rotate, (int)p->draft, &pw, &ph);
    const int ow = run_w ? (int)run_w : pw, oh = run_h ? (int)run_h : ph;
    if (const char* why = size_error((uint32_t)ow, (uint32_t)oh)) return dup_err(fmt("prep output: %s", why));
    out_wh[0] = (uint32_t)ow;
    out_wh[1] = (uint32_t)oh;
    if (!out) return nullptr;
    DustDev* d = nullptr;
    if (p->dust) {
        std::string why = dust_create(p->dust, &d);
        if (!why.empty()) return dup_err(why);
    }
    cudaStream_t cs = e->cs;
    uint16_t *raw = nullptr, *mid = nullptr, *res = nullptr;
    cudaError_t ce = cudaMalloc(&raw, sizeof(uint16_t) * 3 * (size_t)w * h);
    if (ce == cudaSuccess) ce = cudaMalloc(&mid, sizeof(uint16_t) * 3 * (size_t)pw * ph);
    if (ce == cudaSuccess) ce = cudaMalloc(&res, sizeof(uint16_t) * 3 * (size_t)ow * oh);
    const cudaMemcpyKind ki = is_device_ptr(in) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind ko = is_device_ptr(out) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(raw, in, sizeof(uint16_t) * 3 * (size_t)w * h, ki, cs);
    if (ce == cudaSuccess && d && (int)w == d->W && (int)h == d->H) ce = dust_apply_rgb16(d, raw, cs);
    if (ce == cudaSuccess) ce = turn_draft_rgb16(raw, (int)w, (int)h, (int)p->rotate, (int)p->draft, mid, cs);
    if (ce == cudaSuccess) {
        if (ow != pw || oh != ph) ce = resize_rgb16(mid, pw, ph, res, ow, oh, cs);
        else ce = cudaMemcpyAsync(res, mid, sizeof(uint16_t) * 3 * (size_t)ow * oh, cudaMemcpyDeviceToDevice, cs);
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(out, res, sizeof(uint16_t) * 3 * (size_t)ow * oh, ko, cs);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(cs);
    cudaStreamSynchronize(cs);
    cudaFree(raw);
    cudaFree(mid);
    cudaFree(res);
    delete d;
    if (ce != cudaSuccess) return dup_err(fmt("prep: %s", cudaGetErrorString(ce)));
    return nullptr;
}

extern "C" char* lsb_stack_push_f32(lsb_stack* s, const float* const planes[3]) {
    if (!s || !planes) return dup_err("null argument");
    if (s->count >= s->n) return dup_err(fmt("the stack holds %u frames", s->n));
    if (s->ap.enabled && s->n > 1) return dup_err("f32 frames are folded as given: disable alignment");
    if (!s->frames_f32) {
        if (s->count > 0) return dup_err("this stack takes u16 frames");
        void* p = nullptr;
        TRY(cudaMalloc(&p, sizeof(float) * 3 * (size_t)s->n * s->w * s->h));
        s->pool.ptrs.push_back(p);
        s->frames_f32 = (float*)p;
        s->f32src = true;
    }
    const size_t np = (size_t)s->w * s->h;
    for (int c = 0; c < 3; c++) {
        cudaMemcpyKind kind = is_device_ptr(planes[c]) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        TRY(cudaMemcpyAsync(s->frames_f32 + ((size_t)s->count * 3 + c) * np, planes[c], sizeof(float) * np, kind, s->e->s));
    }
    s->count++;
    s->folded = false;
    return nullptr;
}

extern "C" char* lsb_stack_frames_device(lsb_stack* s, uint16_t** frames_dev) {
    if (!s || !frames_dev) return dup_err("null argument");
    *frames_dev = s->frames;
    return nullptr;
}

extern "C" char* lsb_stack_set_count(lsb_stack* s, uint32_t count) {
    if (!s) return dup_err("null argument");
    if (count > s->n) return dup_err("count exceeds the stack's frames");
    s->count = count;
    s->folded = false;
    s->aligned_upto = 0;
    return nullptr;
}

// ------------------------------------------------------------- pipeline
static void free_mask(const lsb_stack* s, bool freem[8]) {
    const bool aff = s->ap.model != 0, proj = s->ap.model == 2;
    const bool m[8] = {s->ap.shift != 0, s->ap.shift != 0, s->ap.scale != 0, s->ap.rotation != 0, aff, aff, proj, proj};
    memcpy(freem, m, sizeof m);
}
// Registration chained on the device (stack.rs:513-530 per frame): frame i's
// luma and pyramid, its search from frame i-1's transform against frame
// i-1's aligned luma, then its own aligned luma as frame i+1's reference.
// Nothing returns to the host between frames.
static bool chained(const lsb_stack* s) { return !s->ap.host_search && s->e->coop; }
static char* run_align_host(lsb_stack* s);
static char* align_frame(lsb_stack* s, int i) {
    lsb_engine* e = s->e;
    AlignCtx& C = e->actx;
    const int W = (int)s->w, H = (int)s->h, n = (int)s->n;
    const uint16_t* f = s->frames + (size_t)i * W * H * 3;
    if (i == 0) {
        static const double id[8] = {0, 0, 1, 0, 1, 0, 0, 0};
        TRY(align_chain_begin(C, s->evals_dev));
        TRY(cudaMemcpyAsync(s->sims_dev, id, sizeof id, cudaMemcpyHostToDevice, e->s));
        TRY(cudaEventRecord(s->searched[0], e->s));
        TRY(luma_u16(f, W, H, s->yr, e->s));
        TRY(gauss_levels(s->yr, W, H, s->pr, e->s));
    } else {
        bool freem[8];
        free_mask(s, freem);
        // the target on the side stream, once its buffer's last reader on s is done
        const int b = i & 1;
        float* yt = s->yt2[b];
        const std::vector<float*>& pt = s->pt2[b];
        TRY(cudaStreamWaitEvent(e->bs, s->tfree[b], 0));
        TRY(cudaStreamWaitEvent(e->bs, s->copied[i], 0));
        TRY(luma_u16(f, W, H, yt, e->bs));
        TRY(gauss_levels(yt, W, H, pt, e->bs));
        TRY(cudaEventRecord(s->tdone[b], e->bs));
        TRY(cudaStreamWaitEvent(e->s, s->tdone[b], 0));
        TRY(multiscale_align_chain(C, s->yr, s->pr, yt, pt, W, H, s->sims_dev + 8 * (size_t)(i - 1), freem, (int)s->ap.coarsen,
                                   s->sims_dev + 8 * (size_t)i, s->warp_dev, s->evals_dev));
        TRY(cudaEventRecord(s->searched[i], e->s));
        if (i + 1 < n) {
            TRY(warp_plane_dev(yt, W, H, s->warp_dev, (int)s->ap.interp, s->yr, e->s));
            TRY(gauss_levels(s->yr, W, H, s->pr, e->s));
        }
        TRY(cudaEventRecord(s->tfree[b], e->s));
    }
    s->aligned_upto = i + 1;
    return nullptr;
}

// Queues the registration of the frames not yet registered; a chained
// registration then finishes in stream_warps and align_finish.
static char* run_align(lsb_stack* s) {
    if (chained(s)) {
        // the side stream reads frames the work stream may have written (a device-side fill)
        TRY(cudaEventRecord(s->e->s_mark, s->e->s));
        TRY(cudaStreamWaitEvent(s->e->bs, s->e->s_mark, 0));
        for (int i = s->aligned_upto; i < (int)s->count; i++)
            if (char* er = align_frame(s, i)) return er;
        return nullptr;
    }
    return run_align_host(s);
}

// The chained registration's end: its status and evaluation count.
static char* align_finish(lsb_stack* s) {
    size_t evals = 0;
    const cudaError_t ce = align_chain_end(s->e->actx, s->evals_dev, &evals);
    if (ce == cudaErrorLaunchTimeout) {  // the search's bounded wait ran out (no fault: the kernel returned)
        s->search_timed_out = true;
        return dup_err("the device search's hand-off wait ran out");
    }
    TRY(ce);
    s->align_evals = evals;
    s->aligned_upto = 0;  // a later run registers the frames again
    return nullptr;
}

// One level's fold arguments (halo control and timing events aside): every
// frame's REDUCE and the selection.
static FoldArgs level_args(const lsb_stack* s, int l, bool warped, bool depth_on, bool* focus, int* src) {
    FoldArgs a{};
    const int n = (int)s->count;
    a.level = l;
    a.nframes = n;
    a.red_k0 = 0;
    a.red_n = n;
    a.select = 1;
    a.sel_k0 = 0;
    a.sel_k1 = n;
    a.W = s->lw[l];
    a.H = s->lh[l];
    a.W1 = s->lw[l + 1];
    a.H1 = s->lh[l + 1];
    a.tiles_x = (a.W + 63) / 64;
    a.tiles_y = (a.H + 31) / 32;
    a.ntiles = a.tiles_x * a.tiles_y;
    a.src_u16 = warped && s->storage != STORE_F32 ? (const uint16_t*)s->warped : s->frames;
    a.src_f32 = warped && s->storage == STORE_F32 ? (const float*)s->warped : s->frames_f32;
    a.xf = s->xf_dev;
    a.interp = (int)s->ap.interp;
    a.src_g = l > 0 ? s->g[l] : nullptr;
    a.dst_g = s->g[l + 1];
    a.acc = s->acc[l];
    a.best = s->best[l];
    a.winner = l == s->depth_level ? s->winner : nullptr;
    a.use_chroma = (int)s->fp.use_chroma;
    a.status = s->status;
    a.no_fused = (s->e->cfg.flags & LSB_FLAG_TWO_KERNEL_FOLD0) != 0;
    *focus = depth_on && l == 0;
    if (*focus) {
        a.slice = s->slices;
        a.dw = s->dw;
        a.dh = s->dh;
        a.bk = s->bk;
        a.focus_kind = (int)s->dp.focus;
        a.sml_step = (int)s->dp.sml_step;
        a.ntaps = (int)focus_taps(s->dp.r_in, s->dp.r_out).size() / 3;
        a.rdf13 = s->dp.focus == 0 && s->dp.r_in == 1 && s->dp.r_out == 3;
    }
    *src = l > 0 ? SRC_G : ((s->f32src || (warped && s->storage == STORE_F32)) ? SRC_F32 : SRC_U16);
    return a;
}

// Levels with too few tiles to fill the GPU: the frames of the selection
// split into groups selected side by side, then merged in order (about 1.5
// work items per block, each group at least 2 frames; the first group resumes
// the state of the frames before, if any).
static void set_groups(const lsb_stack* s, FoldArgs& a) {
    const lsb_engine* e = s->e;
    const int gl = e->grid_select > 0 ? e->grid_select : e->grid;
    const size_t np = (size_t)a.W * a.H;
    int G = std::min((3 * gl / 2 + a.ntiles - 1) / std::max(a.ntiles, 1), std::max(1, (a.sel_k1 - a.sel_k0) / 2));
    while (G > 1 && (size_t)G * 5 * np > s->gsel_floats) G--;
    if (G > 1) {
        a.sel_groups = G;
        a.gacc = s->gsel;
        a.gbest = s->gsel + (size_t)G * 3 * np;
        a.gwin = (int*)(s->gsel + (size_t)G * 4 * np);
    }
}

// Each frame's warp (align.rs:489, stack.rs:662-679) and brightness sums
// (brightness.rs:67) as soon as its search is done, while the chain goes on:
// the transforms come back on rs behind each search, their matrices are
// built on the host (align.rs:200-294, as the host path builds them) and the
// frame's warp and sums are queued on ws, then its gains (brightness.rs:93)
// and, with `reduce` alone, the REDUCE of every pyramid level (pyramid.rs:86,
// the focus slice at level 0): all that depends on that frame alone. With
// `select` too, every SEL_CHUNK frames are folded in level by level, their
// REDUCE then their selection (fuse.rs:414-451, frames in order, resuming
// from the state the chunk before left). The work stream waits for ws.
static char* stream_warps(lsb_stack* s, bool pushed, bool reduce, bool select) {
    lsb_engine* e = s->e;
    const int W = (int)s->w, H = (int)s->h, n = (int)s->count;
    const size_t np = (size_t)W * H;
    const bool u16out = s->storage != STORE_F32, bright = s->brightness && n >= 2;
    const bool depth_on = s->dp.enabled != 0;
    if (depth_on && s->dp.focus == 0) {
        std::vector<float> taps = focus_taps(s->dp.r_in, s->dp.r_out);
        TRY(set_focus_taps(taps.data(), (int)(taps.size() / 3), e->ws));
    }
    TRY(cudaMemsetAsync(s->status, 0, sizeof(int), e->ws));
    int sel_from = 0;
    for (int i = 0; i < n; i++) {
        TRY(cudaStreamWaitEvent(e->rs, s->searched[i], 0));
        TRY(cudaMemcpyAsync(s->sims_pin + 8 * (size_t)i, s->sims_dev + 8 * (size_t)i, sizeof(double) * 8, cudaMemcpyDeviceToHost, e->rs));
        TRY(cudaEventRecord(s->sims_back[i], e->rs));
    }
    for (int i = 0; i < n; i++) {
        TRY(cudaEventSynchronize(s->sims_back[i]));
        double* sim = &s->sims[8 * (size_t)i];
        memcpy(sim, s->sims_pin + 8 * (size_t)i, sizeof(double) * 8);
        FrameXform& X = s->xf_pin[i];
        X = FrameXform{};
        X.warp = !sim_is_id(sim);
        double m[9];
        sim_matrix(sim, W, H, m);
        if (X.warp) mat_inverse(m, X.inv);
        X.affine = X.inv[6] == 0.0 && X.inv[7] == 0.0 && X.inv[8] == 1.0;
        for (int c = 0; c < 3; c++) X.gain[c] = 1.f;  // frame_gain sets them when brightness is on
        X.gscale = 65535.f;
        X.ginv = (float)(1.0 / 65535.0);
        TRY(cudaMemcpyAsync(s->xf_dev + i, &X, sizeof X, cudaMemcpyHostToDevice, e->ws));
        void* out = u16out ? (void*)((uint16_t*)s->warped + (size_t)i * np * 3) : (void*)((float*)s->warped + (size_t)i * np * 3);
        TRY(warp_frames(s->frames + (size_t)i * np * 3, s->xf_dev + i, (int)s->ap.interp, W, H, 1, u16out, out, e->ws));
        if (bright && i >= 1) {
            BrightXform& B = s->bx_pin[i];
            mat_inverse(m, B.inv);
            B.ident = sim_is_id(sim);
            B.affine = B.inv[6] == 0.0 && B.inv[7] == 0.0 && B.inv[8] == 1.0;
            TRY(cudaMemcpyAsync(s->bx_dev + i, &B, sizeof B, cudaMemcpyHostToDevice, e->ws));
            // one short block per part: on the low-priority stream, freed SMs go to the chain's search first
            TRY(bright_sums_frame(s->frames, i, W, H, s->bx_dev, (int)s->ap.interp, BRIGHT_PARTS, s->bpart, BRIGHT_PARTS, e->ws));
            TRY(frame_gain(s->bpart, i, BRIGHT_PARTS, s->xf_dev + i, e->ws));
        }
        for (int l = 0; l < s->levels && reduce && !select; l++) {
            bool focus = false;
            int src = 0;
            FoldArgs a = level_args(s, l, true, depth_on, &focus, &src);
            a.red_k0 = i;
            a.red_n = 1;
            a.select = 0;
            TRY(fold_level(a, src, s->storage, (int)s->fp.energy_radius, focus, e->ws, e->grid));
        }
        // chunks of SEL_CHUNK frames, the stack's last SEL_TAIL frames a chunk of their own: what is left
        // to fold once the last frame lands is small
        const bool cut = i + 1 - sel_from == SEL_CHUNK || i + 1 == n || (n > 2 * SEL_TAIL && i + 1 == n - SEL_TAIL);
        if (reduce && select && cut) {
            // the chunk's frames level by level: their REDUCE (and focus slices), then their selection
            // (level 0: one fused kernel where it applies), beside the registration chain: one
            // persistent CTA per SM, so that the chain's cooperative search keeps room on every SM;
            // the last chunk, after the chain, on the whole GPU
            const int ch = s->chunks;
            const bool last = i + 1 == n;
            for (int l = 0; l < s->levels; l++) {
                bool focus = false;
                int src = 0;
                FoldArgs a = level_args(s, l, true, depth_on, &focus, &src);
                a.red_k0 = sel_from;
                a.red_n = i + 1 - sel_from;
                a.sel_k0 = sel_from;
                a.sel_k1 = i + 1;
                a.beside = last ? 0 : 1;
                set_groups(s, a);
                if (l == 0) {  // the level-0 fold of the chunk, timed: [start, after the fused kernel, end]
                    TRY(cudaEventRecord(s->chunk_ev[3 * ch], e->ws));
                    TRY(cudaEventRecord(s->chunk_ev[3 * ch + 1], e->ws));
                    a.after_fused = s->chunk_ev[3 * ch + 1];
                }
                TRY(fold_level(a, src, s->storage, (int)s->fp.energy_radius, focus, e->ws, last ? e->grid : e->sms));
                if (l == 0) TRY(cudaEventRecord(s->chunk_ev[3 * ch + 2], e->ws));
            }
            s->chunks = ch + 1;
            sel_from = i + 1;
        }
    }
    TRY(cudaEventRecord(s->wdone, e->ws));
    TRY(cudaStreamWaitEvent(e->s, s->wdone, 0));
    return nullptr;
}

static char* run_align_host(lsb_stack* s) {
    lsb_engine* e = s->e;
    const int W = (int)s->w, H = (int)s->h, n = (int)s->count;
    AlignCtx& C = e->actx;
    C.evals = 0;
    bool freem[8];
    {
        bool aff = s->ap.model != 0, proj = s->ap.model == 2;
        bool m[8] = {s->ap.shift != 0, s->ap.shift != 0, s->ap.scale != 0, s->ap.rotation != 0, aff, aff, proj, proj};
        memcpy(freem, m, sizeof m);
    }
    for (int i = 0; i < n; i++) {
        const uint16_t* f = s->frames + (size_t)i * W * H * 3;
        double* sim = &s->sims[8 * (size_t)i];
        const double id[8] = {0, 0, 1, 0, 1, 0, 0, 0};
        memcpy(sim, id, sizeof id);
        TRY(luma_u16(f, W, H, s->yt, e->s));
        if (i > 0) {
            TRY(gauss_levels(s->yt, W, H, s->pt, e->s));
            C.device_search = s->ap.host_search ? 0 : e->coop;
            TRY(multiscale_align(C, s->yr, s->pr, s->yt, s->pt, W, H, &s->sims[8 * (size_t)(i - 1)], freem, (int)s->ap.coarsen, sim));
        }
        if (i + 1 < n) {
            // the next frame's reference: this frame's luma as aligned (stack.rs:527)
            if (sim_is_id(sim)) {
                TRY(cudaMemcpyAsync(s->yr, s->yt, sizeof(float) * W * H, cudaMemcpyDeviceToDevice, e->s));
            } else {
                WarpXform wx;
                double m[9];
                sim_matrix(sim, W, H, m);
                mat_inverse(m, wx.inv);
                wx.affine = wx.inv[6] == 0.0 && wx.inv[7] == 0.0 && wx.inv[8] == 1.0;
                wx.interp = (int)s->ap.interp;
                TRY(warp_plane(s->yt, W, H, wx, s->yr, e->s));
            }
            TRY(gauss_levels(s->yr, W, H, s->pr, e->s));
        }
    }
    s->align_evals = C.evals;
    return nullptr;
}

// brightness.rs:93 `ratio`
static void bratio(const double ref[3], const double frame[3], size_t n, float g[3]) {
    for (int c = 0; c < 3; c++) {
        if (n < 64) {
            g[c] = 1.0f;
            continue;
        }
        float v = frame[c] > 1e-9 ? (float)(ref[c] / frame[c]) : 1.0f;
        g[c] = std::min(std::max(v, 0.25f), 4.0f);
    }
}

static char* run_gains(lsb_stack* s, bool aligned) {
    lsb_engine* e = s->e;
    const int W = (int)s->w, H = (int)s->h, n = (int)s->count;
    for (int k = 0; k < n; k++)
        for (int c = 0; c < 3; c++) s->gains[3 * k + c] = 1.f;
    if (!s->brightness || n < 2 || s->f32src) return nullptr;
    if (aligned) {
        std::vector<BrightXform> bx(n);
        for (int k = 0; k < n; k++) {
            double m[9];
            sim_matrix(&s->sims[8 * (size_t)k], W, H, m);
            mat_inverse(m, bx[k].inv);
            bx[k].ident = sim_is_id(&s->sims[8 * (size_t)k]);
            bx[k].affine = bx[k].inv[6] == 0.0 && bx[k].inv[7] == 0.0 && bx[k].inv[8] == 1.0;
        }
        TRY(cudaMemcpyAsync(s->bx_dev, bx.data(), sizeof(BrightXform) * n, cudaMemcpyHostToDevice, e->s));
        TRY(bright_sums(s->frames, n, W, H, s->bx_dev, (int)s->ap.interp, BRIGHT_PARTS, s->bpart, e->s));
        std::vector<double> part((size_t)n * BRIGHT_PARTS * 7);
        TRY(cudaMemcpyAsync(part.data(), s->bpart, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, e->s));
        TRY(cudaStreamSynchronize(e->s));
        for (int k = 1; k < n; k++) {
            double sm[7] = {0, 0, 0, 0, 0, 0, 0};
            for (int p = 0; p < BRIGHT_PARTS; p++)
                for (int q = 0; q < 7; q++) sm[q] += part[((size_t)k * BRIGHT_PARTS + p) * 7 + q];
            double sf[3] = {sm[0], sm[1], sm[2]}, so[3] = {sm[3], sm[4], sm[5]};
            bratio(so, sf, (size_t)sm[6], &s->gains[3 * (size_t)k]);
        }
    } else {
        // stack.rs LazyFrames: gains_to(means(frame 0), frame)
        TRY(frame_means(s->frames, n, W, H, s->mpart, 64, s->means, e->s));
        std::vector<double> m((size_t)n * 3);
        TRY(cudaMemcpyAsync(m.data(), s->means, sizeof(double) * m.size(), cudaMemcpyDeviceToHost, e->s));
        TRY(cudaStreamSynchronize(e->s));
        for (int k = 1; k < n; k++) bratio(&m[0], &m[3 * (size_t)k], (size_t)-1, &s->gains[3 * (size_t)k]);
    }
    return nullptr;
}

static float ms_between(cudaEvent_t a, cudaEvent_t b) {
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    return t;
}

static void common_area(const std::vector<double>& sims, int n, int w, int h, int interp, uint32_t rect[4]);
static char* run_pipeline_once(lsb_stack* s);
// The pipeline, with one guard: if the device search's bounded wait runs out
// (its cooperative blocks could not all be resident in time), the work queued
// from its transforms is drained and the stack is registered again by the
// host-driven search, which takes the same branches (same transforms and
// evaluation count), then folded as usual.
static char* run_pipeline(lsb_stack* s) {
    s->search_timed_out = false;
    char* err = run_pipeline_once(s);
    if (!err || !s->search_timed_out) return err;
    lsb_free_str(err);
    lsb_engine* e = s->e;
    e->log("registration: the device search's wait ran out; registering again with the host-driven search");
    for (cudaStream_t q : {e->s, e->cs, e->bs, e->rs, e->ws}) TRY(cudaStreamSynchronize(q));
    TRY(cudaMemsetAsync(e->actx.nm_ctl, 0, sizeof(int) * 4, e->s));
    const auto hs = s->ap.host_search;
    s->ap.host_search = 1;
    s->aligned_upto = 0;
    err = run_pipeline_once(s);
    s->ap.host_search = hs;
    return err;
}
static char* run_pipeline_once(lsb_stack* s) {
    lsb_engine* e = s->e;
    cudaStream_t st = e->s;
    const int W = (int)s->w, H = (int)s->h, n = (int)s->count;
    if (n == 0) return dup_err("no frames pushed");
    const bool aligned = s->ap.enabled && n > 1 && !s->f32src;
    cudaEvent_t* ev = e->ev;
    TRY(cudaEventRecord(ev[0], st));
    // Frames registered as they were pushed: the GPU waits on the host copies, so the REDUCEs
    // fill that time too. Frames already on the device: the REDUCEs would only slow the chain.
    const bool pushed = s->aligned_upto > 0;
    if (aligned) {
        char* err = run_align(s);
        if (err) return err;
    }
    TRY(cudaEventRecord(ev[1], st));
    const bool streamed = aligned && chained(s);
    // the fold too, chunk by chunk beside the chain, for pushed frames (not with halo control): the GPU
    // waits on the host copies anyway. Frames already in device memory fold after the chain unless
    // LSB_FLAG_FOLD_BESIDE_CHAIN asks otherwise: beside it (one fold CTA per SM) the fold ran at half its
    // speed and the chain slowed, 572 ms against 530 ms for the C3 step.
    const bool sel_streamed = streamed && !(s->fp.halo > 0.f) && (pushed || (e->cfg.flags & LSB_FLAG_FOLD_BESIDE_CHAIN));
    s->chunks = 0;
    if (streamed) {
        char* err = stream_warps(s, pushed, pushed || sel_streamed, sel_streamed);
        if (!err) err = align_finish(s);
        if (err) return err;
    }
    if (streamed) {
        // the transforms, gains and scales the streamed work used
        s->xf.assign(n, FrameXform{});
        TRY(cudaMemcpy(s->xf.data(), s->xf_dev, sizeof(FrameXform) * n, cudaMemcpyDeviceToHost));
        for (int k = 0; k < n; k++)
            for (int c = 0; c < 3; c++) s->gains[3 * (size_t)k + c] = s->xf[k].gain[c];
    } else {
        char* err = run_gains(s, aligned);
        if (err) return err;
    }
    // align.rs:344 the common area, on a host thread (the transforms are known) while the GPU goes on;
    // the future's destructor waits for it on every way out of this function
    s->crop_rect[0] = 0;
    s->crop_rect[1] = 0;
    s->crop_rect[2] = s->w;
    s->crop_rect[3] = s->h;
    std::future<void> crop_job;
    if (aligned && s->crop)
        crop_job = std::async(std::launch::async, [s, n, W, H] { common_area(s->sims, n, W, H, (int)s->ap.interp, s->crop_rect); });
    // per-frame level-0 transforms
    if (!streamed) s->xf.assign(n, FrameXform{});
    for (int k = 0; k < n && !streamed; k++) {
        FrameXform& X = s->xf[k];
        const double* sim = &s->sims[8 * (size_t)k];
        X.warp = aligned && !sim_is_id(sim);
        if (X.warp) {
            double m[9];
            sim_matrix(sim, W, H, m);
            mat_inverse(m, X.inv);
        }
        X.affine = X.inv[6] == 0.0 && X.inv[7] == 0.0 && X.inv[8] == 1.0;
        X.gain_on = 0;
        float maxg = 1.f;
        for (int c = 0; c < 3; c++) {
            X.gain[c] = s->gains[3 * (size_t)k + c];
            if (fabsf(X.gain[c] - 1.0f) > 1e-6f) X.gain_on |= 1 << c;
            maxg = std::max(maxg, X.gain[c]);
        }
        // the frame's fixed-point levels span [0, its largest gain]: each is a convex
        // combination of its gained inputs in [0, 1]
        if (s->f32src) maxg = 1.f;
        X.gscale = (float)(65535.0 / maxg);
        X.ginv = (float)(maxg / 65535.0);
    }
    if (!streamed) TRY(cudaMemcpyAsync(s->xf_dev, s->xf.data(), sizeof(FrameXform) * n, cudaMemcpyHostToDevice, st));
    // the aligned frames, written once (align.rs:489 with stack.rs:668's fallback); the fold reads them
    const bool warped = aligned;
    if (warped && !streamed) TRY(warp_frames(s->frames, s->xf_dev, (int)s->ap.interp, W, H, n, s->storage != STORE_F32, s->warped, st));
    if (!streamed) TRY(cudaMemsetAsync(s->status, 0, sizeof(int), st));  // else stream_warps cleared it
    TRY(cudaEventRecord(ev[2], st));
    // ---- the fold, level by level over all frames
    const bool depth_on = s->dp.enabled != 0;
    if (depth_on && s->dp.focus == 0) {
        std::vector<float> taps = focus_taps(s->dp.r_in, s->dp.r_out);
        TRY(set_focus_taps(taps.data(), (int)(taps.size() / 3), st));
    }
    // fuse.rs:120 halo_guide: the guide level and the hardness, when on (fuse.rs:112 HALO_MAX = 8)
    const bool halo = s->fp.halo > 0.f;
    const int guide = std::min((int)s->fp.depth_level, s->levels - 1);
    if (halo && s->halo_w.empty()) {
        s->halo_w.assign(s->levels + 1, nullptr);
        for (int l = guide; l <= s->levels; l++) TRY(s->pool.get(&s->halo_w[l], (size_t)s->n * s->lw[l] * s->lh[l]));
    }
    if (sel_streamed)  // the level-0 timings of a fold that ran on ws: none here
        for (int q : {8, 10, 9}) TRY(cudaEventRecord(ev[q], st));
    for (int l = 0; l < s->levels && !sel_streamed; l++) {
        bool focus = false;
        int src = 0;
        FoldArgs a = level_args(s, l, warped, depth_on, &focus, &src);
        if (streamed && pushed) a.red_n = 0;  // stream_warps has REDUCEd every frame
        if (!(halo && l >= guide)) set_groups(s, a);
        if (halo && l >= guide) {
            a.halo_mode = l == guide ? 1 : 2;
            a.halo_p = std::min(s->fp.halo, 8.0f);
            a.halo_w = s->halo_w[l];
            if (l > guide) TRY(reduce_weights(s->halo_w[l - 1], s->lw[l - 1], s->lh[l - 1], n, s->halo_w[l], s->lw[l], s->lh[l], st));
        }
        a.between = l == 0 ? ev[10] : nullptr;
        if (l == 0) TRY(cudaEventRecord(ev[8], st));
        TRY(fold_level(a, src, s->storage, (int)s->fp.energy_radius, focus, st, e->grid_select > 0 ? e->grid_select : e->grid));
        if (l == 0) TRY(cudaEventRecord(ev[9], st));
    }
    TRY(cudaEventRecord(ev[3], st));
    // ---- residual, collapse
    {
        const int wt = s->lw[s->levels], ht = s->lh[s->levels];
        const int r = (int)s->fp.top_radius, nwin = (2 * r + 1) * (2 * r + 1);
        std::vector<float> lnp(128, 0.f);
        const float inv_n = 1.0f / (float)nwin;
        for (int c = 1; c <= nwin; c++) lnp[c] = logf((float)c * inv_n);
        TRY(cudaMemcpyAsync(s->lnp, lnp.data(), sizeof(float) * 128, cudaMemcpyHostToDevice, st));
        if (halo) {
            // fuse.rs:453-475 below the guide, fuse.rs:505-510 the weighted means
            const int L = s->levels;
            TRY(reduce_weights(s->halo_w[L - 1], s->lw[L - 1], s->lh[L - 1], n, s->halo_w[L], wt, ht, st));
            TRY(halo_top(s->g[L], s->storage, s->xf_dev, s->halo_w[L], n, wt, ht, s->top, s->dev_s, st));
            TRY(halo_divide(s->top, s->dev_s, wt, ht, st));
            for (int l = guide + 1; l < L; l++) TRY(halo_divide(s->acc[l], s->best[l], s->lw[l], s->lh[l], st));
        } else {
            ResidualArgs ra{s->g[s->levels], n, wt, ht, (int)s->fp.top_rule, r, (int)s->fp.entropy_bins, s->dev_s, s->ent_s, s->top, s->xf_dev};
            TRY(fuse_residuals(ra, s->storage, s->lnp, st));
        }
        const float* coarse = s->top;
        for (int l = s->levels - 1; l >= 0; l--) {
            // even levels land in img, odd ones in img_tmp: a level never overwrites its coarser input
            float* out = (l % 2 == 0) ? s->img : s->img_tmp;
            TRY(collapse_level(s->acc[l], coarse, out, s->lw[l], s->lh[l], s->lw[l + 1], s->lh[l + 1], l == 0, s->img_u16, st));
            coarse = out;
        }
    }
    TRY(cudaEventRecord(ev[4], st));
    s->folded = true;
    if (lsb_result* r = s->early) {
        // the fused planes and the winner map go back on rs while the depth pass runs on s
        const int dl = s->depth_level;
        if (!s->winner_full) TRY(s->pool.get(&s->winner_full, (size_t)W * H));
        if (!s->fused_ev) TRY(cudaEventCreateWithFlags(&s->fused_ev, cudaEventDisableTiming));
        TRY(upsample_index(s->winner, s->lw[dl], s->lh[dl], 1 << dl, W, H, s->winner_full, st));
        TRY(cudaEventRecord(s->fused_ev, st));
        TRY(cudaStreamWaitEvent(e->rs, s->fused_ev, 0));
        const size_t np = (size_t)W * H;
        TRY(cudaMemcpyAsync(r->image_u16, s->img_u16, sizeof(uint16_t) * 3 * np, cudaMemcpyDeviceToHost, e->rs));
        TRY(cudaMemcpyAsync(r->image_f32, s->img, sizeof(float) * 3 * np, cudaMemcpyDeviceToHost, e->rs));
        TRY(cudaMemcpyAsync(r->winner, s->winner_full, sizeof(float) * np, cudaMemcpyDeviceToHost, e->rs));
    }
    // ---- depth
    if (depth_on) {
        const int k = s->bk, dw = s->dw, dh = s->dh;
        const size_t m = (size_t)dw * dh;
        TRY(luma_and_guide(s->img, W, H, k, s->yfull, s->guide, dw, dh, st));
        if (s->dp.agg_radius > 0) gf_stats(s->guide, dw, dh, (int)s->dp.agg_radius, s->tmp, s->mi, s->vi, st);
        AggArgs ag{s->slices, n, dw, dh, (int)s->dp.agg_radius, s->dp.agg_eps, s->guide, s->mi, s->vi, s->state, 0, 0};
        TRY(aggregate_peaks(ag, s->storage != STORE_F32, st, e->grid_agg > 0 ? e->grid_agg : e->grid,
                            !(e->cfg.flags & LSB_FLAG_DIRECT_WINDOW_SUMS)));
        TRY(cudaEventRecord(ev[5], st));
        const size_t cnt = (m + 6) / 7;
        TRY(select_kth(s->state + 7 * m, cnt, 7, cnt / 2, e->hist, e->sel, e->scal + 0, st));
        TRY(peak_finish(s->state, m, n, e->scal + 0, s->dp.gate, s->draw, s->conf, s->mins, st));
        if (s->dp.median) TRY(median3(s->draw, s->dmed, dw, dh, st));
        else TRY(cudaMemcpyAsync(s->dmed, s->draw, sizeof(float) * m, cudaMemcpyDeviceToDevice, st));
        TRY(select_kth(s->conf, cnt, 7, std::min(cnt * 9 / 10, cnt - 1), e->hist, e->sel, e->scal + 1, st));
        TRY(conf_scale(s->conf, m, e->scal + 1, st));
        s->iters = s->iters_first = 0;
        s->rel = 0.f;
        s->rel64 = 0.0;
        const float* dsol = s->dmed;
        TRY(cudaEventRecord(ev[11], st));
        if (s->dp.lambda > 0.f) {
            cudaError_t ce;
            WlsSolver* ws = stack_solver(s, dw, dh, s->dp, st, &ce);
            if (ce != cudaSuccess) return dup_err(fmt("wls: %s", cudaGetErrorString(ce)));
            bool given = false;
            cudaError_t r1 = warm_start(s, dw, dh, n, st, &given);
            auto start = [&]() {
                return given ? cudaMemcpyAsync(s->u, s->x0, sizeof(float) * m, cudaMemcpyDeviceToDevice, st) : cudaSuccess;
            };
            if (r1 == cudaSuccess) r1 = wls_set_weights(ws, s->conf, st);
            float rel = 0.f;
            int it = 0;
            if (r1 == cudaSuccess) r1 = start();
            if (r1 == cudaSuccess) r1 = wls_solve(ws, s->dmed, (int)s->dp.cg_iters, s->u, &rel, &it, st, (int)s->dp.vcycle_mode, given, &s->rel64);
            s->iters_first = it;
            if (r1 == cudaSuccess && s->dp.robust > 0.f) {
                r1 = robust_weights(s->conf, s->dmed, s->u, s->dp.robust, s->w2, m, st);
                if (r1 == cudaSuccess) r1 = wls_set_weights(ws, s->w2, st);
                if (r1 == cudaSuccess) r1 = start();
                if (r1 == cudaSuccess) r1 = wls_solve(ws, s->dmed, (int)s->dp.cg_iters, s->u, &rel, &it, st, (int)s->dp.vcycle_mode, given, &s->rel64);
            }
            if (r1 != cudaSuccess) return dup_err(fmt("wls: %s", cudaGetErrorString(r1)));
            s->rel = rel;
            s->iters = it;
            dsol = s->u;
        }
        TRY(cudaEventRecord(ev[6], st));
        const float max_d = (float)(n - 1);
        if (s->dp.upsample == 1) {
            gf_stats(s->guide, dw, dh, (int)s->dp.up_radius, s->tmp, s->mi, s->vi, st);
            gf_coeffs(s->guide, s->mi, s->vi, dsol, dw, dh, (int)s->dp.up_radius, s->dp.up_eps, s->t0, s->t1, s->t2, s->tmp, s->abar,
                      s->bbar, st);
            TRY(upsample(s->abar, s->bbar, s->yfull, s->guide, s->conf, W, H, dw, dh, k, max_d, true, s->dfull, s->cfull, st));
        } else {
            TRY(upsample(nullptr, dsol, s->yfull, s->guide, s->conf, W, H, dw, dh, k, max_d, false, s->dfull, s->cfull, st));
        }
    } else {
        TRY(cudaEventRecord(ev[5], st));
        TRY(cudaEventRecord(ev[11], st));
        TRY(cudaEventRecord(ev[6], st));
    }
    TRY(cudaEventRecord(ev[7], st));
    TRY(cudaEventSynchronize(ev[7]));
    if (crop_job.valid()) crop_job.get();
    int status = 0;
    TRY(cudaMemcpy(&status, s->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status) return dup_err(fmt("device status 0x%x (a kernel met a shape it was not built for)", status));
    if (depth_on) {
        float sc[2];
        TRY(cudaMemcpy(sc, e->scal, sizeof sc, cudaMemcpyDeviceToHost));
        s->floor_v = sc[0];
        s->p90 = sc[1];
    }
    s->ms[0] = ms_between(ev[0], ev[1]);
    s->ms[1] = ms_between(ev[1], ev[2]);
    s->ms[2] = ms_between(ev[2], ev[3]);
    s->ms[3] = ms_between(ev[3], ev[4]);
    s->ms[4] = ms_between(ev[4], ev[5]);
    s->ms[5] = ms_between(ev[5], ev[6]);
    s->ms[6] = ms_between(ev[6], ev[7]);
    s->ms[7] = ms_between(ev[0], ev[7]);
    s->ms[8] = ms_between(ev[8], ev[9]);
    s->ms[9] = ms_between(ev[10], ev[9]);   // select, level 0
    s->ms[10] = ms_between(ev[8], ev[10]);  // REDUCE (+ focus slices), level 0
    s->ms[11] = ms_between(ev[11], ev[6]);  // the WLS solves (warm start included)
    if (sel_streamed) {  // the level-0 fold ran chunk by chunk on ws: the sums of its parts
        s->ms[8] = s->ms[9] = s->ms[10] = 0.0;
        for (int c = 0; c < s->chunks; c++) {
            s->ms[8] += ms_between(s->chunk_ev[3 * c], s->chunk_ev[3 * c + 2]);
            s->ms[10] += ms_between(s->chunk_ev[3 * c], s->chunk_ev[3 * c + 1]);
            s->ms[9] += ms_between(s->chunk_ev[3 * c + 1], s->chunk_ev[3 * c + 2]);
        }
    }
    return nullptr;
}

extern "C" char* lsb_stack_run(lsb_stack* s, double* ms_out12) {
    if (!s) return dup_err("null stack");
    char* err = run_pipeline(s);
    if (err) return err;
    if (ms_out12) memcpy(ms_out12, s->ms, sizeof s->ms);
    return nullptr;
}

// fuse.rs:315 from the device counts
static char* shares_of(lsb_stack* s, float* out) {
    const int dl = s->depth_level;
    const int cells = s->lw[dl] * s->lh[dl];
    TRY(winner_counts(s->winner, s->best[dl], cells, (int)s->count, s->counts, s->mx, s->e->s));
    std::vector<unsigned> c(s->count);
    TRY(cudaMemcpyAsync(c.data(), s->counts, sizeof(unsigned) * s->count, cudaMemcpyDeviceToHost, s->e->s));
    TRY(cudaStreamSynchronize(s->e->s));
    size_t total = 0;
    for (unsigned v : c) total += v;
    for (uint32_t k = 0; k < s->count; k++) out[k] = total > 0 ? (float)c[k] / (float)total : 0.0f;
    return nullptr;
}

extern "C" char* lsb_stack_shares(lsb_stack* s, float* out_n) {
    if (!s || !out_n) return dup_err("null argument");
    if (!s->folded) {
        char* err = run_pipeline(s);
        if (err) return err;
    }
    return shares_of(s, out_n);
}

// align.rs:344 `common_area` (host, on the transforms found)
static void common_area(const std::vector<double>& sims, int n, int w, int h, int interp, uint32_t rect[4]) {
    rect[0] = 0;
    rect[1] = 0;
    rect[2] = w;
    rect[3] = h;
    std::vector<std::array<double, 9>> invs;
    for (int k = 0; k < n; k++) {
        if (sim_is_id(&sims[8 * (size_t)k])) continue;
        double m[9];
        std::array<double, 9> inv;
        sim_matrix(&sims[8 * (size_t)k], w, h, m);
        mat_inverse(m, inv.data());
        invs.push_back(inv);
    }
    if (invs.empty()) return;
    const double mg = (double)((interp == 0 ? 1 : interp == 1 ? 2 : interp <= 3 ? 4 : 6) / 2);
    const double xmax = (double)(w - 1) - mg, ymax = (double)(h - 1) - mg;
    std::vector<std::pair<long, long>> rows;
    for (int y = 0; y < h; y++) {
        double lo = 0.0, hi = (double)(w - 1), yf = (double)y;
        for (auto& inv : invs) {
            double g = inv[6], d = inv[7] * yf + inv[8];
            if (d <= 0.0 || g * (double)(w - 1) + d <= 0.0) {
                lo = 1.0;
                hi = 0.0;
                break;
            }
            double A[2] = {inv[0], inv[3]}, K[2] = {inv[1] * yf + inv[2], inv[4] * yf + inv[5]};
            double smin[2] = {mg, mg}, smax[2] = {xmax, ymax};
            for (int ax = 0; ax < 2; ax++) {
                double a = A[ax], kk = K[ax];
                double pq[2][2] = {{a - smin[ax] * g, kk - smin[ax] * d}, {smax[ax] * g - a, smax[ax] * d - kk}};
                for (int t = 0; t < 2; t++) {
                    double p = pq[t][0], q = pq[t][1];
                    if (fabs(p) < 1e-12) {
                        if (q < 0.0) {
                            lo = 1.0;
                            hi = 0.0;
                        }
                    } else if (p > 0.0) {
                        lo = std::max(lo, -q / p);
                    } else {
                        hi = std::min(hi, -q / p);
                    }
                }
            }
        }
        rows.push_back(lo <= hi ? std::make_pair((long)ceil(lo), (long)floor(hi)) : std::make_pair(1L, 0L));
    }
    size_t bx = 0, by = 0, bw = 0, bh = 0;
    for (int y0 = 0; y0 < h; y0++) {
        long lo = rows[y0].first, hi = rows[y0].second;
        for (int y1 = y0; y1 < h; y1++) {
            lo = std::max(lo, rows[y1].first);
            hi = std::min(hi, rows[y1].second);
            if (lo > hi) break;
            size_t rw = (size_t)(hi - lo + 1), rh = (size_t)(y1 - y0 + 1);
            if (rw * rh > bw * bh) {
                bx = (size_t)lo;
                by = (size_t)y0;
                bw = rw;
                bh = rh;
            }
        }
    }
    if (bw * bh > 0) {
        rect[0] = (uint32_t)bx;
        rect[1] = (uint32_t)by;
        rect[2] = (uint32_t)bw;
        rect[3] = (uint32_t)bh;
    }
}

// Page-locked host blocks for the large result planes: the device -> host
// copies run at the link's speed, and a freed result's blocks serve the next
// result of the same size instead of being pinned again (at most
// HB_CACHE_BYTES are kept unused).
static std::mutex g_hb_mu;
static std::multimap<size_t, void*> g_hb_free;
static std::unordered_map<void*, size_t> g_hb_size;
static size_t g_hb_cached = 0;
constexpr size_t HB_CACHE_BYTES = (size_t)8 << 30;
static void* hb_get(size_t bytes) {
    {
        std::lock_guard<std::mutex> lk(g_hb_mu);
        auto it = g_hb_free.find(bytes);
        if (it != g_hb_free.end()) {
            void* p = it->second;
            g_hb_free.erase(it);
            g_hb_cached -= bytes;
            return p;
        }
    }
    void* p = nullptr;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return malloc(bytes);  // pageable: slower copies, same results
    }
    std::lock_guard<std::mutex> lk(g_hb_mu);
    g_hb_size[p] = bytes;
    return p;
}
static void hb_release(void* p) {
    if (!p) return;
    {
        std::lock_guard<std::mutex> lk(g_hb_mu);
        auto it = g_hb_size.find(p);
        if (it != g_hb_size.end()) {
            if (g_hb_cached + it->second <= HB_CACHE_BYTES) {
                g_hb_free.emplace(it->second, p);
                g_hb_cached += it->second;
                return;
            }
            g_hb_size.erase(it);
        } else {
            free(p);
            return;
        }
    }
    cudaFreeHost(p);
}

// lsb_stack_finish's body: every error return leaves the caller to free r.
static char* stack_finish(lsb_stack* s, lsb_result* r) {
    const size_t W = s->w, H = s->h;
    cudaStream_t st = s->e->s;
    r->image_u16 = (uint16_t*)hb_get(sizeof(uint16_t) * 3 * W * H);
    r->image_f32 = (float*)hb_get(sizeof(float) * 3 * W * H);
    r->winner = (float*)hb_get(sizeof(float) * W * H);
    if (!r->image_u16 || !r->image_f32 || !r->winner) return dup_err("out of host memory");
    if (s->dp.enabled) {  // page-locked, so that every copy back is asynchronous
        r->depth = (float*)hb_get(sizeof(float) * W * H);
        r->conf = (float*)hb_get(sizeof(float) * W * H);
        r->floor_cells = (float*)hb_get(sizeof(float) * (size_t)s->dw * s->dh);
        if (!r->depth || !r->conf || !r->floor_cells) return dup_err("out of host memory");
    }
    s->early = r;  // run_pipeline sends the fused planes back as soon as they exist
    char* err = run_pipeline(s);
    s->early = nullptr;
    if (err) return err;
    const size_t N = s->count;
    r->w = s->w;
    r->h = s->h;
    r->n_frames = s->count;
    r->levels = s->levels;
    r->sims = (double*)malloc(sizeof(double) * 8 * N);
    r->gains = (float*)malloc(sizeof(float) * 3 * N);
    r->shares = (float*)malloc(sizeof(float) * N);
    if (!r->sims || !r->gains || !r->shares) return dup_err("out of host memory");
    if (s->dp.enabled) {
        const size_t m = (size_t)s->dw * s->dh;
        r->dw = s->dw;
        r->dh = s->dh;
        TRY(cudaMemcpyAsync(r->depth, s->dfull, sizeof(float) * W * H, cudaMemcpyDeviceToHost, st));
        TRY(cudaMemcpyAsync(r->conf, s->cfull, sizeof(float) * W * H, cudaMemcpyDeviceToHost, st));
        TRY(cudaMemcpyAsync(r->floor_cells, s->mins, sizeof(float) * m, cudaMemcpyDeviceToHost, st));
    }
    TRY(cudaStreamSynchronize(st));
    TRY(cudaStreamSynchronize(s->e->rs));
    memcpy(r->sims, s->sims.data(), sizeof(double) * 8 * N);
    memcpy(r->gains, s->gains.data(), sizeof(float) * 3 * N);
    err = shares_of(s, r->shares);
    if (err) return err;
    memcpy(r->crop, s->crop_rect, sizeof s->crop_rect);
    r->floor_value = s->floor_v;
    r->p90 = s->p90;
    r->wls_rel = s->rel;
    r->wls_rel64 = s->rel64;
    r->wls_iters = s->iters;
    r->wls_iters_first = s->iters_first;
    r->align_evals = (uint32_t)s->align_evals;
    memcpy(r->ms, s->ms, sizeof s->ms);
    return nullptr;
}

extern "C" char* lsb_stack_finish(lsb_stack* s, lsb_result* r) {
    if (!s || !r) return dup_err("null argument");
    memset(r, 0, sizeof *r);
    char* err = stack_finish(s, r);
    if (err) {
        // copies into r may still be in flight on either stream: wait for them, then hand r's blocks back
        cudaStreamSynchronize(s->e->s);
        cudaStreamSynchronize(s->e->rs);
        cudaGetLastError();
        lsb_result_free(r);
    }
    return err;
}

extern "C" void lsb_stack_destroy(lsb_stack* s) {
    if (!s) return;
    // cudaFree waits for the device; the engine (and its stream) may already be gone
    delete s;
}

extern "C" void lsb_result_free(lsb_result* r) {
    if (!r) return;
    hb_release(r->image_u16);
    hb_release(r->image_f32);
    hb_release(r->winner);
    hb_release(r->depth);
    hb_release(r->conf);
    hb_release(r->floor_cells);
    free(r->sims);
    free(r->gains);
    free(r->shares);
    memset(r, 0, sizeof *r);
}

// ------------------------------------------------- standalone entry points
extern "C" char* lsb_depth_from_slices(lsb_engine* e, const float* slices, uint32_t n, const float* fused, uint32_t w, uint32_t h,
                                       const lsb_depth_params* p, lsb_result* out) {
    if (!e || !slices || !fused || !p || !out) return dup_err("null argument");
    // a stack with the fold skipped: its depth buffers, the fused image and the slices uploaded
    lsb_fuse_params fp{1, 1, 2, 2, 256, 0, 0, 0.f};
    lsb_depth_params dp = *p;
    dp.enabled = 1;
    lsb_stack* s = nullptr;
    lsb_config saved = e->cfg;
    e->cfg.storage = 0;
    char* err = lsb_stack_begin(e, w, h, n, &fp, nullptr, &dp, 0, 0, &s);
    e->cfg = saved;
    if (err) return err;
    cudaStream_t st = e->s;
    const int k = s->bk, dw = s->dw, dh = s->dh;
    const size_t m = (size_t)dw * dh;
    memset(out, 0, sizeof *out);
    auto fail = [&](char* m_) {  // out holds nothing on an error: copies into it are waited for, its buffers freed
        cudaStreamSynchronize(st);
        cudaGetLastError();
        lsb_result_free(out);
        lsb_stack_destroy(s);
        return m_;
    };
#define TRYS(x)                                                                                        \
    do {                                                                                               \
        cudaError_t _e = (x);                                                                          \
        if (_e != cudaSuccess) return fail(dup_err(fmt("%s: %s", #x, cudaGetErrorString(_e))));       \
    } while (0)
    TRYS(cudaMemcpyAsync(s->img, fused, sizeof(float) * 3 * w * h, cudaMemcpyHostToDevice, st));
    TRYS(cudaMemcpyAsync(s->slices, slices, sizeof(float) * n * m, cudaMemcpyHostToDevice, st));
    TRYS(luma_and_guide(s->img, (int)w, (int)h, k, s->yfull, s->guide, dw, dh, st));
    if (dp.agg_radius > 0) gf_stats(s->guide, dw, dh, (int)dp.agg_radius, s->tmp, s->mi, s->vi, st);
    AggArgs ag{s->slices, (int)n, dw, dh, (int)dp.agg_radius, dp.agg_eps, s->guide, s->mi, s->vi, s->state, 0, 0};
    TRYS(aggregate_peaks(ag, false, st, e->grid, !(e->cfg.flags & LSB_FLAG_DIRECT_WINDOW_SUMS)));
    const size_t cnt = (m + 6) / 7;
    TRYS(select_kth(s->state + 7 * m, cnt, 7, cnt / 2, e->hist, e->sel, e->scal + 0, st));
    TRYS(peak_finish(s->state, m, (int)n, e->scal + 0, dp.gate, s->draw, s->conf, s->mins, st));
    if (dp.median) TRYS(median3(s->draw, s->dmed, dw, dh, st));
    else TRYS(cudaMemcpyAsync(s->dmed, s->draw, sizeof(float) * m, cudaMemcpyDeviceToDevice, st));
    TRYS(select_kth(s->conf, cnt, 7, std::min(cnt * 9 / 10, cnt - 1), e->hist, e->sel, e->scal + 1, st));
    TRYS(conf_scale(s->conf, m, e->scal + 1, st));
    const float* dsol = s->dmed;
    float rel = 0.f;
    int it = 0, it1 = 0;
    double rel64 = 0.0;
    if (dp.lambda > 0.f) {
        cudaError_t ce;
        WlsSolver* ws = stack_solver(s, dw, dh, dp, st, &ce);
        if (ce == cudaSuccess) ce = wls_set_weights(ws, s->conf, st);
        if (ce == cudaSuccess) ce = wls_solve(ws, s->dmed, (int)dp.cg_iters, s->u, &rel, &it, st, (int)dp.vcycle_mode, false, &rel64);
        it1 = it;
        if (ce == cudaSuccess && dp.robust > 0.f) {
            ce = robust_weights(s->conf, s->dmed, s->u, dp.robust, s->w2, m, st);
            if (ce == cudaSuccess) ce = wls_set_weights(ws, s->w2, st);
            if (ce == cudaSuccess) ce = wls_solve(ws, s->dmed, (int)dp.cg_iters, s->u, &rel, &it, st, (int)dp.vcycle_mode, false, &rel64);
        }
        if (ce != cudaSuccess) return fail(dup_err(fmt("wls: %s", cudaGetErrorString(ce))));
        dsol = s->u;
    }
    const float max_d = (float)(n - 1);
    if (dp.upsample == 1) {
        gf_stats(s->guide, dw, dh, (int)dp.up_radius, s->tmp, s->mi, s->vi, st);
        gf_coeffs(s->guide, s->mi, s->vi, dsol, dw, dh, (int)dp.up_radius, dp.up_eps, s->t0, s->t1, s->t2, s->tmp, s->abar, s->bbar, st);
        TRYS(upsample(s->abar, s->bbar, s->yfull, s->guide, s->conf, (int)w, (int)h, dw, dh, k, max_d, true, s->dfull, s->cfull, st));
    } else {
        TRYS(upsample(nullptr, dsol, s->yfull, s->guide, s->conf, (int)w, (int)h, dw, dh, k, max_d, false, s->dfull, s->cfull, st));
    }
    out->w = w;
    out->h = h;
    out->n_frames = n;
    out->dw = dw;
    out->dh = dh;
    out->depth = (float*)malloc(sizeof(float) * w * h);
    out->conf = (float*)malloc(sizeof(float) * w * h);
    out->floor_cells = (float*)malloc(sizeof(float) * m);
    if (!out->depth || !out->conf || !out->floor_cells) return fail(dup_err("out of host memory"));
    TRYS(cudaMemcpyAsync(out->depth, s->dfull, sizeof(float) * w * h, cudaMemcpyDeviceToHost, st));
    TRYS(cudaMemcpyAsync(out->conf, s->cfull, sizeof(float) * w * h, cudaMemcpyDeviceToHost, st));
    TRYS(cudaMemcpyAsync(out->floor_cells, s->mins, sizeof(float) * m, cudaMemcpyDeviceToHost, st));
    float sc[2];
    TRYS(cudaMemcpyAsync(sc, e->scal, sizeof sc, cudaMemcpyDeviceToHost, st));
    TRYS(cudaStreamSynchronize(st));
    out->floor_value = sc[0];
    out->p90 = sc[1];
    out->wls_rel = rel;
    out->wls_rel64 = rel64;
    out->wls_iters = it;
    out->wls_iters_first = it1;
    lsb_stack_destroy(s);
    return nullptr;
#undef TRYS
}

extern "C" char* lsb_wls_solve(lsb_engine* e, const float* d, const float* conf, const float* guide, uint32_t w, uint32_t h,
                               float lambda, float sigma_c, uint32_t max_iters, uint32_t edge_mode, uint32_t vcycle_mode, float* u,
                               float* rel, uint32_t* iters, double* ms) {
    if (!e || !d || !conf || !guide || !u) return dup_err("null argument");
    if (edge_mode > 1 || vcycle_mode > 1) return dup_err("edge_mode and vcycle_mode must be 0 or 1");
    if (const char* bad = size_error(w, h)) return dup_err(bad);
    cudaStream_t st = e->s;
    const size_t m = (size_t)w * h;
    DevPool P;
    float *dd, *cc, *gg, *uu;
    TRY(P.get(&dd, m));
    TRY(P.get(&cc, m));
    TRY(P.get(&gg, m));
    TRY(P.get(&uu, m));
    TRY(cudaMemcpyAsync(dd, d, sizeof(float) * m, cudaMemcpyHostToDevice, st));
    TRY(cudaMemcpyAsync(cc, conf, sizeof(float) * m, cudaMemcpyHostToDevice, st));
    TRY(cudaMemcpyAsync(gg, guide, sizeof(float) * m, cudaMemcpyHostToDevice, st));
    TRY(cudaMemsetAsync(uu, 0, sizeof(float) * m, st));
    cudaError_t ce;
    WlsSolver* ws = wls_alloc((int)w, (int)h, &ce);  // planes first: the timed part is the solve
    if (ce == cudaSuccess) ce = cudaEventRecord(e->ev[0], st);
    if (ce == cudaSuccess) ce = wls_prepare(ws, gg, lambda, sigma_c, (int)edge_mode, st);
    if (ce == cudaSuccess) ce = wls_set_weights(ws, cc, st);
    float r = 0.f;
    int it = 0;
    if (ce == cudaSuccess) ce = wls_solve(ws, dd, (int)max_iters, uu, &r, &it, st, (int)vcycle_mode, false, nullptr);
    TRY(cudaEventRecord(e->ev[1], st));
    wls_destroy(ws);
    if (ce != cudaSuccess) return dup_err(fmt("wls: %s", cudaGetErrorString(ce)));
    TRY(cudaMemcpyAsync(u, uu, sizeof(float) * m, cudaMemcpyDeviceToHost, st));
    TRY(cudaStreamSynchronize(st));
    if (rel) *rel = r;
    if (iters) *iters = (uint32_t)it;
    if (ms) *ms = ms_between(e->ev[0], e->ev[1]);
    return nullptr;
}

extern "C" char* lsb_align_pair(lsb_engine* e, const float* rf, const float* tg, uint32_t w, uint32_t h, const double* init8,
                                const uint8_t* free8, uint32_t coarsen, double* out8, uint32_t* evals) {
    if (!e || !rf || !tg || !out8) return dup_err("null argument");
    if (const char* bad = size_error(w, h)) return dup_err(bad);
    cudaStream_t st = e->s;
    DevPool P;
    float *a, *b;
    TRY(P.get(&a, (size_t)w * h));
    TRY(P.get(&b, (size_t)w * h));
    TRY(cudaMemcpyAsync(a, rf, sizeof(float) * w * h, cudaMemcpyHostToDevice, st));
    TRY(cudaMemcpyAsync(b, tg, sizeof(float) * w * h, cudaMemcpyHostToDevice, st));
    std::vector<std::pair<int, int>> dims;
    gauss_dims((int)w, (int)h, dims);
    std::vector<float*> pr, pt;
    for (auto& dd : dims) {
        float *x, *y;
        TRY(P.get(&x, (size_t)dd.first * dd.second));
        TRY(P.get(&y, (size_t)dd.first * dd.second));
        pr.push_back(x);
        pt.push_back(y);
    }
    TRY(gauss_levels(a, (int)w, (int)h, pr, st));
    TRY(gauss_levels(b, (int)w, (int)h, pt, st));
    const double id[8] = {0, 0, 1, 0, 1, 0, 0, 0};
    bool fr[8];
    for (int k = 0; k < 8; k++) fr[k] = free8 ? free8[k] != 0 : (k < 4);
    e->actx.evals = 0;
    e->actx.device_search = e->coop;
    TRY(multiscale_align(e->actx, a, pr, b, pt, (int)w, (int)h, init8 ? init8 : id, fr, (int)coarsen, out8));
    if (evals) *evals = (uint32_t)e->actx.evals;
    return nullptr;
}

extern "C" char* lsb_warp_cost(lsb_engine* e, const float* rf, uint32_t aw, uint32_t ah, const float* tgt, uint32_t tw, uint32_t th,
                               const double* sim8, double* cost) {
    if (!e || !rf || !tgt || !sim8 || !cost) return dup_err("null argument");
    if (const char* bad = size_error(aw, ah)) return dup_err(bad);
    if (const char* bad = size_error(tw, th)) return dup_err(bad);
    cudaStream_t st = e->s;
    DevPool P;
    float *a, *b;
    TRY(P.get(&a, (size_t)aw * ah));
    TRY(P.get(&b, (size_t)tw * th));
    TRY(cudaMemcpyAsync(a, rf, sizeof(float) * aw * ah, cudaMemcpyHostToDevice, st));
    TRY(cudaMemcpyAsync(b, tgt, sizeof(float) * tw * th, cudaMemcpyHostToDevice, st));
    TRY(cost_single(e->actx, a, (int)aw, (int)ah, b, (int)tw, (int)th, sim8, cost));
    return nullptr;
}

// stack.rs:857 `weighted` -> wav.rs:92 `weighted_average` over the frames of the last run
extern "C" char* lsb_stack_weighted_average(lsb_stack* s, const lsb_wav_params* p, float* out) {
    if (!s || !p || !out) return dup_err("null argument");
    if (!s->folded || !s->dp.enabled) return dup_err("the weighted average needs a run with the depth pass (its focus measure and noise floor)");
    if (!(p->power >= 0.f) || !(p->gate >= 0.f) || p->smooth > 64) return dup_err("wav: power and gate must be >= 0, smooth at most 64");
    lsb_engine* e = s->e;
    cudaStream_t st = e->s;
    const int n = (int)s->count, dw = s->dw, dh = s->dh;
    const size_t m = (size_t)dw * dh;
    if (s->wav_frames < n) {
        if (s->wav_w) cudaFree(s->wav_w);
        s->wav_w = nullptr;
        s->wav_frames = 0;
        TRY(cudaMalloc(&s->wav_w, sizeof(float) * m * n));
        s->wav_frames = n;
    }
    // the guided filter's statistics for radius `smooth` on the depth pass's guide (the fused luma's block mean)
    const int r = (int)p->smooth;
    const bool edge = p->edge != 0 && r > 0;
    if (edge) gf_stats(s->guide, dw, dh, r, s->tmp, s->mi, s->vi, st);
    WavScratch t{s->w2, s->draw, s->t0, s->t1, s->t2, s->tmp, s->abar, s->bbar};
    const bool half = s->storage != STORE_F32;
    for (int k = 0; k < n; k++) {
        const void* slice = (const char*)s->slices + (size_t)k * m * gs_bytes(s);
        TRY(wav_weights(slice, half, s->mins, dw, dh, p->gate, p->power, r, edge, s->guide, s->mi, s->vi, s->dp.agg_eps, t,
                        s->wav_w + (size_t)k * m, st));
    }
    bool focus = false;
    int src = 0;
    const bool aligned = s->ap.enabled && n > 1 && !s->f32src;
    FoldArgs a = level_args(s, 0, aligned, false, &focus, &src);
    TRY(wav_accumulate(a, src, s->wav_w, n, dw, dh, s->bk, s->img_tmp, st));
    TRY(cudaMemcpyAsync(out, s->img_tmp, sizeof(float) * 3 * (size_t)s->w * s->h, cudaMemcpyDeviceToHost, st));
    TRY(cudaStreamSynchronize(st));
    return nullptr;
}

// stack.rs:76 `slab_ranges`
extern "C" uint32_t lsb_slab_ranges(uint32_t count, uint32_t size, uint32_t overlap, uint32_t* lohi, uint32_t max_slabs) {
    if (count == 0) return 0;
    size = std::min(std::max(size, 1u), count);
    overlap = std::min(overlap, size - 1);
    uint32_t k = 0, lo = 0;
    for (;;) {
        const uint32_t hi = std::min(lo + size - 1, count - 1);
        if (lohi && k < max_slabs) {
            lohi[2 * k] = lo;
            lohi[2 * k + 1] = hi;
        }
        k++;
        if (hi + 1 >= count) return k;
        lo = hi + 1 - overlap;
    }
}

// stack.rs:740 `fuse_range` over frames lo..hi of the last run, as a fuser of their own would fold them:
// every level's selection over those frames alone from a fresh state (their Gaussian levels and level-0
// frames are the run's, which a fresh fuser would build the same), the residual over their tops and the
// collapse, into slab_img. The run's accumulators, residual, winner map and image are left as they were.
static char* slab_fold(lsb_stack* s, int lo, int hi) {
    lsb_engine* e = s->e;
    cudaStream_t st = e->s;
    const int n = hi - lo + 1, L = s->levels;
    const size_t gsb = gs_bytes(s);
    if (s->slab_acc.empty()) {
        s->slab_acc.assign(L, nullptr);
        s->slab_best.assign(L, nullptr);
        for (int l = 0; l < L; l++) {
            TRY(s->pool.get(&s->slab_acc[l], 3 * (size_t)s->lw[l] * s->lh[l]));
            TRY(s->pool.get(&s->slab_best[l], (size_t)s->lw[l] * s->lh[l]));
        }
        TRY(s->pool.get(&s->slab_top, 3 * (size_t)s->lw[L] * s->lh[L]));
        TRY(s->pool.get(&s->slab_img, 3 * (size_t)s->w * s->h));
    }
    const bool aligned = s->ap.enabled && s->count > 1 && !s->f32src;
    const bool halo = s->fp.halo > 0.f;
    const int guide = std::min((int)s->fp.depth_level, L - 1);
    auto frame_g = [&](int l) { return (size_t)lo * 3 * s->lw[l] * s->lh[l] * gsb; };
    auto frame_w = [&](int l) { return (size_t)lo * s->lw[l] * s->lh[l]; };
    TRY(cudaMemsetAsync(s->status, 0, sizeof(int), st));
    for (int l = 0; l < L; l++) {
        bool focus = false;
        int src = 0;
        FoldArgs a = level_args(s, l, aligned, false, &focus, &src);
        // frames lo..hi as a stack of their own: sources, transforms and levels offset to frame lo
        a.nframes = n;
        a.red_n = 0;
        a.sel_k0 = 0;
        a.sel_k1 = n;
        if (l == 0) {
            if (a.src_u16) a.src_u16 += (size_t)lo * s->w * s->h * 3;
            if (a.src_f32) a.src_f32 += (size_t)lo * 3 * s->w * s->h;
        } else {
            a.src_g = (const char*)a.src_g + frame_g(l);
        }
        a.dst_g = (char*)a.dst_g + frame_g(l + 1);
        a.xf = s->xf_dev + lo;
        a.acc = s->slab_acc[l];
        a.best = s->slab_best[l];
        a.winner = nullptr;
        if (halo && l >= guide) {
            a.halo_mode = l == guide ? 1 : 2;
            a.halo_p = std::min(s->fp.halo, 8.0f);
            a.halo_w = s->halo_w[l] + frame_w(l);
            if (l > guide)
                TRY(reduce_weights(s->halo_w[l - 1] + frame_w(l - 1), s->lw[l - 1], s->lh[l - 1], n, a.halo_w, s->lw[l], s->lh[l], st));
        } else {
            set_groups(s, a);
        }
        TRY(fold_level(a, src, s->storage, (int)s->fp.energy_radius, false, st, e->grid_select > 0 ? e->grid_select : e->grid));
    }
    const int wt = s->lw[L], ht = s->lh[L];
    const void* tops = (const char*)s->g[L] + frame_g(L);
    if (halo) {
        TRY(reduce_weights(s->halo_w[L - 1] + frame_w(L - 1), s->lw[L - 1], s->lh[L - 1], n, s->halo_w[L] + frame_w(L), wt, ht, st));
        TRY(halo_top(tops, s->storage, s->xf_dev + lo, s->halo_w[L] + frame_w(L), n, wt, ht, s->slab_top, s->dev_s, st));
        TRY(halo_divide(s->slab_top, s->dev_s, wt, ht, st));
        for (int l = guide + 1; l < L; l++) TRY(halo_divide(s->slab_acc[l], s->slab_best[l], s->lw[l], s->lh[l], st));
    } else {
        // the log table of the top rule's entropy window is the run's (lnp, written for the same radius)
        ResidualArgs ra{tops, n, wt, ht, (int)s->fp.top_rule, (int)s->fp.top_radius, (int)s->fp.entropy_bins, s->dev_s, s->ent_s,
                        s->slab_top, s->xf_dev + lo};
        TRY(fuse_residuals(ra, s->storage, s->lnp, st));
    }
    const float* coarse = s->slab_top;
    for (int l = L - 1; l >= 0; l--) {
        float* out = (l % 2 == 0) ? s->slab_img : s->img_tmp;
        TRY(collapse_level(s->slab_acc[l], coarse, out, s->lw[l], s->lh[l], s->lw[l + 1], s->lh[l + 1], l == 0, nullptr, st));
        coarse = out;
    }
    return nullptr;
}

// stack.rs:872 `fuse_slabs` for one slab: fuse_range, the cut (pyramid.rs:31) and the resize (prep.rs:46)
extern "C" char* lsb_stack_fuse_range(lsb_stack* s, uint32_t lo, uint32_t hi, const uint32_t* rect, uint32_t out_w, uint32_t out_h,
                                      uint32_t interp, float* out) {
    if (!s || !out) return dup_err("null argument");
    if (!s->folded) return dup_err("fuse_range needs a finished (or run) stack: it fuses the frames as that run folded them");
    if (lo > hi || hi >= s->count) return dup_err(fmt("fuse_range: frames %u..%u of a %u-frame stack", lo, hi, s->count));
    if (interp > 5) return dup_err(fmt("fuse_range: interp %u out of range (0..5)", interp));
    uint32_t r[4] = {0, 0, s->w, s->h};
    if (rect) memcpy(r, rect, sizeof r);
    if (r[2] == 0 || r[3] == 0 || r[0] >= s->w || r[1] >= s->h || r[2] > s->w - r[0] || r[3] > s->h - r[1])
        return dup_err(fmt("fuse_range: the rectangle %u,%u %ux%u is not inside the %ux%u frame", r[0], r[1], r[2], r[3], s->w, s->h));
    if ((out_w == 0) != (out_h == 0)) return dup_err("fuse_range: give both output dimensions or neither");
    const uint32_t ow = out_w ? out_w : r[2], oh = out_h ? out_h : r[3];
    if (const char* why = size_error(ow, oh)) return dup_err(fmt("fuse_range output: %s", why));
    if (s->fp.halo > 0.f && s->halo_w.empty()) return dup_err("fuse_range: the halo weights of the run are missing");
    char* err = slab_fold(s, (int)lo, (int)hi);
    if (err) return err;
    cudaStream_t st = s->e->s;
    const size_t of = 3 * (size_t)ow * oh;
    if (s->slab_out_floats < of) {
        if (s->slab_out) cudaFree(s->slab_out);
        s->slab_out = nullptr;
        s->slab_out_floats = 0;
        TRY(cudaMalloc(&s->slab_out, sizeof(float) * of));
        s->slab_out_floats = of;
    }
    TRY(resize_planes(s->slab_img, s->w, (size_t)s->w * s->h, 3, (int)r[0], (int)r[1], (int)r[2], (int)r[3], (int)ow, (int)oh, (int)interp,
                      s->slab_out, st));
    TRY(cudaMemcpyAsync(out, s->slab_out, sizeof(float) * of, cudaMemcpyDeviceToHost, st));
    TRY(cudaStreamSynchronize(st));
    int status = 0;
    TRY(cudaMemcpy(&status, s->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status) return dup_err(fmt("device status 0x%x (a kernel met a shape it was not built for)", status));
    return nullptr;
}

// prep.rs:46 `resize` / :63 `resize_plane` of host planes, on the engine's stream
extern "C" char* lsb_resize(lsb_engine* e, const float* src, uint32_t planes, uint32_t pw, uint32_t ph, uint32_t w, uint32_t h,
                            uint32_t interp, float* out) {
    if (!e || !src || !out) return dup_err("null argument");
    if (interp > 5) return dup_err(fmt("resize: interp %u out of range (0..5)", interp));
    if (planes == 0 || planes > 64) return dup_err("resize: 1 to 64 planes");
    if (const char* why = size_error(pw, ph)) return dup_err(fmt("resize source: %s", why));
    if (const char* why = size_error(w, h)) return dup_err(fmt("resize output: %s", why));
    const size_t ni = (size_t)planes * pw * ph, no = (size_t)planes * w * h;
    float *di = nullptr, *dout = nullptr;
    cudaError_t ce = cudaMalloc(&di, sizeof(float) * ni);
    if (ce == cudaSuccess) ce = cudaMalloc(&dout, sizeof(float) * no);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(di, src, sizeof(float) * ni, cudaMemcpyHostToDevice, e->s);
    if (ce == cudaSuccess) ce = resize_planes(di, pw, (size_t)pw * ph, (int)planes, 0, 0, (int)pw, (int)ph, (int)w, (int)h, (int)interp, dout, e->s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(out, dout, sizeof(float) * no, cudaMemcpyDeviceToHost, e->s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->s);
    cudaFree(di);
    cudaFree(dout);
    if (ce != cudaSuccess) return dup_err(fmt("resize: %s", cudaGetErrorString(ce)));
    return nullptr;
}

extern "C" char* lsb_stack_set_warm_start(lsb_stack* s, lsb_unet* u) {
    if (!s) return dup_err("lsb_stack_set_warm_start: null stack");
    s->net = u;
    return nullptr;
}

extern "C" char* lsb_stack_depth_planes(lsb_stack* s, const float** guide, const float** d, const float** conf, const float** u,
                                        uint32_t* dw, uint32_t* dh) {
    if (!s || !s->folded || !s->dp.enabled) return dup_err("lsb_stack_depth_planes: run the stack with the depth pass first");
    *guide = s->guide;
    *d = s->dmed;
    *conf = s->conf;
    *u = s->dp.lambda > 0.f ? s->u : s->dmed;
    *dw = (uint32_t)s->dw;
    *dh = (uint32_t)s->dh;
    return nullptr;
}

// Several stacks at once (no counterpart in the reference, whose caller loops over stacks,
// stack.rs:1011): the stacks of one engine run back to back on its streams; the stacks of
// different engines on the same device run side by side, one host thread per engine. Each
// engine's persistent kernels and device search take the CTAs its grid limit allows, so that
// engines created with a share of the SMs each (lsb_config.grid_limit) fill the GPU together:
// one stack's registration chain, which leaves most of the GPU idle, beside another's fold.
extern "C" char* lsb_batch_run(lsb_stack* const* stacks, uint32_t n_stacks, lsb_result* outs) {
    if (!stacks || !outs) return dup_err("null argument");
    for (uint32_t i = 0; i < n_stacks; i++) memset(&outs[i], 0, sizeof(lsb_result));
    std::vector<lsb_engine*> engines;
    std::vector<std::vector<uint32_t>> work;
    for (uint32_t i = 0; i < n_stacks; i++) {
        const lsb_stack* s = stacks[i];
        if (!s) return dup_err(fmt("stack %u is null", i));
        if (s->e->device != stacks[0]->e->device) return dup_err("the stacks of a batch run on one device");
        // the focus measure's taps are one constant-memory copy per device
        if (s->dp.enabled && stacks[0]->dp.enabled && s->e != stacks[0]->e &&
            (s->dp.focus != stacks[0]->dp.focus || s->dp.r_in != stacks[0]->dp.r_in || s->dp.r_out != stacks[0]->dp.r_out))
            return dup_err(fmt("stack %u: stacks of different engines in one batch share the focus measure and its radii", i));
        const size_t k = std::find(engines.begin(), engines.end(), s->e) - engines.begin();
        if (k == engines.size()) engines.push_back(s->e), work.emplace_back();
        work[k].push_back(i);
    }
    std::vector<char*> errs(n_stacks, nullptr);
    auto run = [&](size_t k) {
        if (cudaSetDevice(engines[k]->device) != cudaSuccess) {
            errs[work[k][0]] = dup_err("cudaSetDevice failed");
            return;
        }
        for (uint32_t i : work[k])
            if ((errs[i] = lsb_stack_finish(stacks[i], &outs[i])) != nullptr) break;
    };
    if (engines.size() == 1) {
        run(0);
    } else {
        std::vector<std::future<void>> th;
        for (size_t k = 1; k < engines.size(); k++) th.push_back(std::async(std::launch::async, run, k));
        run(0);
        for (auto& t : th) t.get();
    }
    for (uint32_t i = 0; i < n_stacks; i++) {
        if (!errs[i]) continue;
        char* msg = dup_err(fmt("stack %u: %s", i, errs[i]));
        for (uint32_t j = 0; j < n_stacks; j++) {
            lsb_result_free(&outs[j]);
            free(errs[j]);
        }
        return msg;
    }
    return nullptr;
}

// The project's autotuner: the persistent kernels' grid sizes (the fold's select
// kernel and the depth aggregation; CTAs walk tiles, so any grid gives the same
// results) timed on this stack's own frames, one full run per candidate, the
// fastest kept in the engine for every later run.
extern "C" char* lsb_stack_autotune(lsb_stack* s, lsb_tuning* out) {
    if (!s || !out) return dup_err("null argument");
    lsb_engine* e = s->e;
    const int cand[3] = {e->sms, (3 * e->sms) / 2, 2 * e->sms};
    double best_sel = 1e300, best_agg = 1e300;
    int gs = cand[0], ga = cand[0];
    memset(out, 0, sizeof *out);
    for (int i = 0; i < 3; i++) {
        e->grid_select = cand[i];
        e->grid_agg = cand[i];
        char* err = run_pipeline(s);
        if (!err) err = run_pipeline(s);  // the second run is the one timed
        if (err) {
            e->grid_select = e->grid_agg = 0;
            return err;
        }
        const double sel = s->ms[2], agg = s->ms[4];  // the fold, the aggregation
        out->candidates[i] = (uint32_t)cand[i];
        out->fold_ms[i] = sel;
        out->aggregate_ms[i] = agg;
        if (sel < best_sel) best_sel = sel, gs = cand[i];
        if (agg < best_agg) best_agg = agg, ga = cand[i];
    }
    e->grid_select = gs;
    e->grid_agg = ga;
    out->grid_select = (uint32_t)gs;
    out->grid_aggregate = (uint32_t)ga;
    return nullptr;
}
