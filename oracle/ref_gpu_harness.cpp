// Measurement infrastructure, not the product: the reference's own GPU path
// (crates/lapstack-core/src/gpu.rs) timed on this GPU, to compare the engine
// with the reference's kernels on the same hardware.
//
// The kernels are the reference's, unchanged: oracle/ref_gpu.py extracts
// gpu.rs's NVRTC sources into oracle/_ref/ and `make ref` compiles them to PTX
// for compute_86 as gpu.rs:316 does (the driver JIT-compiles it at load). This
// file is the host side: it loads the two modules through the driver API and
// drives them in gpu.rs's order and launch shapes (cfg1: 1024-thread blocks,
// cfg2: 32 x 8), with the reference's host steps restated from the oracle
// (Nelder-Mead and its level steps, the brightness ratio, the residual rule,
// the medians of the depth pass):
//
//   per frame   GpuFrames::process (gpu.rs:751): planes up, luma, registration
//               pyramid, the host-driven search (one warp_cost launch and read
//               back per evaluation, gpu.rs:692), the warp, the next reference,
//               the brightness sums and gains, the focus slice (read back);
//               GpuFuser::push_device (gpu.rs:451): the Laplacian pyramid, the
//               energy, window and selection per level, the top read back.
//   after       GpuFuser::finish (gpu.rs:517): the residual rule on the host,
//               the collapse, the image read back; depth_from_slices
//               (gpu.rs:1327): slices up one at a time, guided filter and peak
//               tracker, the medians on the host, the WLS solve (gpu.rs:1240,
//               the residual read back every iteration), the guided upsampling.
//
// Usage: ref_gpu_harness <fuse.ptx> <depth.ptx> <w> <h> <n_total> <n_sample> <coarsen> <agg_radius> [seed]
//        [--check] [--noalign]
// Frames are the seeded synthetic stack of the benchmark (oracle/orc_synth.hpp),
// made on the host one at a time; frames 0 .. n_sample-1 are processed and
// folded. With n_sample < n_total the per-frame cost is extrapolated to n_total
// frames and the depth pass runs over n_total slices (the sample's repeated in
// order). --check runs the oracle over the same frames and reports how far the
// reference GPU path's transforms and fused image lie from its CPU path;
// --noalign keeps every frame at the identity. Prints one JSON line.
#include <cuda.h>
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "orc_stack.hpp"
#include "orc_synth.hpp"

using namespace orc;

#define CU(x)                                                                              \
    do {                                                                                   \
        CUresult r_ = (x);                                                                 \
        if (r_ != CUDA_SUCCESS) {                                                          \
            const char* s_ = nullptr;                                                      \
            cuGetErrorString(r_, &s_);                                                     \
            fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #x, s_ ? s_ : "?");      \
            exit(2);                                                                       \
        }                                                                                  \
    } while (0)
#define RT(x)                                                                              \
    do {                                                                                   \
        cudaError_t r_ = (x);                                                              \
        if (r_ != cudaSuccess) {                                                           \
            fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(r_)); \
            exit(2);                                                                       \
        }                                                                                  \
    } while (0)

static double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static std::string read_file(const char* path) {
    FILE* f = fopen(path, "rb");
    if (!f) {
        fprintf(stderr, "cannot read %s\n", path);
        exit(2);
    }
    std::string s;
    char buf[65536];
    size_t k;
    while ((k = fread(buf, 1, sizeof buf, f)) > 0) s.append(buf, k);
    fclose(f);
    return s;
}

// one NVRTC-style module (gpu.rs:317-321): PTX loaded by the driver, kernels by name
struct Module {
    CUmodule m = nullptr;
    explicit Module(const char* ptx_path) {
        std::string ptx = read_file(ptx_path);
        CU(cuModuleLoadData(&m, ptx.c_str()));
    }
    CUfunction f(const char* name) const {
        CUfunction fn;
        CU(cuModuleGetFunction(&fn, m, name));
        return fn;
    }
};

static CUstream g_s;

// gpu.rs:280 cfg2 (32 x 8 blocks over w x h) and cudarc's for_num_elems (1024-thread blocks)
struct Cfg {
    unsigned gx, gy, bx, by;
};
static Cfg cfg2(size_t w, size_t h) { return {(unsigned)((w + 31) / 32), (unsigned)((h + 7) / 8), 32, 8}; }
static Cfg cfg1(size_t n) { return {(unsigned)((n + 1023) / 1024), 1, 1024, 1}; }

template <class... A>
static void launch(CUfunction f, Cfg c, A... a) {
    void* args[] = {(void*)&a...};
    CU(cuLaunchKernel(f, c.gx, c.gy, 1, c.bx, c.by, 1, 0, g_s, args, nullptr));
}

static float* dalloc(size_t n) {
    float* p = nullptr;
    RT(cudaMalloc(&p, sizeof(float) * std::max<size_t>(n, 1)));
    RT(cudaMemset(p, 0, sizeof(float) * std::max<size_t>(n, 1)));
    return p;
}
static void sync() { CU(cuStreamSynchronize(g_s)); }
static void d2h(void* dst, const void* src, size_t bytes) {
    RT(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)g_s));
    sync();
}
static void h2d(void* dst, const void* src, size_t bytes) { RT(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, (cudaStream_t)g_s)); }
static void d2d(void* dst, const void* src, size_t bytes) { RT(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)g_s)); }

// ------------------------------------------------------------------ the fuser
// gpu.rs:326 GpuFuser (no halo control: the benchmark's settings)
struct RefFuser {
    const Module& M;
    CUfunction redH, redV, expH, expV, subk, addk, clampk, energy_y, winH, winV, selk;
    size_t w, h, levels, depth_level;
    std::vector<std::pair<size_t, size_t>> dims;
    std::vector<std::array<float*, 3>> acc, cur;
    std::vector<float*> best;
    float *win, *wt, *tmp_half, *tmp_full, *en, *en2;
    int klen;
    std::vector<Img3<float>> tops;
    int count = 0;
    RefFuser(const Module& m, size_t w_, size_t h_, const FuseParams& p) : M(m), w(w_), h(h_) {
        redH = M.f("redH"), redV = M.f("redV"), expH = M.f("expH"), expV = M.f("expV"), subk = M.f("subk"), addk = M.f("addk");
        clampk = M.f("clampk"), energy_y = M.f("energy_y"), winH = M.f("winH"), winV = M.f("winV"), selk = M.f("selk");
        levels = std::max<size_t>(p.levels ? p.levels : auto_levels(w, h, 32), 1);
        depth_level = std::min(p.depth_level, levels - 1);
        dims.push_back({w, h});
        for (size_t l = 0; l < levels; l++) dims.push_back({half(dims.back().first), half(dims.back().second)});
        for (size_t l = 0; l <= levels; l++) {
            const size_t n = dims[l].first * dims[l].second;
            acc.push_back({dalloc(n), dalloc(n), dalloc(n)});
            if (l >= 1) cur.push_back({dalloc(n), dalloc(n), dalloc(n)});
            float* b = dalloc(n);
            std::vector<float> neg(n, -1.0f);
            h2d(b, neg.data(), sizeof(float) * n);
            best.push_back(b);
        }
        win = dalloc(dims[depth_level].first * dims[depth_level].second);
        std::vector<float> wv = binomial<float>(p.energy_radius);
        klen = (int)wv.size();
        wt = dalloc(wv.size());
        h2d(wt, wv.data(), sizeof(float) * wv.size());
        tmp_half = dalloc(std::max(half(w) * h, half(h) * w));
        tmp_full = dalloc(w * h);
        en = dalloc(w * h);
        en2 = dalloc(w * h);
        sync();
    }
    // gpu.rs:412 `build`: the Laplacian pyramid of p0 in place
    void build(std::array<float*, 3>& p0) {
        for (size_t li = 0; li < levels; li++) {
            const int fw = (int)dims[li].first, fh = (int)dims[li].second, cw = (int)dims[li + 1].first, ch = (int)dims[li + 1].second;
            for (int c = 0; c < 3; c++) {
                float* fp = li == 0 ? p0[c] : cur[li - 1][c];
                float* cp = cur[li][c];
                launch(redH, cfg2(cw, fh), (const float*)fp, tmp_half, fw, fh, cw);
                launch(redV, cfg2(cw, ch), (const float*)tmp_half, cp, fh, cw, ch);
                launch(expH, cfg2(fw, ch), (const float*)cp, tmp_half, cw, ch, fw);
                launch(expV, cfg2(fw, fh), (const float*)tmp_half, tmp_full, ch, fw, fh);
                launch(subk, cfg1((size_t)fw * fh), fp, (const float*)tmp_full, fw * fh);
            }
        }
    }
    // gpu.rs:451 `push_device`
    void push_device(std::array<float*, 3>& p0) {
        build(p0);
        const float idx = (float)count;
        for (size_t li = 0; li < levels; li++) {
            const size_t lw = dims[li].first, lh = dims[li].second, n = lw * lh;
            const std::array<float*, 3>& np = li == 0 ? p0 : cur[li - 1];
            launch(energy_y, cfg1(n), (const float*)np[0], (const float*)np[1], (const float*)np[2], en, (int)n);
            if (klen > 1) {
                launch(winH, cfg2(lw, lh), (const float*)en, en2, (int)lw, (int)lh, (const float*)wt, klen);
                launch(winV, cfg2(lw, lh), (const float*)en2, en, (int)lw, (int)lh, (const float*)wt, klen);
            }
            const int rec = li == depth_level;
            launch(selk, cfg1(n), (const float*)en, best[li], acc[li][0], acc[li][1], acc[li][2], (const float*)np[0], (const float*)np[1],
                   (const float*)np[2], win, idx, rec, (int)n);
        }
        // the residual level back to the host
        const size_t tw = dims[levels].first, th = dims[levels].second;
        Img3<float> t(tw, th);
        for (int c = 0; c < 3; c++) d2h(t.p[c].data(), cur[levels - 1][c], sizeof(float) * tw * th);
        tops.push_back(std::move(t));
        count++;
    }
    // gpu.rs:517 `finish`: the residual rule on the host, the collapse, the image back
    Img3<float> finish(const FuseParams& p) {
        Img3<float> top = fuse_residuals<float>(tops, p);
        for (int c = 0; c < 3; c++) h2d(acc[levels][c], top.p[c].data(), sizeof(float) * top.w * top.h);
        for (size_t li = levels; li-- > 0;) {
            const int fw = (int)dims[li].first, fh = (int)dims[li].second, cw = (int)dims[li + 1].first, ch = (int)dims[li + 1].second;
            for (int c = 0; c < 3; c++) {
                launch(expH, cfg2(fw, ch), (const float*)acc[li + 1][c], tmp_half, cw, ch, fw);
                launch(expV, cfg2(fw, fh), (const float*)tmp_half, tmp_full, ch, fw, fh);
                launch(addk, cfg1((size_t)fw * fh), acc[li][c], (const float*)tmp_full, fw * fh);
            }
        }
        Img3<float> img(w, h);
        for (int c = 0; c < 3; c++) {
            launch(clampk, cfg1(w * h), acc[0][c], (int)(w * h));
            d2h(img.p[c].data(), acc[0][c], sizeof(float) * w * h);
        }
        std::vector<float> wn(dims[depth_level].first * dims[depth_level].second);
        d2h(wn.data(), win, sizeof(float) * wn.size());
        return img;
    }
};

// ------------------------------------------------------------------ the frames
struct DLvl {
    float* p;
    size_t w, h;
};
// gpu.rs:560 `pyr_dims`: the registration levels above full resolution
static std::vector<std::pair<size_t, size_t>> pyr_dims(size_t w, size_t h) {
    std::vector<std::pair<size_t, size_t>> d;
    size_t cw = w, ch = h;
    while (ch > 64 && cw > 8) {
        cw = half(cw);
        ch = half(ch);
        d.push_back({cw, ch});
    }
    return d;
}

// gpu.rs:602 GpuFrames (similarity model, Spline4x4, brightness on, the RDF focus measure)
struct Frames {
    const Module& M;
    CUfunction warp_cost, lumak, burtH, burtV, warpk, gridk, bsumk, gaink, rdfk, bmeank;
    size_t w, h, gw, gh;
    int interp;
    std::array<float*, 3> src, out;
    float *yt, *yr, *tmp;
    std::vector<DLvl> pt, pr;
    bool have_ref = false;
    std::array<float*, 3> grid{nullptr, nullptr, nullptr};
    double *sums, *cost;
    float* taps = nullptr;
    int ntaps = 0;
    float* slice = nullptr;
    size_t evals = 0;
    static constexpr size_t BSTEP = 4;
    Frames(const Module& m, size_t w_, size_t h_, int interp_) : M(m), w(w_), h(h_), interp(interp_) {
        warp_cost = M.f("warp_cost"), lumak = M.f("lumak"), burtH = M.f("burtH"), burtV = M.f("burtV"), warpk = M.f("warpk");
        gridk = M.f("gridk"), bsumk = M.f("bsumk"), gaink = M.f("gaink"), rdfk = M.f("rdfk"), bmeank = M.f("bmeank");
        const size_t n = w * h;
        for (int c = 0; c < 3; c++) src[c] = dalloc(n), out[c] = dalloc(n);
        yt = dalloc(n), yr = dalloc(n), tmp = dalloc(n);
        for (auto& d : pyr_dims(w, h)) {
            pt.push_back({dalloc(d.first * d.second), d.first, d.second});
            pr.push_back({dalloc(d.first * d.second), d.first, d.second});
        }
        gw = (w + BSTEP - 1) / BSTEP, gh = (h + BSTEP - 1) / BSTEP;
        RT(cudaMalloc(&sums, sizeof(double) * 7));
        RT(cudaMalloc(&cost, sizeof(double) * 3));
    }
    // gpu.rs:661 `reduce_chain`
    void reduce_chain(const float* y, std::vector<DLvl>& lv) {
        size_t fw = w, fh = h;
        for (size_t l = 0; l < lv.size(); l++) {
            const float* fine = l == 0 ? y : lv[l - 1].p;
            const int fwi = (int)fw, fhi = (int)fh, cwi = (int)lv[l].w, chi = (int)lv[l].h;
            launch(burtH, cfg2(lv[l].w, fh), fine, tmp, fwi, fhi, cwi);
            launch(burtV, cfg2(lv[l].w, lv[l].h), (const float*)tmp, lv[l].p, fwi, fhi, cwi, chi);
            fw = lv[l].w, fh = lv[l].h;
        }
    }
    void luma(const std::array<float*, 3>& p, float* y) {
        launch(lumak, cfg1(w * h), (const float*)p[0], (const float*)p[1], (const float*)p[2], y, (int)(w * h));
    }
    // gpu.rs:692 `search`: the CPU's multiscale_align with each cost a launch and a read-back
    Sim search(const Sim& guess, const bool free[8], size_t coarsen) {
        std::vector<size_t> free_idx;
        for (size_t k = 0; k < 8; k++)
            if (free[k]) free_idx.push_back(k);
        const size_t nlv = std::min(pt.size(), pr.size()) + 1;
        const size_t finest = std::min(coarsen, nlv - 1);
        auto lvl_of = [&](std::vector<DLvl>& p, float* y, size_t l) { return l == 0 ? DLvl{y, w, h} : p[l - 1]; };
        double cur[8];
        for (int k = 0; k < 8; k++) cur[k] = guess.v[k];
        std::vector<double> lo_f, hi_f;
        for (size_t k : free_idx) lo_f.push_back(guess.v[k] - SIM_SPAN[k]), hi_f.push_back(guess.v[k] + SIM_SPAN[k]);
        for (size_t lvl = nlv; lvl-- > finest;) {
            const DLvl rd = lvl_of(pr, yr, lvl), td = lvl_of(pt, yt, lvl);
            double snap[8];
            memcpy(snap, cur, sizeof snap);
            auto costf = [&](const std::vector<double>& xf) -> double {
                Sim s;
                memcpy(s.v, snap, sizeof snap);
                for (size_t k = 0; k < free_idx.size(); k++) s.v[free_idx[k]] = xf[k];
                Mat3 m, inv;
                sim_matrix(s, td.w, td.h, m);
                mat_inverse(m, inv);
                const float ia = (float)inv[0][0], ib = (float)inv[0][1], itx = (float)inv[0][2];
                const float id_ = (float)inv[1][0], ie = (float)inv[1][1], ity = (float)inv[1][2];
                const float ig0 = (float)inv[2][0], ig1 = (float)inv[2][1];
                RT(cudaMemsetAsync(cost, 0, sizeof(double) * 3, (cudaStream_t)g_s));
                launch(warp_cost, cfg2(rd.w, rd.h), (const float*)td.p, (int)td.w, (int)td.h, (const float*)rd.p, (int)rd.w, (int)rd.h, ia, ib,
                       itx, id_, ie, ity, ig0, ig1, cost);
                double r[3];
                d2h(r, cost, sizeof r);
                evals++;
                if (r[2] < 16.0) return 1e9;
                return std::sqrt(std::max((r[1] - r[0] * r[0] / r[2]) / r[2], 0.0));
            };
            std::vector<double> x0, step, tol;
            for (size_t k : free_idx) x0.push_back(cur[k]);
            level_steps(free_idx, lvl, w, h, step, tol);
            std::vector<double> best = nelder_mead(costf, x0, lo_f, hi_f, step, tol);
            for (size_t k = 0; k < free_idx.size(); k++) cur[free_idx[k]] = best[k];
        }
        Sim s;
        memcpy(s.v, cur, sizeof cur);
        return s;
    }
    // gpu.rs:751 `process` of one frame (planar f32 on the host); returns the transform, gains, focus slice
    Sim process(const Img3<float>& img, const Sim& guess, const bool free[8], size_t coarsen, const DepthParams& dp, float gains[3],
                std::vector<float>& focus) {
        const size_t n = w * h;
        for (int c = 0; c < 3; c++) h2d(src[c], img.p[c].data(), sizeof(float) * n);
        const bool first = !have_ref;
        if (!first) {
            luma(src, yt);
            reduce_chain(yt, pt);
        }
        const Sim sim = first ? Sim() : search(guess, free, coarsen);
        Mat3 m, inv;
        sim_matrix(sim, w, h, m);
        mat_inverse(m, inv);
        if (sim.is_id()) {
            for (int c = 0; c < 3; c++) d2d(out[c], src[c], sizeof(float) * n);
        } else {
            for (int c = 0; c < 3; c++)
                launch(warpk, cfg2(w, h), (const float*)src[c], out[c], (int)w, (int)h, inv[0][0], inv[0][1], inv[0][2], inv[1][0], inv[1][1],
                       inv[1][2], inv[2][0], inv[2][1], interp);
        }
        luma(out, yr);
        reduce_chain(yr, pr);
        have_ref = true;
        gains[0] = gains[1] = gains[2] = 1.0f;
        if (first) {
            for (int c = 0; c < 3; c++) {
                grid[c] = dalloc(gw * gh);
                launch(gridk, cfg2(gw, gh), (const float*)out[c], grid[c], (int)w, (int)gw, (int)gh, (int)BSTEP);
            }
        } else {
            RT(cudaMemsetAsync(sums, 0, sizeof(double) * 7, (cudaStream_t)g_s));
            launch(bsumk, cfg2(gw, gh), (const float*)out[0], (const float*)out[1], (const float*)out[2], (const float*)grid[0],
                   (const float*)grid[1], (const float*)grid[2], (int)w, (int)h, (int)gw, (int)gh, (int)BSTEP, (int)sim.is_id(), inv[0][0],
                   inv[0][1], inv[0][2], inv[1][0], inv[1][1], inv[1][2], inv[2][0], inv[2][1], sums);
            double r[7];
            d2h(r, sums, sizeof r);
            const double rf[3] = {r[3], r[4], r[5]}, fr[3] = {r[0], r[1], r[2]};
            bratio(rf, fr, (size_t)r[6], gains);
        }
        for (int c = 0; c < 3; c++)
            if (std::fabs(gains[c] - 1.0f) > 1e-6f) launch(gaink, cfg1(n), out[c], gains[c], (int)n);
        // the focus slice of the frame as fused (RDF)
        luma(out, yt);
        if (!taps) {
            std::vector<Tap<float>> t = rdf_taps<float>(dp.r_in, dp.r_out);
            std::vector<float> tv;
            for (auto& q : t) tv.push_back((float)q.dy), tv.push_back((float)q.dx), tv.push_back(q.w);
            ntaps = (int)t.size();
            taps = dalloc(tv.size());
            h2d(taps, tv.data(), sizeof(float) * tv.size());
        }
        launch(rdfk, cfg2(w, h), (const float*)yt, tmp, (int)w, (int)h, (const float*)taps, ntaps);
        const size_t k = (size_t)1 << dp.scale, dw = blocks(w, k), dh = blocks(h, k);
        if (!slice) slice = dalloc(dw * dh);
        launch(bmeank, cfg2(dw, dh), (const float*)tmp, slice, (int)w, (int)h, (int)k, (int)dw, (int)dh);
        focus.resize(dw * dh);
        d2h(focus.data(), slice, sizeof(float) * dw * dh);
        return sim;
    }
};

// ------------------------------------------------------------------ the depth pass
// the multigrid constants are the oracle's (depth.rs:770-777)
struct DLevel {
    size_t w, h;
    float *wd, *ax, *ay, *dinv, *x, *b, *r;
};

// gpu.rs:1154 DWls
struct DWls {
    const Module& M;
    CUfunction edgew, coarse_wd, coarse_ax, coarse_ay, dinvk, stencil, jac0, restrictk, prolongk, dotk, scalk, axpyk, pupdk, mulk, fgs_rows,
        fgs_cols;
    std::vector<DLevel> lv;
    float *cp, *dp, *f, *r, *z, *p, *ap;
    double *acc, *scal;
    size_t readbacks = 0;
    DWls(const Module& m, const float* guide, size_t w, size_t h, float lambda, float sigma_c) : M(m) {
        edgew = M.f("edgew"), coarse_wd = M.f("coarse_wd"), coarse_ax = M.f("coarse_ax"), coarse_ay = M.f("coarse_ay"), dinvk = M.f("dinvk");
        stencil = M.f("stencil"), jac0 = M.f("jac0"), restrictk = M.f("restrictk"), prolongk = M.f("prolongk"), dotk = M.f("dotk");
        scalk = M.f("scalk"), axpyk = M.f("axpyk"), pupdk = M.f("pupdk"), mulk = M.f("mulk"), fgs_rows = M.f("fgs_rows"), fgs_cols = M.f("fgs_cols");
        auto mk = [](size_t w, size_t h) {
            const size_t n = w * h;
            return DLevel{w, h, dalloc(n), dalloc(n), dalloc(n), dalloc(n), dalloc(n), dalloc(n), dalloc(n)};
        };
        lv.push_back(mk(w, h));
        launch(edgew, cfg2(w, h), guide, lv[0].ax, lv[0].ay, (int)w, (int)h, -1.0f / std::max(sigma_c, 1e-6f), lambda);
        while (std::max(lv.back().w, lv.back().h) > MG_MIN) {
            const DLevel f0 = lv.back();
            DLevel c = mk(half(f0.w), half(f0.h));
            launch(coarse_ax, cfg2(c.w, c.h), (const float*)f0.ax, c.ax, (int)f0.w, (int)f0.h, (int)c.w, (int)c.h);
            launch(coarse_ay, cfg2(c.w, c.h), (const float*)f0.ay, c.ay, (int)f0.w, (int)f0.h, (int)c.w, (int)c.h);
            lv.push_back(c);
        }
        const size_t n = w * h;
        cp = dalloc(n), dp = dalloc(n), f = dalloc(n), r = dalloc(n), z = dalloc(n), p = dalloc(n), ap = dalloc(n);
        RT(cudaMalloc(&acc, sizeof(double)));
        RT(cudaMalloc(&scal, sizeof(double) * 5));
        RT(cudaMemset(acc, 0, sizeof(double)));
        RT(cudaMemset(scal, 0, sizeof(double) * 5));
    }
    void set_weights() {
        for (size_t l = 0; l < lv.size(); l++) {
            const DLevel& c = lv[l];
            if (l > 0) {
                const DLevel& f0 = lv[l - 1];
                launch(coarse_wd, cfg2(c.w, c.h), (const float*)f0.wd, c.wd, (int)f0.w, (int)f0.h, (int)c.w, (int)c.h);
            }
            launch(dinvk, cfg2(c.w, c.h), (const float*)c.wd, (const float*)c.ax, (const float*)c.ay, c.dinv, (int)c.w, (int)c.h);
        }
    }
    void sten(size_t l, const float* x, const float* b, float* o, int mode) {
        const DLevel& c = lv[l];
        launch(stencil, cfg2(c.w, c.h), x, b, (const float*)c.wd, (const float*)c.ax, (const float*)c.ay, (const float*)c.dinv, o, (int)c.w,
               (int)c.h, mode, MG_OMEGA);
    }
    void jacobi(size_t l, bool zero_start) {
        DLevel& c = lv[l];
        const size_t n = c.w * c.h;
        if (zero_start) {
            launch(jac0, cfg1(n), (const float*)c.b, (const float*)c.dinv, c.x, (int)n, MG_OMEGA);
        } else {
            sten(l, c.x, c.b, c.r, 2);
            std::swap(c.x, c.r);
        }
    }
    void vcycle(size_t l) {
        if (l + 1 == lv.size()) {
            for (size_t k = 0; k < MG_COARSE; k++) jacobi(l, k == 0);
            return;
        }
        for (size_t k = 0; k < MG_PRE; k++) jacobi(l, k == 0);
        sten(l, lv[l].x, lv[l].b, lv[l].r, 1);
        launch(restrictk, cfg2(lv[l + 1].w, lv[l + 1].h), (const float*)lv[l].r, lv[l + 1].b, (int)lv[l].w, (int)lv[l].h, (int)lv[l + 1].w,
               (int)lv[l + 1].h);
        vcycle(l + 1);
        launch(prolongk, cfg2(lv[l].w, lv[l].h), lv[l].x, (const float*)lv[l + 1].x, (int)lv[l].w, (int)lv[l].h, (int)lv[l + 1].w);
        for (size_t k = 0; k < MG_POST; k++) jacobi(l, false);
    }
    void dot(const float* a, const float* b, size_t n, int mode) {
        const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 1024);
        launch(dotk, Cfg{blocks, 1, 256, 1}, a, b, acc, (int)n);
        launch(scalk, Cfg{1, 1, 1, 1}, acc, scal, mode);
    }
    double scal4() {
        double s[5];
        d2h(s, scal, sizeof s);
        readbacks++;
        return s[4];
    }
    // gpu.rs:1240 `solve`
    void solve(const float* d, float* u, size_t max_iters, float* rel_out, size_t* iters_out) {
        const size_t w = lv[0].w, h = lv[0].h, n = w * h;
        d2d(f, d, sizeof(float) * n);
        const int T = 3;
        for (int t = 1; t <= T; t++) {
            const float lam_t = 1.5f * std::pow(4.0f, (float)(T - t)) / (std::pow(4.0f, (float)T) - 1.0f);
            const int unit = t != 1;
            launch(fgs_rows, cfg1(h), (const float*)f, u, (const float*)lv[0].wd, (const float*)lv[0].ax, cp, dp, (int)w, (int)h, lam_t, unit);
            d2d(f, u, sizeof(float) * n);
            launch(fgs_cols, cfg1(w), (const float*)f, u, (const float*)lv[0].wd, (const float*)lv[0].ay, cp, dp, (int)w, (int)h, lam_t, 1);
            d2d(f, u, sizeof(float) * n);
        }
        launch(mulk, cfg1(n), (const float*)lv[0].wd, d, f, (int)n);
        dot(f, f, n, 3);
        const double bnorm = std::max(std::sqrt(scal4()), 1e-30);
        sten(0, u, f, r, 1);
        auto precond = [&]() {
            d2d(lv[0].b, r, sizeof(float) * n);
            vcycle(0);
            d2d(z, lv[0].x, sizeof(float) * n);
        };
        precond();
        d2d(p, z, sizeof(float) * n);
        dot(r, z, n, 0);
        dot(r, r, n, 3);
        float res = (float)(std::sqrt(scal4()) / bnorm);
        size_t iters = 0;
        for (size_t it = 0; it < max_iters; it++) {
            if (res < 1e-5f) break;
            iters++;
            sten(0, p, f, ap, 0);
            dot(p, ap, n, 1);
            launch(axpyk, cfg1(n), u, (const float*)p, (const double*)scal, (int)n, 1.0f);
            launch(axpyk, cfg1(n), r, (const float*)ap, (const double*)scal, (int)n, -1.0f);
            dot(r, r, n, 3);
            res = (float)(std::sqrt(scal4()) / bnorm);
            if (res < 1e-5f) break;
            precond();
            dot(r, z, n, 2);
            launch(pupdk, cfg1(n), p, (const float*)z, (const double*)scal, (int)n);
        }
        *rel_out = res;
        *iters_out = iters;
    }
};

// gpu.rs:1327 `depth_from_slices` (guided filter r, guided upsampling, the WLS with one robust reweighting)
struct DepthOut {
    std::vector<float> depth, conf;
    float rel = 0.f;
    size_t iters = 0, readbacks = 0;
};
static DepthOut depth_from_slices(const Module& M, const std::vector<std::vector<float>>& slices, size_t n, const Img3<float>& fused,
                                  const DepthParams& p) {
    CUfunction bmeank = M.f("bmeank"), boxH = M.f("boxH"), boxV = M.f("boxV"), mulk = M.f("mulk"), gfvar = M.f("gfvar"), gfab = M.f("gfab");
    CUfunction gfapply = M.f("gfapply"), peak_init = M.f("peak_init"), peak_push = M.f("peak_push"), peak_finish = M.f("peak_finish");
    CUfunction median3k = M.f("median3k"), wdk = M.f("wdk"), robustk = M.f("robustk"), upbil = M.f("upbil"), upapply = M.f("upapply");
    const size_t w = fused.w, h = fused.h, k = (size_t)1 << p.scale, dw = blocks(w, k), dh = blocks(h, k), m = dw * dh;
    const int wi = (int)w, hi = (int)h, dwi = (int)dw, dhi = (int)dh, mi = (int)m;
    std::vector<float> yl = luma(fused);
    float* yfull = dalloc(w * h);
    h2d(yfull, yl.data(), sizeof(float) * w * h);
    float* guide = dalloc(m);
    launch(bmeank, cfg2(dw, dh), (const float*)yfull, guide, wi, hi, (int)k, dwi, dhi);
    float* bt = dalloc(m);
    auto boxf = [&](const float* src, float* dst, size_t r) {
        launch(boxH, cfg2(dw, dh), src, bt, dwi, dhi, (int)r);
        launch(boxV, cfg2(dw, dh), (const float*)bt, dst, dwi, dhi, (int)r);
    };
    float *mean_i = dalloc(m), *var_i = dalloc(m), *t0 = dalloc(m), *t1 = dalloc(m), *t2 = dalloc(m), *t3 = dalloc(m);
    auto stats = [&](size_t r) {
        boxf(guide, mean_i, r);
        launch(mulk, cfg1(m), (const float*)guide, (const float*)guide, t0, mi);
        boxf(t0, t1, r);
        launch(gfvar, cfg1(m), (const float*)mean_i, (const float*)t1, var_i, mi);
    };
    auto coeffs = [&](const float* src, size_t r, float eps) {
        boxf(src, t0, r);
        launch(mulk, cfg1(m), (const float*)guide, src, t1, mi);
        boxf(t1, t2, r);
        launch(gfab, cfg1(m), (const float*)t0, (const float*)t2, (const float*)mean_i, (const float*)var_i, t2, t3, eps, mi);
        boxf(t2, t1, r);
        boxf(t3, t0, r);
    };
    if (p.agg_radius > 0) stats(p.agg_radius);
    float* state = dalloc(9 * m);
    launch(peak_init, cfg1(m), state, mi);
    float *sl = dalloc(m), *agg = dalloc(m);
    for (size_t i = 0; i < n; i++) {
        const std::vector<float>& c = slices[i % slices.size()];
        h2d(sl, c.data(), sizeof(float) * m);
        if (p.agg_radius > 0) {
            coeffs(sl, p.agg_radius, p.agg_eps);
            launch(gfapply, cfg1(m), (const float*)t1, (const float*)t0, (const float*)guide, agg, mi, 1);
            launch(peak_push, cfg1(m), (const float*)agg, state, mi, (int)i);
        } else {
            launch(peak_push, cfg1(m), (const float*)sl, state, mi, (int)i);
        }
    }
    sync();
    std::vector<float> cmin(m);
    d2h(cmin.data(), state + 7 * m, sizeof(float) * m);
    std::vector<float> mins;
    for (size_t i = 0; i < m; i += 7) mins.push_back(cmin[i]);
    const float floor_v = select_nth(mins, mins.size() / 2);
    float *d = sl, *conf = agg;
    launch(peak_finish, cfg1(m), state, t2, conf, mi, (int)n, floor_v, p.gate);
    if (p.median) launch(median3k, cfg2(dw, dh), (const float*)t2, d, dwi, dhi);
    else d2d(d, t2, sizeof(float) * m);
    std::vector<float> conf_h(m);
    d2h(conf_h.data(), conf, sizeof(float) * m);
    normalize_conf(conf_h);
    h2d(conf, conf_h.data(), sizeof(float) * m);
    float* u = dalloc(m);
    DepthOut o;
    if (p.lambda > 0.f) {
        const float EPS_DATA = 1e-4f;
        DWls wls(M, guide, dw, dh, p.lambda, p.sigma_c);
        launch(wdk, cfg1(m), (const float*)conf, wls.lv[0].wd, mi, 1.0f, EPS_DATA);
        wls.set_weights();
        wls.solve(d, u, p.cg_iters, &o.rel, &o.iters);
        if (p.robust > 0.f) {
            launch(robustk, cfg1(m), (const float*)conf, (const float*)d, (const float*)u, wls.lv[0].wd, mi, p.robust, EPS_DATA);
            wls.set_weights();
            wls.solve(d, u, p.cg_iters, &o.rel, &o.iters);
        }
        o.readbacks = wls.readbacks;
    } else {
        d2d(u, d, sizeof(float) * m);
    }
    sync();
    const float max_d = (float)(n - 1);
    float* full = dalloc(w * h);
    stats(p.up_radius);
    coeffs(u, p.up_radius, p.up_eps);
    launch(upapply, cfg2(w, h), (const float*)t1, (const float*)t0, (const float*)yfull, full, wi, hi, dwi, dhi, (int)k, max_d);
    o.depth.resize(w * h);
    d2h(o.depth.data(), full, sizeof(float) * w * h);
    launch(upbil, cfg2(w, h), (const float*)conf, full, wi, hi, dwi, dhi, (int)k);
    o.conf.resize(w * h);
    d2h(o.conf.data(), full, sizeof(float) * w * h);
    for (float* q : {yfull, guide, bt, mean_i, var_i, t0, t1, t2, t3, state, sl, agg, u, full}) cudaFree(q);
    return o;
}

int main(int argc, char** argv) {
    if (argc < 9) {
        fprintf(stderr, "usage: %s fuse.ptx depth.ptx w h n_total n_sample coarsen agg_radius [seed] [--check] [--noalign]\n", argv[0]);
        return 2;
    }
    const size_t w = strtoul(argv[3], nullptr, 10), h = strtoul(argv[4], nullptr, 10);
    const size_t n_total = strtoul(argv[5], nullptr, 10), n_sample = std::min(strtoul(argv[6], nullptr, 10), n_total);
    const size_t coarsen = strtoul(argv[7], nullptr, 10), agg_r = strtoul(argv[8], nullptr, 10);
    const uint64_t seed = argc > 9 && argv[9][0] != '-' ? strtoull(argv[9], nullptr, 0) : 0x1A957ACCull;
    bool check = false, noalign = false;
    for (int i = 9; i < argc; i++) {
        check |= strcmp(argv[i], "--check") == 0;
        noalign |= strcmp(argv[i], "--noalign") == 0;
    }
    if (n_sample < 2) {  // frame 0 has no search
        fprintf(stderr, "n_sample must be at least 2\n");
        return 2;
    }
    RT(cudaSetDevice(0));
    RT(cudaFree(nullptr));
    CU(cuStreamCreate(&g_s, CU_STREAM_NON_BLOCKING));
    const double t_load = now_ms();
    Module fuse_m(argv[1]), depth_m(argv[2]);
    const double load_ms = now_ms() - t_load;
    // the benchmark's synthetic stack (aligned: a seeded similarity warp per frame), made one frame at a time
    SynthDesc sd{(uint32_t)w, (uint32_t)h, (uint32_t)n_total, noalign ? 0u : 1u, seed, 0.0f, 0.002f, 6.0f, 0.004f, 0.2f, 8.0f};
    std::vector<double> truth(4 * n_total);
    std::vector<uint16_t> raw(w * h * 3);
    std::vector<std::vector<uint16_t>> kept;  // the frames, for the check
    auto frame_of = [&](size_t i) {
        if (!synth_stack(sd, raw.data(), truth.data(), (uint32_t)i, 1)) {
            fprintf(stderr, "synth failed\n");
            exit(2);
        }
        if (check) kept.push_back(raw);
        return img_of_u16<float>(raw.data(), w, h);
    };
    FuseParams fp;
    DepthParams dp;
    dp.agg_radius = agg_r;
    AlignParams ap;
    ap.coarsen = coarsen;
    bool freem[8];
    free_mask(ap, freem);
    if (noalign)
        for (bool& b : freem) b = false;
    // a warm-up pass over two frames (first launches, allocations), then the timed run
    {
        Frames F(fuse_m, w, h, ap.interp);
        RefFuser U(fuse_m, w, h, fp);
        float g[3];
        std::vector<float> foc;
        Img3<float> f0 = frame_of(0), f1 = frame_of(1);
        kept.clear();
        Sim s = F.process(f0, Sim(), freem, coarsen, dp, g, foc);
        U.push_device(F.out);
        s = F.process(f1, s, freem, coarsen, dp, g, foc);
        U.push_device(F.out);
        sync();
    }
    Frames F(fuse_m, w, h, ap.interp);
    RefFuser U(fuse_m, w, h, fp);
    std::vector<std::vector<float>> slices(n_sample);
    std::vector<Sim> sims;
    std::vector<double> frame_ms, fold_ms;
    Sim guess;
    double upload_ms = 0;
    for (size_t i = 0; i < n_sample; i++) {
        const Img3<float> fr = frame_of(i);
        if (i == 1) {  // the planes' upload (pageable, as the reference's Vec<f32> frames) timed on its own
            const double tu = now_ms();
            for (int c = 0; c < 3; c++) h2d(F.yt, fr.p[c].data(), sizeof(float) * w * h);
            sync();
            upload_ms = now_ms() - tu;
        }
        const double t0 = now_ms();
        float g[3];
        guess = F.process(fr, guess, freem, coarsen, dp, g, slices[i]);
        sync();
        const double t1 = now_ms();
        U.push_device(F.out);
        sync();
        const double t2 = now_ms();
        frame_ms.push_back(t2 - t0);
        fold_ms.push_back(t2 - t1);
        sims.push_back(guess);
    }
    double t0 = now_ms();
    Img3<float> img = U.finish(fp);
    sync();
    const double finish_ms = now_ms() - t0;
    t0 = now_ms();
    DepthOut dout = depth_from_slices(depth_m, slices, n_total, img, dp);
    sync();
    const double depth_ms = now_ms() - t0;
    double later = 0, fold_later = 0;
    for (size_t i = 1; i < n_sample; i++) later += frame_ms[i], fold_later += fold_ms[i];
    later /= (double)(n_sample - 1);
    fold_later /= (double)(n_sample - 1);
    const double evals_per_frame = (double)F.evals / (double)(n_sample - 1);
    const double total = frame_ms[0] + (double)(n_total - 1) * later + finish_ms + depth_ms;
    printf("{\"w\": %zu, \"h\": %zu, \"n_total\": %zu, \"n_sample\": %zu, \"module_load_ms\": %.1f, \"frame0_ms\": %.3f, "
           "\"frame_ms\": %.3f, \"fold_ms_per_frame\": %.3f, \"upload_ms_per_frame\": %.3f, \"evals_per_frame\": %.1f, "
           "\"finish_ms\": %.3f, \"depth_ms\": %.3f, \"wls_iters\": %zu, \"wls_rel\": %.3g, \"wls_readbacks\": %zu, "
           "\"total_ms_extrapolated\": %.1f, \"total_ms_without_uploads\": %.1f",
           w, h, n_total, n_sample, load_ms, frame_ms[0], later, fold_later, upload_ms, evals_per_frame, finish_ms, depth_ms, dout.iters,
           dout.rel, dout.readbacks, total, total - (double)n_total * upload_ms);
    if (check) {
        // the oracle (the reference's CPU path, FP32) over the same frames: transforms and the fused image
        StackParams sp;
        sp.align = !noalign;
        sp.al = ap;
        sp.depth = false;
        std::vector<const uint16_t*> fr;
        for (size_t i = 0; i < n_sample; i++) fr.push_back(kept[i].data());
        StackOutput<float> ref = run_stack<float>(fr.data(), n_sample, w, h, sp);
        double dsim = 0, dimg = 0, dsum = 0;
        size_t over = 0;
        for (size_t i = 0; i < n_sample; i++)
            for (int k = 0; k < 8; k++) dsim = std::max(dsim, std::fabs(ref.sims[i].v[k] - sims[i].v[k]));
        for (int c = 0; c < 3; c++)
            for (size_t i = 0; i < w * h; i++) {
                const double d = std::fabs((double)ref.image.p[c][i] - (double)img.p[c][i]);
                dimg = std::max(dimg, d);
                dsum += d;
                over += d > 1e-3;
            }
        printf(", \"check_max_sim_diff\": %.3g, \"check_max_image_diff\": %.3g, \"check_mean_image_diff\": %.3g, "
               "\"check_frac_over_1e-3\": %.3g",
               dsim, dimg, dsum / (3.0 * w * h), (double)over / (3.0 * w * h));
    }
    printf("}\n");
    return 0;
}
