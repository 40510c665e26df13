// Oracle C API (test infrastructure only; see orc_core.hpp). Loaded by the
// tests, smoke() and bench.py's CPU legs through ctypes (oracle/oracle.py).
// Parameter blocks are flat double arrays, laid out in oracle/oracle.py.
#include <array>
#include "orc_stack.hpp"
#include "orc_synth.hpp"
#include "orc_dust.hpp"
#include <omp.h>

using namespace orc;

namespace {

FuseParams fuse_of(const double* a) {
    FuseParams p;
    p.levels = (size_t)a[0];
    p.energy_radius = (size_t)a[1];
    p.top_rule = (int)a[2];
    p.top_radius = (size_t)a[3];
    p.entropy_bins = (size_t)a[4];
    p.use_chroma = a[5] != 0.0;
    p.depth_level = (size_t)a[6];
    p.halo = (float)a[7];
    return p;
}
AlignParams align_of(const double* a) {
    AlignParams p;
    p.shift = a[0] != 0.0;
    p.scale = a[1] != 0.0;
    p.rotation = a[2] != 0.0;
    p.model = (int)a[3];
    p.coarsen = (size_t)a[4];
    p.interp = (int)a[5];
    return p;
}
DepthParams depth_of(const double* a) {
    DepthParams p;
    p.scale = (size_t)a[0];
    p.focus = (int)a[1];
    p.r_in = (size_t)a[2];
    p.r_out = (size_t)a[3];
    p.sml_step = (size_t)a[4];
    p.agg_radius = (size_t)a[5];
    p.agg_eps = (float)a[6];
    p.lambda = (float)a[7];
    p.sigma_c = (float)a[8];
    p.cg_iters = (size_t)a[9];
    p.median = a[10] != 0.0;
    p.upsample = (int)a[11];
    p.up_radius = (size_t)a[12];
    p.up_eps = (float)a[13];
    p.gate = (float)a[14];
    p.robust = (float)a[15];
    return p;
}
Sim sim_of(const double* v) {
    Sim s;
    for (int k = 0; k < 8; k++) s.v[k] = v[k];
    return s;
}
template <class T>
Img3<T> img_of(const T* planes, size_t w, size_t h) {
    Img3<T> im(w, h);
    for (int c = 0; c < 3; c++) std::copy(planes + c * w * h, planes + (c + 1) * w * h, im.p[c].begin());
    return im;
}
template <class T>
void put_img(const Img3<T>& im, T* out) {
    for (int c = 0; c < 3; c++) std::copy(im.p[c].begin(), im.p[c].end(), out + c * im.w * im.h);
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------ pyramid
size_t orc_reflect(long i, size_t n) { return reflect(i, n); }
size_t orc_auto_levels(size_t w, size_t h, size_t min_top) { return auto_levels(w, h, min_top); }
void orc_reduce_f(const float* src, size_t w, size_t h, float* out) {
    std::vector<float> o;
    size_t ow, oh;
    reduce<float>(src, w, h, o, ow, oh);
    std::copy(o.begin(), o.end(), out);
}
void orc_expand_f(const float* c, size_t cw, size_t ch, size_t ow, size_t oh, float* out) {
    std::vector<float> o = expand<float>(c, cw, ch, ow, oh);
    std::copy(o.begin(), o.end(), out);
}
// build then collapse (pyramid.rs:282 perfect reconstruction)
void orc_build_collapse_f(const float* planes, size_t w, size_t h, size_t levels, float* out) {
    Img3<float> im = img_of(planes, w, h);
    put_img(collapse(build(im, levels)), out);
}

// --------------------------------------------------------------------- fuse
void orc_binomial_f(size_t r, float* out) {
    std::vector<float> b = binomial<float>(r);
    std::copy(b.begin(), b.end(), out);
}
void orc_window_sum_f(const float* src, size_t w, size_t h, const float* wt, size_t klen, float* out) {
    std::vector<float> o = window_sum<float>(src, w, h, std::vector<float>(wt, wt + klen));
    std::copy(o.begin(), o.end(), out);
}
void orc_region_energy_f(const float* planes, size_t w, size_t h, size_t radius, int use_chroma, float* out) {
    std::vector<float> o = region_energy(img_of(planes, w, h), radius, use_chroma != 0);
    std::copy(o.begin(), o.end(), out);
}
float orc_halo_weight(float re, float p) { return halo_weight<float>(re, p); }
void orc_winner_shares(const uint16_t* win, const float* best, size_t cells, size_t frames, float* out) {
    std::vector<float> s = winner_shares(win, best, cells, frames);
    std::copy(s.begin(), s.end(), out);
}
void orc_deviation_entropy_f(const float* y, size_t w, size_t h, size_t radius, size_t bins, float* dev, float* ent) {
    std::vector<float> d, e;
    deviation_entropy<float>(y, w, h, radius, bins, d, e);
    std::copy(d.begin(), d.end(), dev);
    std::copy(e.begin(), e.end(), ent);
}
void orc_fuse_residuals_f(const float* tops, size_t n, size_t w, size_t h, const double* fp, float* out) {
    std::vector<Img3<float>> t;
    for (size_t k = 0; k < n; k++) t.push_back(img_of(tops + k * 3 * w * h, w, h));
    put_img(fuse_residuals(t, fuse_of(fp)), out);
}

#define FUSER_API(S, T)                                                                                    \
    void* orc_fuser_new_##S(size_t w, size_t h, const double* fp) { return new Fuser<T>(w, h, fuse_of(fp)); } \
    size_t orc_fuser_levels_##S(void* f) { return ((Fuser<T>*)f)->levels; }                                  \
    void orc_fuser_push_##S(void* f, const T* planes) {                                                       \
        Fuser<T>* F = (Fuser<T>*)f;                                                                           \
        F->push(img_of(planes, F->w, F->h));                                                                  \
    }                                                                                                         \
    size_t orc_fuser_shares_##S(void* f, float* out) {                                                        \
        std::vector<float> s = ((Fuser<T>*)f)->shares();                                                      \
        std::copy(s.begin(), s.end(), out);                                                                   \
        return s.size();                                                                                      \
    }                                                                                                         \
    void orc_fuser_winner_##S(void* f, uint16_t* out) {                                                       \
        auto& w = ((Fuser<T>*)f)->winner;                                                                     \
        std::copy(w.begin(), w.end(), out);                                                                   \
    }                                                                                                         \
    void orc_fuser_finish_##S(void* f, T* img, float* depth) {                                                \
        Img3<T> im;                                                                                           \
        std::vector<float> d;                                                                                 \
        ((Fuser<T>*)f)->finish(im, d);                                                                        \
        put_img(im, img);                                                                                     \
        std::copy(d.begin(), d.end(), depth);                                                                 \
    }                                                                                                         \
    void orc_fuser_free_##S(void* f) { delete (Fuser<T>*)f; }
FUSER_API(f, float)
FUSER_API(d, double)

// -------------------------------------------------------------------- align
void orc_sim_matrix(const double* sim8, size_t w, size_t h, double* m9) {
    Mat3 m;
    sim_matrix(sim_of(sim8), w, h, m);
    for (int i = 0; i < 9; i++) m9[i] = m[i / 3][i % 3];
}
void orc_mat_inverse(const double* m9, double* inv9) {
    Mat3 m, inv;
    for (int i = 0; i < 9; i++) m[i / 3][i % 3] = m9[i];
    mat_inverse(m, inv);
    for (int i = 0; i < 9; i++) inv9[i] = inv[i / 3][i % 3];
}
int orc_interp_weights(int k, double t, double* w6) { return interp_weights(k, t, w6); }
void orc_spline4f(float t, float* w4) { spline4f<float>(t, w4); }
void orc_warp_plane_f(const float* src, size_t w, size_t h, const double* sim8, size_t ow, size_t oh, int interp, float* out,
                      uint8_t* valid) {
    std::vector<float> o;
    std::vector<uint8_t> v;
    warp_plane<float>(src, w, h, sim_of(sim8), ow, oh, interp, o, valid ? &v : nullptr);
    std::copy(o.begin(), o.end(), out);
    if (valid) std::copy(v.begin(), v.end(), valid);
}
double orc_warp_cost_f(const float* rf, size_t aw, size_t ah, const float* tgt, size_t tw, size_t th, const double* sim8) {
    return warp_cost<float>(rf, aw, ah, tgt, tw, th, sim_of(sim8));
}
void orc_reduce_burt_f(const float* src, size_t w, size_t h, float* out) {
    std::vector<float> o;
    size_t ow, oh;
    reduce_burt<float>(src, w, h, o, ow, oh);
    std::copy(o.begin(), o.end(), out);
}
// all levels of align.rs:741 `gauss_levels`, concatenated; returns the count
size_t orc_gauss_levels_f(const float* y, size_t w, size_t h, size_t* dims, float* out) {
    std::vector<Lvl<float>> lv = gauss_levels<float>(y, w, h);
    size_t o = 0;
    for (size_t l = 0; l < lv.size(); l++) {
        dims[2 * l] = lv[l].w;
        dims[2 * l + 1] = lv[l].h;
        if (out) std::copy(lv[l].d.begin(), lv[l].d.end(), out + o);
        o += lv[l].d.size();
    }
    return lv.size();
}
void orc_level_steps(const size_t* free_idx, size_t nfree, size_t lvl, size_t w, size_t h, double* step, double* tol) {
    std::vector<double> s, t;
    level_steps(std::vector<size_t>(free_idx, free_idx + nfree), lvl, w, h, s, t);
    std::copy(s.begin(), s.end(), step);
    std::copy(t.begin(), t.end(), tol);
}
typedef double (*orc_cost_fn)(const double* x, size_t n);
void orc_nelder_mead(orc_cost_fn f, size_t n, const double* x0, const double* lo, const double* hi, const double* step,
                     const double* tol, double* out, size_t* evals) {
    auto F = [&](const std::vector<double>& v) { return f(v.data(), v.size()); };
    size_t ne = 0;
    std::vector<double> r = nelder_mead(F, std::vector<double>(x0, x0 + n), std::vector<double>(lo, lo + n),
                                        std::vector<double>(hi, hi + n), std::vector<double>(step, step + n),
                                        std::vector<double>(tol, tol + n), &ne);
    std::copy(r.begin(), r.end(), out);
    if (evals) *evals = ne;
}
// The oracle's Nelder-Mead step counts (orc::g_nm_steps) into out5; reset clears them after reading.
void orc_nm_step_kinds(size_t* out5, int reset) {
    for (int k = 0; k < 5; k++) out5[k] = reset ? orc::g_nm_steps[k].exchange(0) : orc::g_nm_steps[k].load();
}

void orc_multiscale_align_f(const float* rf, const float* tg, size_t w, size_t h, const double* init8, const uint8_t* free8,
                            size_t coarsen, double* out8, size_t* evals) {
    bool fr[8];
    for (int k = 0; k < 8; k++) fr[k] = free8[k] != 0;
    size_t ne = 0;
    Sim s = multiscale_align<float>(rf, tg, w, h, sim_of(init8), fr, coarsen, &ne);
    for (int k = 0; k < 8; k++) out8[k] = s.v[k];
    if (evals) *evals = ne;
}
void orc_common_area(const double* sims, size_t n, size_t w, size_t h, int interp, size_t* rect4) {
    std::vector<Sim> v;
    for (size_t i = 0; i < n; i++) v.push_back(sim_of(sims + 8 * i));
    Rect r = common_area(v, w, h, interp);
    rect4[0] = r.x;
    rect4[1] = r.y;
    rect4[2] = r.w;
    rect4[3] = r.h;
}
// brightness.rs:57 `Reference::gains` of `frame` (already warped by sim) to `ref`
void orc_brightness_gains_f(const float* ref3, const float* frame3, size_t w, size_t h, const double* sim8, float* g3) {
    BReference<float> r;
    r.init(img_of(ref3, w, h));
    double sf[3], so[3];
    size_t n;
    bsums<float>(img_of(frame3, w, h), &r, sim_of(sim8), sf, so, n);
    bratio(so, sf, n, g3);
}
void orc_brightness_gains_to_f(const float* ref3, const float* frame3, size_t w, size_t h, float* g3) {
    double rm[3], fm[3];
    bmeans<float>(img_of(ref3, w, h), rm);
    bmeans<float>(img_of(frame3, w, h), fm);
    bratio(rm, fm, (size_t)-1, g3);
}

// -------------------------------------------------------------------- depth
void orc_box_mean_f(const float* src, size_t w, size_t h, size_t r, float* out) {
    BoxFilter<float> bf(w, h, r);
    bf.mean_into(src, out);
}
void orc_guided_filter_f(const float* guide, const float* p, size_t w, size_t h, size_t r, float eps, float* out) {
    GuidedFilter<float> gf(std::vector<float>(guide, guide + w * h), w, h, r, eps);
    gf.filter_into(p, out);
}
size_t orc_rdf_taps_f(size_t r_in, size_t r_out, float* out3) {
    std::vector<Tap<float>> t = rdf_taps<float>(r_in, r_out);
    for (size_t i = 0; i < t.size(); i++) {
        out3[3 * i] = (float)t[i].dy;
        out3[3 * i + 1] = (float)t[i].dx;
        out3[3 * i + 2] = t[i].w;
    }
    return t.size();
}
void orc_focus_measure_f(const float* y, size_t w, size_t h, const double* dp, float* out) {
    std::vector<float> f = focus_measure<float>(y, w, h, depth_of(dp));
    std::copy(f.begin(), f.end(), out);
}
void orc_focus_slice_f(const float* planes, size_t w, size_t h, const double* dp, float* out) {
    size_t dw, dh;
    std::vector<float> s = focus_slice<float>(img_of(planes, w, h), depth_of(dp), dw, dh);
    std::copy(s.begin(), s.end(), out);
}
void orc_block_mean_f(const float* src, size_t w, size_t h, size_t k, float* out) {
    size_t dw, dh;
    std::vector<float> s = block_mean<float>(src, w, h, k, dw, dh);
    std::copy(s.begin(), s.end(), out);
}
void orc_upsample_bilinear_f(const float* g, size_t dw, size_t dh, size_t w, size_t h, size_t k, float* out) {
    std::vector<float> s = upsample_bilinear<float>(g, dw, dh, w, h, k);
    std::copy(s.begin(), s.end(), out);
}
void orc_peak_track_f(const float* slices, size_t n, size_t m, float gate, float* depth, float* conf, float* mins, float* floor_) {
    PeakTracker<float> t(m);
    for (size_t k = 0; k < n; k++) t.push(slices + k * m);
    std::vector<float> d, c, mn;
    float fl;
    t.finish(gate, d, c, mn, fl);
    std::copy(d.begin(), d.end(), depth);
    std::copy(c.begin(), c.end(), conf);
    if (mins) std::copy(mn.begin(), mn.end(), mins);
    if (floor_) *floor_ = fl;
}
float orc_normalize_conf_f(float* conf, size_t n) {
    std::vector<float> c(conf, conf + n);
    float p = normalize_conf(c);
    std::copy(c.begin(), c.end(), conf);
    return p;
}
void orc_median3_f(const float* src, size_t w, size_t h, float* out) {
    std::vector<float> o = median3<float>(src, w, h);
    std::copy(o.begin(), o.end(), out);
}
#define WLS_API(S, T)                                                                                                   \
    void orc_wls_solve_##S(const T* d, const T* conf, const T* guide, size_t w, size_t h, T lambda, T sigma_c, size_t iters, \
                           T* u, T* rel, size_t* it, int edge_mode) {                                                   \
        WlsSolver<T> s(guide, w, h, lambda, sigma_c, edge_mode);                                                        \
        s.set_weights(conf);                                                                                            \
        std::fill(u, u + w * h, T(0));                                                                                  \
        auto r = s.solve(d, iters, u);                                                                                  \
        if (rel) *rel = r.first;                                                                                        \
        if (it) *it = r.second;                                                                                         \
    }                                                                                                                   \
    size_t orc_wls_levels_##S(const T* guide, size_t w, size_t h) {                                                     \
        WlsSolver<T> s(guide, w, h, T(1), T(0.04));                                                                     \
        return s.levels.size();                                                                                         \
    }
WLS_API(f, float)
WLS_API(d, double)

// depth.rs:1119; stats = [floor, p90, rel, iters, iters_first, dw, dh]
#define DFS_API(S, T)                                                                                                \
    void orc_depth_from_slices_##S(const T* slices, size_t n, size_t m, const T* fused3, size_t w, size_t h,       \
                                   const double* dp, T* depth, T* conf, T* floor_cells, double* stats) {           \
        std::vector<std::vector<T>> sl;                                                                              \
        for (size_t k = 0; k < n; k++) sl.emplace_back(slices + k * m, slices + (k + 1) * m);                        \
        DepthMap<T> d = depth_from_slices<T>(sl, img_of(fused3, w, h), depth_of(dp));                                \
        std::copy(d.depth.begin(), d.depth.end(), depth);                                                            \
        std::copy(d.conf.begin(), d.conf.end(), conf);                                                               \
        if (floor_cells) std::copy(d.floor_cells.begin(), d.floor_cells.end(), floor_cells);                        \
        double st[7] = {(double)d.floor_, (double)d.p90, (double)d.rel, (double)d.iters, (double)d.iters_first,      \
                        (double)d.dw, (double)d.dh};                                                                 \
        std::copy(st, st + 7, stats);                                                                                \
    }
DFS_API(f, float)
DFS_API(d, double)

// -------------------------------------------------------------------- stack
// sp = fuse[8] | align[6] | depth[16] | flags[4] = (align_on, depth_on, brightness, crop)
struct StackRes {
    StackOutput<float> f;
    StackOutput<double> d;
    bool dbl;
    size_t n, w, h;
};
static StackParams stack_params_of(const double* sp) {
    StackParams p;
    p.fuse = fuse_of(sp);
    p.al = align_of(sp + 8);
    p.dp = depth_of(sp + 14);
    p.align = sp[30] != 0.0;
    p.depth = sp[31] != 0.0;
    p.brightness = sp[32] != 0.0;
    p.crop = sp[33] != 0.0;
    p.wav = sp[34] != 0.0;
    p.wp.power = (float)sp[35];
    p.wp.smooth = (size_t)sp[36];
    p.wp.gate = (float)sp[37];
    p.wp.edge = sp[38] != 0.0;
    p.storage = (int)sp[39];
    p.slab_size = (size_t)sp[40];
    p.slab_overlap = (size_t)sp[41];
    return p;
}
void* orc_run_stack(const uint16_t* frames, size_t n, size_t w, size_t h, const double* sp, int fp64) {
    std::vector<const uint16_t*> fr(n);
    for (size_t i = 0; i < n; i++) fr[i] = frames + i * w * h * 3;
    StackRes* r = new StackRes();
    r->dbl = fp64 != 0;
    r->n = n;
    r->w = w;
    r->h = h;
    if (r->dbl) r->d = run_stack<double>(fr.data(), n, w, h, stack_params_of(sp));
    else r->f = run_stack<float>(fr.data(), n, w, h, stack_params_of(sp));
    return r;
}
void orc_stack_free(void* p) { delete (StackRes*)p; }
// fused image as planar f64 (exact for both precisions) and as interleaved u16
void orc_stack_image(void* p, double* planes, uint16_t* rgb) {
    StackRes* r = (StackRes*)p;
    size_t n = r->w * r->h;
    for (int c = 0; c < 3; c++)
        for (size_t i = 0; i < n; i++) {
            double v = r->dbl ? r->d.image.p[c][i] : (double)r->f.image.p[c][i];
            if (planes) planes[c * n + i] = v;
            if (rgb) rgb[3 * i + c] = r->dbl ? u16_of<double>(r->d.image.p[c][i]) : u16_of<float>(r->f.image.p[c][i]);
        }
}
void orc_stack_winner(void* p, float* out) {
    StackRes* r = (StackRes*)p;
    auto& v = r->dbl ? r->d.winner : r->f.winner;
    std::copy(v.begin(), v.end(), out);
}
// depth, conf at full resolution; floor cells on the working grid
void orc_stack_depth(void* p, double* depth, double* conf, double* floor_cells) {
    StackRes* r = (StackRes*)p;
    if (r->dbl) {
        std::copy(r->d.dm.depth.begin(), r->d.dm.depth.end(), depth);
        std::copy(r->d.dm.conf.begin(), r->d.dm.conf.end(), conf);
        if (floor_cells) std::copy(r->d.dm.floor_cells.begin(), r->d.dm.floor_cells.end(), floor_cells);
    } else {
        std::copy(r->f.dm.depth.begin(), r->f.dm.depth.end(), depth);
        std::copy(r->f.dm.conf.begin(), r->f.dm.conf.end(), conf);
        if (floor_cells) std::copy(r->f.dm.floor_cells.begin(), r->f.dm.floor_cells.end(), floor_cells);
    }
}
// [levels, dw, dh, floor, p90, rel, iters, iters_first, align_evals, crop x, y, w, h]
void orc_stack_stats(void* p, double* st) {
    StackRes* r = (StackRes*)p;
    auto fill = [&](auto& o) {
        double v[13] = {(double)o.levels, (double)o.dm.dw, (double)o.dm.dh, (double)o.dm.floor_, (double)o.dm.p90,
                        (double)o.dm.rel, (double)o.dm.iters, (double)o.dm.iters_first, (double)o.align_evals,
                        (double)o.crop.x, (double)o.crop.y, (double)o.crop.w, (double)o.crop.h};
        std::copy(v, v + 13, st);
    };
    if (r->dbl) fill(r->d);
    else fill(r->f);
}
void orc_stack_sims(void* p, double* sims8, float* gains3, float* shares) {
    StackRes* r = (StackRes*)p;
    auto fill = [&](auto& o) {
        for (size_t i = 0; i < o.sims.size(); i++) {
            for (int k = 0; k < 8; k++) sims8[8 * i + k] = o.sims[i].v[k];
            for (int c = 0; c < 3; c++) gains3[3 * i + c] = o.gains[i][c];
        }
        if (shares) std::copy(o.shares.begin(), o.shares.end(), shares);
        return o.shares.size();
    };
    if (r->dbl) fill(r->d);
    else fill(r->f);
}

// ---- the stack one frame at a time (the CPU baseline times the per-frame work and the finish apart)
struct StackInc {
    bool dbl;
    size_t n, w, h;
    StackRun<float>* f = nullptr;
    StackRun<double>* d = nullptr;
    ~StackInc() {
        delete f;
        delete d;
    }
};
void* orc_stack_begin(size_t n, size_t w, size_t h, const double* sp, int fp64) {
    StackInc* s = new StackInc();
    s->dbl = fp64 != 0;
    s->n = n;
    s->w = w;
    s->h = h;
    if (s->dbl) s->d = new StackRun<double>(w, h, n, stack_params_of(sp));
    else s->f = new StackRun<float>(w, h, n, stack_params_of(sp));
    return s;
}
void orc_stack_push(void* p, const uint16_t* frame, int last) {
    StackInc* s = (StackInc*)p;
    if (s->dbl) s->d->push(frame, last != 0);
    else s->f->push(frame, last != 0);
}
// For timing only: the focus slices pushed so far repeated in order until there are n_total, so that
// the depth pass runs over a whole stack's slices after a sample of its frames was pushed.
void orc_stack_cycle_slices(void* p, size_t n_total) {
    StackInc* s = (StackInc*)p;
    auto grow = [&](auto& sl) {
        const size_t k = sl.size();
        for (size_t i = k; i < n_total && k > 0; i++) sl.push_back(sl[i % k]);
    };
    if (s->dbl) grow(s->d->slices);
    else grow(s->f->slices);
}
// Finishes and frees the handle; the result is read with the orc_stack_* accessors and freed by orc_stack_free.
void* orc_stack_end(void* p) {
    StackInc* s = (StackInc*)p;
    StackRes* r = new StackRes();
    r->dbl = s->dbl;
    r->w = s->w;
    r->h = s->h;
    if (s->dbl) {
        s->d->finish();
        r->n = s->d->out.sims.size();
        r->d = std::move(s->d->out);
    } else {
        s->f->finish();
        r->n = s->f->out.sims.size();
        r->f = std::move(s->f->out);
    }
    delete s;
    return r;
}
void orc_stack_abort(void* p) { delete (StackInc*)p; }

// wav.rs:92 weighted_average over n planar f32 frames [n][3][h][w]; dp as depth_of reads it; wp = [power,
// smooth, gate, edge]; floor on the depth grid; guide planar [3][h][w] or null
void orc_weighted_average_f(const float* frames, size_t n, size_t w, size_t h, const double* dp, const double* wp, const float* floor,
                            const float* guide, float* out) {
    std::vector<Img3<float>> fr(n, Img3<float>(w, h));
    for (size_t k = 0; k < n; k++)
        for (int c = 0; c < 3; c++) std::copy(frames + (k * 3 + c) * w * h, frames + (k * 3 + c + 1) * w * h, fr[k].p[c].begin());
    DepthParams d = depth_of(dp);
    WavParams p;
    p.power = (float)wp[0];
    p.smooth = (size_t)wp[1];
    p.gate = (float)wp[2];
    p.edge = wp[3] != 0.0;
    const size_t k = (size_t)1 << d.scale;
    std::vector<float> fl(floor, floor + blocks(w, k) * blocks(h, k));
    Img3<float> g(w, h);
    if (guide)
        for (int c = 0; c < 3; c++) std::copy(guide + c * w * h, guide + (c + 1) * w * h, g.p[c].begin());
    Img3<float> o = weighted_average<float>(fr, d, p, fl, guide ? &g : nullptr);
    for (int c = 0; c < 3; c++) std::copy(o.p[c].begin(), o.p[c].end(), out + c * w * h);
}

// the weighted average (planar f64, exact for both precisions); 0 when the run made none
int orc_stack_wav(void* p, double* planes) {
    StackRes* r = (StackRes*)p;
    auto fill = [&](auto& o) {
        if (o.wav.w == 0) return 0;
        const size_t n = o.wav.w * o.wav.h;
        for (int c = 0; c < 3; c++)
            for (size_t i = 0; i < n; i++) planes[c * n + i] = (double)o.wav.p[c][i];
        return 1;
    };
    return r->dbl ? fill(r->d) : fill(r->f);
}

// the slabs of the run: their count; with lohi, (lo, hi) pairs; with planes, each slab's fused image
// (planar f64 [k][3][h][w], exact for both precisions)
size_t orc_stack_slabs(void* p, uint64_t* lohi, double* planes) {
    StackRes* r = (StackRes*)p;
    auto fill = [&](auto& o) {
        const size_t n = r->w * r->h;
        for (size_t k = 0; k < o.slabs.size(); k++) {
            if (lohi) {
                lohi[2 * k] = o.slab_rng[k][0];
                lohi[2 * k + 1] = o.slab_rng[k][1];
            }
            if (planes)
                for (int c = 0; c < 3; c++)
                    for (size_t i = 0; i < n; i++) planes[(k * 3 + c) * n + i] = (double)o.slabs[k].p[c][i];
        }
        return o.slabs.size();
    };
    return r->dbl ? fill(r->d) : fill(r->f);
}

// stack.rs:76 slab_ranges: the count; the first max (lo, hi) pairs into lohi
size_t orc_slab_ranges(size_t count, size_t size, size_t overlap, uint64_t* lohi, size_t max) {
    auto v = slab_ranges(count, size, overlap);
    for (size_t k = 0; k < v.size() && k < max; k++) {
        lohi[2 * k] = v[k][0];
        lohi[2 * k + 1] = v[k][1];
    }
    return v.size();
}

// prep.rs:63 resize_plane (f32) of `planes` planes pw x ph -> w x h
void orc_resize_f(const float* src, size_t planes, size_t pw, size_t ph, size_t w, size_t h, int interp, float* out) {
    for (size_t c = 0; c < planes; c++) {
        std::vector<float> o = resize_plane<float>(src + c * pw * ph, pw, ph, w, h, interp);
        std::copy(o.begin(), o.end(), out + c * w * h);
    }
}

// a dust map from flat arrays: rects [n][4] (x, y, w, h), the masks and (flat mode) the gains concatenated
static DustMap dust_of(const uint64_t* rects, size_t n, const uint8_t* masks, const float* gains, size_t mw, size_t mh, int mode) {
    DustMap m;
    m.w = mw;
    m.h = mh;
    m.mode = mode;
    size_t off = 0;
    for (size_t k = 0; k < n; k++) {
        DustSpot s;
        s.x = rects[4 * k];
        s.y = rects[4 * k + 1];
        s.w = rects[4 * k + 2];
        s.h = rects[4 * k + 3];
        s.mask.assign(masks + off, masks + off + s.w * s.h);
        if (gains) s.gain.assign(gains + off, gains + off + s.w * s.h);
        else s.gain.assign(s.w * s.h, 1.0f);
        off += s.w * s.h;
        m.spots.push_back(std::move(s));
    }
    return m;
}

// dust.rs:487 apply_rgb16 in place on an interleaved u16 frame (w x h; a frame of another size is left alone)
void orc_dust_apply_rgb16(const uint64_t* rects, size_t n, const uint8_t* masks, const float* gains, size_t mw, size_t mh, int mode,
                          uint16_t* rgb, size_t w, size_t h) {
    dust_apply_rgb16(dust_of(rects, n, masks, gains, mw, mh, mode), rgb, w, h);
}

// dust.rs:478 apply in place on planar f32 planes [3][h][w]
void orc_dust_apply_f(const uint64_t* rects, size_t n, const uint8_t* masks, const float* gains, size_t mw, size_t mh, int mode,
                      float* planes, size_t w, size_t h) {
    Img3<float> f(w, h);
    for (int c = 0; c < 3; c++) std::copy(planes + c * w * h, planes + (c + 1) * w * h, f.p[c].begin());
    dust_apply(dust_of(rects, n, masks, gains, mw, mh, mode), f);
    for (int c = 0; c < 3; c++) std::copy(f.p[c].begin(), f.p[c].end(), planes + c * w * h);
}

// dust.rs:591 pull_push (f32)
void orc_pull_push_f(const float* v, const float* wt, size_t w, size_t h, float* out) {
    std::vector<float> a(v, v + w * h), b(wt, wt + w * h);
    std::vector<float> f = pull_push<float>(a, b, w, h);
    std::copy(f.begin(), f.end(), out);
}

// prep.rs:16 rotate and prep.rs:77 reduce of planar f32 planes; out sized by the caller
void orc_rotate_f(const float* planes, size_t w, size_t h, int quarters, int flip, float* out) {
    Img3<float> f(w, h);
    for (int c = 0; c < 3; c++) std::copy(planes + c * w * h, planes + (c + 1) * w * h, f.p[c].begin());
    Img3<float> o = rotate(f, quarters, flip != 0);
    for (int c = 0; c < 3; c++) std::copy(o.p[c].begin(), o.p[c].end(), out + c * o.w * o.h);
}
void orc_draft_reduce_f(const float* planes, size_t w, size_t h, int levels, float* out) {
    Img3<float> f(w, h);
    for (int c = 0; c < 3; c++) std::copy(planes + c * w * h, planes + (c + 1) * w * h, f.p[c].begin());
    Img3<float> o = draft_reduce(f, levels);
    for (int c = 0; c < 3; c++) std::copy(o.p[c].begin(), o.p[c].end(), out + c * o.w * o.h);
}

// lapstack-web lib.rs:766-784 on an interleaved u16 frame: the dust map (n_spots 0: none), the turn, the draft
// reduction and the run's size (rw, rh; 0: as prepared); out sized by the caller, its dims into odims[2]
void orc_prep_rgb16(const uint64_t* rects, size_t n, const uint8_t* masks, const float* gains, size_t mw, size_t mh, int mode, int quarters,
                    int draft, const uint16_t* in, size_t w, size_t h, size_t rw, size_t rh, uint16_t* out, uint64_t* odims) {
    DustMap m = dust_of(rects, n, masks, gains, mw, mh, mode);
    size_t ow, oh;
    std::vector<uint16_t> f = prep_rgb16(n ? &m : nullptr, quarters, draft, std::vector<uint16_t>(in, in + w * h * 3), w, h, rw, rh, ow, oh);
    if (out) std::copy(f.begin(), f.end(), out);
    odims[0] = ow;
    odims[1] = oh;
}

// f32 -> IEEE half bits (round to nearest even) and back, as the 16-bit storage emulation does them
void orc_f16_round(const float* in, size_t n, uint16_t* bits, float* back) {
    for (size_t i = 0; i < n; i++) {
        bits[i] = f16_bits(in[i]);
        back[i] = f16_value(bits[i]);
    }
}

// OpenMP threads of every later oracle call (0: all the host's)
void orc_set_threads(int n) { omp_set_num_threads(n > 0 ? n : omp_get_num_procs()); }
int orc_threads(void) { return omp_get_max_threads(); }

// the seeded synthetic stack (orc_synth.hpp): d = [w, h, n, warp, seed_lo, seed_hi, mag_step, noise_std,
// blur_px, warp_scale, warp_rot_deg, warp_shift]; frames k0 .. k0+count-1 of the stack into out
int orc_synth_stack(const double* d, uint16_t* out, double* truth, uint32_t k0, uint32_t count) {
    SynthDesc sd;
    sd.w = (uint32_t)d[0];
    sd.h = (uint32_t)d[1];
    sd.n = (uint32_t)d[2];
    sd.warp = (uint32_t)d[3];
    sd.seed = (uint64_t)d[4] | ((uint64_t)d[5] << 32);
    sd.mag_step = (float)d[6];
    sd.noise_std = (float)d[7];
    sd.blur_px = (float)d[8];
    sd.warp_scale = (float)d[9];
    sd.warp_rot_deg = (float)d[10];
    sd.warp_shift = (float)d[11];
    return synth_stack(sd, out, truth, k0, count) ? 0 : 1;
}

}  // extern "C"
