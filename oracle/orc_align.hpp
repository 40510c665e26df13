// Oracle (test infrastructure only; see orc_core.hpp): align.rs and
// brightness.rs of crates/lapstack-core/src restated.
#pragma once
#include <atomic>

#include "orc_core.hpp"

namespace orc {

typedef double Mat3[3][3];

// align.rs:52-70 `AlignParams` / align.rs:128 `Interp` (ids in Interp::ALL order)
enum Interp { INTERP_NEAREST = 0, INTERP_BILINEAR = 1, INTERP_BICUBIC = 2, INTERP_SPLINE4 = 3, INTERP_SPLINE6 = 4, INTERP_LANCZOS3 = 5 };
enum AlignModel { MODEL_SIMILARITY = 0, MODEL_AFFINE = 1, MODEL_PROJECTIVE = 2 };

struct AlignParams {
    bool shift = true, scale = true, rotation = true;
    int model = MODEL_SIMILARITY;
    size_t coarsen = 0;
    int interp = INTERP_SPLINE4;
};

// align.rs:115 `free_mask`
inline void free_mask(const AlignParams& a, bool out[8]) {
    bool affine = a.model != MODEL_SIMILARITY, proj = a.model == MODEL_PROJECTIVE;
    bool m[8] = {a.shift, a.shift, a.scale, a.rotation, affine, affine, proj, proj};
    for (int k = 0; k < 8; k++) out[k] = m[k];
}

// align.rs:178 `taps`, :190 `margin`
inline size_t interp_taps(int k) { return k == INTERP_NEAREST ? 1 : k == INTERP_BILINEAR ? 2 : k <= INTERP_SPLINE4 ? 4 : 6; }
inline double interp_margin(int k) { return (double)(interp_taps(k) / 2); }

// align.rs:200 `Sim`: [xoff, yoff, scale, rot, aspect, shear, px, py]
struct Sim {
    double v[8] = {0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 0.0};
    bool is_id() const {
        static const double id[8] = {0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < 8; k++)
            if (v[k] != id[k]) return false;
        return true;
    }
};
// align.rs:220 `Sim::SPAN`
static const double SIM_SPAN[8] = {0.10, 0.10, 0.10, 0.087266462599716474, 0.05, 0.05, 0.05, 0.05};

// align.rs:241 `Sim::matrix`
inline void sim_matrix(const Sim& s, size_t w, size_t h, Mat3 m) {
    double cx = (double)w / 2.0, cy = (double)h / 2.0;
    double c = std::cos(s.v[3]), sn = std::sin(s.v[3]);
    double sc = s.v[2], shear = s.v[5], aspect = s.v[4];
    double a = sc * c, b = sc * (c * shear - sn * aspect), d = sc * sn, e = sc * (sn * shear + c * aspect);
    double gx = s.v[6] / (double)w, gy = s.v[7] / (double)h;
    double a2 = a + cx * gx, b2 = b + cx * gy, d2 = d + cy * gx, e2 = e + cy * gy;
    double tx = cx + s.v[0] * (double)w - (a2 * cx + b2 * cy);
    double ty = cy + s.v[1] * (double)h - (d2 * cx + e2 * cy);
    m[0][0] = a2; m[0][1] = b2; m[0][2] = tx;
    m[1][0] = d2; m[1][1] = e2; m[1][2] = ty;
    m[2][0] = gx; m[2][1] = gy; m[2][2] = 1.0 - gx * cx - gy * cy;
}

// align.rs:258 `inverse`
inline void mat_inverse(const Mat3 m, Mat3 inv) {
    if (m[2][0] == 0.0 && m[2][1] == 0.0 && m[2][2] == 1.0) {
        double a = m[0][0], b = m[0][1], tx = m[0][2], d = m[1][0], e = m[1][1], ty = m[1][2];
        double det = a * e - b * d;
        double ia = e / det, ib = -b / det, id = -d / det, ie = a / det;
        inv[0][0] = ia; inv[0][1] = ib; inv[0][2] = -(ia * tx + ib * ty);
        inv[1][0] = id; inv[1][1] = ie; inv[1][2] = -(id * tx + ie * ty);
        inv[2][0] = 0.0; inv[2][1] = 0.0; inv[2][2] = 1.0;
        return;
    }
    auto cof = [&](int i, int j) {
        int r0 = (i + 1) % 3, r1 = (i + 2) % 3, c0 = (j + 1) % 3, c1 = (j + 2) % 3;
        return m[r0][c0] * m[r1][c1] - m[r0][c1] * m[r1][c0];
    };
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) inv[i][j] = cof(j, i);
    double k = inv[2][2];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) inv[i][j] /= k;
}

// align.rs:291 `map`
inline void mat_map(const Mat3 inv, double x, double y, double& sx, double& sy) {
    double d = inv[2][0] * x + inv[2][1] * y + inv[2][2];
    sx = (inv[0][0] * x + inv[0][1] * y + inv[0][2]) / d;
    sy = (inv[1][0] * x + inv[1][1] * y + inv[1][2]) / d;
}

inline bool mat_is_affine(const Mat3 inv) { return inv[2][0] == 0.0 && inv[2][1] == 0.0 && inv[2][2] == 1.0; }

// align.rs:485 `affine_row` + `map`: the source point of destination (x, y).
inline void source_point(const Mat3 inv, bool aff, double x, double y, double& sx, double& sy) {
    if (aff) {
        double x0 = inv[0][1] * y + inv[0][2], y0 = inv[1][1] * y + inv[1][2];
        sx = x0 + inv[0][0] * x;
        sy = y0 + inv[1][0] * x;
    } else {
        mat_map(inv, x, y, sx, sy);
    }
}

// align.rs:416 `spline4`
inline void spline4(double t, double w[4]) {
    w[0] = ((-1.0 / 3.0 * t + 0.8) * t - 0.46666667) * t;
    w[1] = ((t - 1.8) * t - 0.2) * t + 1.0;
    w[2] = ((1.2 - t) * t + 0.8) * t;
    w[3] = ((1.0 / 3.0 * t - 0.2) * t - 0.13333334) * t;
}
// align.rs:427 `keys`
inline double keys(double d) {
    if (d < 1.0) return (1.5 * d - 2.5) * d * d + 1.0;
    if (d < 2.0) return ((-0.5 * d + 2.5) * d - 4.0) * d + 2.0;
    return 0.0;
}
// align.rs:433 `spline36`
inline double spline36(double d) {
    if (d < 1.0) return ((13.0 / 11.0 * d - 453.0 / 209.0) * d - 3.0 / 209.0) * d + 1.0;
    if (d < 2.0) {
        double u = d - 1.0;
        return ((-6.0 / 11.0 * u + 270.0 / 209.0) * u - 156.0 / 209.0) * u;
    }
    if (d < 3.0) {
        double u = d - 2.0;
        return ((1.0 / 11.0 * u - 45.0 / 209.0) * u + 26.0 / 209.0) * u;
    }
    return 0.0;
}
// align.rs:449 `lanczos3`
inline double lanczos3(double d) {
    if (d < 1e-9) return 1.0;
    if (d < 3.0) {
        double a = M_PI * d, b = M_PI * d / 3.0;
        return std::sin(a) / a * (std::sin(b) / b);
    }
    return 0.0;
}
// align.rs:463 `taps_of`
template <int N>
inline void taps_of(double (*k)(double), double t, double w[N]) {
    double sum = 0.0;
    for (int i = 0; i < N; i++) {
        w[i] = k(std::fabs(t - ((double)i + 1.0 - (double)(N / 2))));
        sum += w[i];
    }
    for (int i = 0; i < N; i++) w[i] /= sum;
}
// align.rs:542 `warp_plane`'s kernels: the weights of kernel `k` at fraction t.
inline int interp_weights(int k, double t, double w[6]) {
    switch (k) {
        case INTERP_NEAREST: w[0] = t < 0.5 ? 1.0 : 0.0; w[1] = t < 0.5 ? 0.0 : 1.0; return 2;
        case INTERP_BILINEAR: w[0] = 1.0 - t; w[1] = t; return 2;
        case INTERP_BICUBIC: taps_of<4>(keys, t, w); return 4;
        case INTERP_SPLINE4: spline4(t, w); return 4;
        case INTERP_SPLINE6: taps_of<6>(spline36, t, w); return 6;
        default: taps_of<6>(lanczos3, t, w); return 6;
    }
}

// align.rs:489 `warp_with` / :542 `warp_plane`: f64 coordinates, f32 taps and sums.
template <class T>
void warp_plane(const T* src, size_t w, size_t h, const Sim& sim, size_t ow, size_t oh, int interp, std::vector<T>& out,
                std::vector<uint8_t>* valid) {
    Mat3 m, inv;
    sim_matrix(sim, w, h, m);
    mat_inverse(m, inv);
    bool aff = mat_is_affine(inv);
    double xmax = (double)(w - 1), ymax = (double)(h - 1);
    out.assign(ow * oh, T(0));
    if (valid) valid->assign(ow * oh, 0);
#pragma omp parallel for schedule(static)
    for (long y = 0; y < (long)oh; y++) {
        double yf = (double)y;
        for (size_t x = 0; x < ow; x++) {
            double sx, sy;
            source_point(inv, aff, (double)x, yf, sx, sy);
            if (valid) (*valid)[(size_t)y * ow + x] = (sx >= 0.0 && sx <= xmax && sy >= 0.0 && sy <= ymax) ? 1 : 0;
            long x0 = (long)std::floor(sx), y0 = (long)std::floor(sy);
            double wxd[6], wyd[6];
            int n = interp_weights(interp, sx - (double)x0, wxd);
            interp_weights(interp, sy - (double)y0, wyd);
            T wx[6], wy[6];
            for (int i = 0; i < n; i++) {
                wx[i] = (T)wxd[i];
                wy[i] = (T)wyd[i];
            }
            long start = 1 - n / 2;
            long xs = x0 + start, ys = y0 + start;
            T acc = T(0);
            for (int j = 0; j < n; j++) {
                long yy = std::min(std::max(ys + j, 0L), (long)h - 1);
                T r = T(0);
                for (int i = 0; i < n; i++) {
                    long xx = std::min(std::max(xs + i, 0L), (long)w - 1);
                    r += wx[i] * src[(size_t)yy * w + (size_t)xx];
                }
                acc += wy[j] * r;
            }
            out[(size_t)y * ow + x] = acc;
        }
    }
}

// align.rs:639 `spline4f`
template <class T>
inline void spline4f(T t, T w[4]) {
    w[0] = ((LIT(-1.0) / LIT(3.0) * t + LIT(0.8)) * t - LIT(0.46666667)) * t;
    w[1] = ((t - LIT(1.8)) * t - LIT(0.2)) * t + LIT(1.0);
    w[2] = ((LIT(1.2) - t) * t + LIT(0.8)) * t;
    w[3] = ((LIT(1.0) / LIT(3.0) * t - LIT(0.2)) * t - LIT(0.13333334)) * t;
}

// align.rs:581 `warp_cost`: the DC-removed RMS of ref - warped target over the
// valid pixels; f64 coordinates and sums, f32 taps. Rows are summed in order
// (the reference's rayon reduction order is unspecified; this one is fixed).
template <class T>
double warp_cost(const T* rf, size_t aw, size_t ah, const T* tgt, size_t tw, size_t th, const Sim& sim) {
    Mat3 m, inv;
    sim_matrix(sim, tw, th, m);
    mat_inverse(m, inv);
    bool aff = mat_is_affine(inv);
    double xmax = (double)(tw - 1), ymax = (double)(th - 1);
    std::vector<double> rs(ah), rs2(ah);
    std::vector<size_t> rc(ah);
#pragma omp parallel for schedule(static)
    for (long y = 0; y < (long)ah; y++) {
        double sd = 0.0, sd2 = 0.0;
        size_t cnt = 0;
        double yf = (double)y;
        const T* row = rf + (size_t)y * aw;
        for (size_t x = 0; x < aw; x++) {
            double sx, sy;
            source_point(inv, aff, (double)x, yf, sx, sy);
            if (!(sx >= 0.0 && sx <= xmax && sy >= 0.0 && sy <= ymax)) continue;
            long x0 = (long)std::floor(sx), y0 = (long)std::floor(sy);
            T wx[4], wy[4];
            spline4f<T>((T)(sx - (double)x0), wx);
            spline4f<T>((T)(sy - (double)y0), wy);
            T acc = T(0);
            for (int j = 0; j < 4; j++) {
                long yy = std::min(std::max(y0 + j - 1, 0L), (long)th - 1);
                T r = T(0);
                for (int i = 0; i < 4; i++) {
                    long xx = std::min(std::max(x0 + i - 1, 0L), (long)tw - 1);
                    r += wx[i] * tgt[(size_t)yy * tw + (size_t)xx];
                }
                acc += wy[j] * r;
            }
            double d = (double)(row[x] - acc);
            sd += d;
            sd2 += d * d;
            cnt++;
        }
        rs[y] = sd;
        rs2[y] = sd2;
        rc[y] = cnt;
    }
    double sd = 0.0, sd2 = 0.0;
    size_t cnt = 0;
    for (size_t y = 0; y < ah; y++) {
        sd += rs[y];
        sd2 += rs2[y];
        cnt += rc[y];
    }
    if (cnt < 16) return 1e9;
    double n = (double)cnt;
    return std::sqrt(std::max((sd2 - sd * sd / n) / n, 0.0));
}

// align.rs:650 `burt_kernel`, :658 `norm_full`, :674 `reduce_burt`
template <class T>
inline void burt_kernel(T k[5]) {
    T a = LIT(0.33), b = LIT(0.25), c = LIT(0.25) - a / LIT(2.0);
    k[0] = c; k[1] = b; k[2] = a; k[3] = b; k[4] = c;
}
template <class T>
std::vector<T> norm_full(size_t n, const T k[5]) {
    std::vector<T> o(n);
    for (size_t i = 0; i < n; i++) {
        T s = T(0);
        for (int t = 0; t < 5; t++) {
            long x = (long)i + t - 2;
            if (x >= 0 && (size_t)x < n) s += k[t];
        }
        o[i] = s;
    }
    return o;
}
template <class T>
void reduce_burt(const T* src, size_t w, size_t h, std::vector<T>& out, size_t& ow, size_t& oh) {
    T k[5];
    burt_kernel<T>(k);
    ow = (w + 1) / 2;
    oh = (h + 1) / 2;
    std::vector<T> cn = norm_full<T>(w, k), rn = norm_full<T>(h, k);
    std::vector<T> htmp(h * ow);
    size_t oww = ow;
#pragma omp parallel for schedule(static) if (h * ow >= (1u << 15))
    for (long y = 0; y < (long)h; y++) {
        const T* s = src + (size_t)y * w;
        for (size_t oj = 0; oj < oww; oj++) {
            long c = 2 * (long)oj;
            T a = T(0);
            for (int t = 0; t < 5; t++) {
                long i = c + t - 2;
                if (i >= 0 && (size_t)i < w) a += k[t] * s[i];
            }
            htmp[(size_t)y * oww + oj] = a;
        }
    }
    out.assign(oh * ow, T(0));
#pragma omp parallel for schedule(static) if (oh * ow >= (1u << 15))
    for (long oi = 0; oi < (long)oh; oi++) {
        long cy = 2 * oi;
        T r = rn[(size_t)cy];
        T* row = &out[(size_t)oi * oww];
        for (int t = 0; t < 5; t++) {
            long s = cy + t - 2;
            if (s >= 0 && (size_t)s < h) {
                const T* hr = &htmp[(size_t)s * oww];
                for (size_t oj = 0; oj < oww; oj++) row[oj] += k[t] * hr[oj];
            }
        }
        for (size_t oj = 0; oj < oww; oj++) row[oj] /= r * cn[2 * oj];
    }
}

template <class T>
struct Lvl {
    std::vector<T> d;
    size_t w, h;
};

// align.rs:741 `gauss_levels`: levels above full resolution while h > 64 && w > 8.
template <class T>
std::vector<Lvl<T>> gauss_levels(const T* y, size_t w, size_t h) {
    std::vector<Lvl<T>> levels;
    size_t cw = w, ch = h;
    while (ch > 64 && cw > 8) {
        Lvl<T> l;
        reduce_burt<T>(levels.empty() ? y : levels.back().d.data(), cw, ch, l.d, l.w, l.h);
        cw = l.w;
        ch = l.h;
        levels.push_back(std::move(l));
    }
    return levels;
}

// align.rs:766 `param_gain`, :784 `level_steps`
inline void param_gain(size_t w, size_t h, double g[8]) {
    double wf = (double)w, hf = (double)h, r = std::max(wf, hf) / 2.0;
    double v[8] = {wf, hf, r, r, hf / 2.0, hf / 2.0, wf / 4.0, hf / 4.0};
    for (int k = 0; k < 8; k++) g[k] = v[k];
}
constexpr double STEP_PX = 1.0, TOL_PX = 0.1;
inline void level_steps(const std::vector<size_t>& free_idx, size_t lvl, size_t w, size_t h, std::vector<double>& step,
                        std::vector<double>& tol) {
    double g[8];
    param_gain(w, h, g);
    double px = (double)((uint64_t)1 << lvl);
    step.clear();
    tol.clear();
    for (size_t k : free_idx) {
        step.push_back(STEP_PX * px / g[k]);
        tol.push_back(TOL_PX * px / g[k]);
    }
}

// align.rs:888 `converged`
inline bool nm_converged(const std::vector<std::vector<double>>& s, const std::vector<double>& fv, const std::vector<double>& tol) {
    size_t n = tol.size();
    if (std::fabs(fv[n] - fv[0]) > 1e-4 * (1.0 + std::fabs(fv[0]))) return false;
    for (size_t i = 1; i < s.size(); i++)
        for (size_t k = 0; k < n; k++)
            if (!(std::fabs(s[i][k] - s[0][k]) <= tol[k])) return false;
    return true;
}

// Nelder-Mead steps by kind over every search since the last reset: [0] reflection accepted,
// [1] expansion evaluated, [2] contraction accepted, [3] shrink, [4] searches. Instrumentation
// only: the search's arithmetic and branches do not depend on it.
inline std::atomic<size_t> g_nm_steps[5];

// align.rs:796 `nelder_mead` (bounded; stable sort of the vertices each iteration)
inline std::vector<double> nelder_mead(const std::function<double(const std::vector<double>&)>& f, const std::vector<double>& x0,
                                       const std::vector<double>& lo, const std::vector<double>& hi, const std::vector<double>& step,
                                       const std::vector<double>& tol, size_t* evals = nullptr) {
    size_t n = x0.size();
    if (n == 0) return {};
    size_t ne = 0;
    auto F = [&](const std::vector<double>& v) {
        ne++;
        return f(v);
    };
    auto clampv = [&](std::vector<double>& v) {
        for (size_t k = 0; k < n; k++) v[k] = std::min(std::max(v[k], lo[k]), hi[k]);
    };
    std::vector<std::vector<double>> simplex{x0};
    for (size_t k = 0; k < n; k++) {
        std::vector<double> v = x0;
        v[k] += step[k];
        clampv(v);
        simplex.push_back(v);
    }
    std::vector<double> fv;
    for (auto& v : simplex) fv.push_back(F(v));
    g_nm_steps[4]++;
    const double alpha = 1.0, gamma = 2.0, rho = 0.5, sigma = 0.5;
    for (int it = 0; it < 200; it++) {
        std::vector<size_t> idx(n + 1);
        for (size_t i = 0; i <= n; i++) idx[i] = i;
        std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return fv[a] < fv[b]; });
        std::vector<std::vector<double>> s2;
        std::vector<double> f2;
        for (size_t i : idx) {
            s2.push_back(simplex[i]);
            f2.push_back(fv[i]);
        }
        simplex.swap(s2);
        fv.swap(f2);
        if (nm_converged(simplex, fv, tol)) break;
        std::vector<double> c(n, 0.0);
        for (size_t i = 0; i < n; i++)
            for (size_t k = 0; k < n; k++) c[k] += simplex[i][k];
        for (size_t k = 0; k < n; k++) c[k] /= (double)n;
        std::vector<double> xr(n);
        for (size_t k = 0; k < n; k++) xr[k] = c[k] + alpha * (c[k] - simplex[n][k]);
        clampv(xr);
        double fr = F(xr);
        if (fr < fv[0]) {
            std::vector<double> xe(n);
            for (size_t k = 0; k < n; k++) xe[k] = c[k] + gamma * (xr[k] - c[k]);
            clampv(xe);
            double fe = F(xe);
            g_nm_steps[1]++;
            if (fe < fr) {
                simplex[n] = xe;
                fv[n] = fe;
            } else {
                simplex[n] = xr;
                fv[n] = fr;
            }
        } else if (fr < fv[n - 1]) {
            g_nm_steps[0]++;
            simplex[n] = xr;
            fv[n] = fr;
        } else {
            std::vector<double> xc(n);
            for (size_t k = 0; k < n; k++) xc[k] = c[k] + rho * (simplex[n][k] - c[k]);
            clampv(xc);
            double fc = F(xc);
            if (fc < fv[n]) {
                g_nm_steps[2]++;
                simplex[n] = xc;
                fv[n] = fc;
            } else {
                g_nm_steps[3]++;
                for (size_t i = 1; i <= n; i++) {
                    for (size_t k = 0; k < n; k++) simplex[i][k] = simplex[0][k] + sigma * (simplex[i][k] - simplex[0][k]);
                    clampv(simplex[i]);
                    fv[i] = F(simplex[i]);
                }
            }
        }
    }
    size_t best = 0;
    for (size_t i = 1; i <= n; i++)
        if (fv[i] < fv[best]) best = i;
    if (evals) *evals += ne;
    return simplex[best];
}

// align.rs:896 `multiscale_align`
template <class T>
Sim multiscale_align(const T* rf, const T* tg, size_t w, size_t h, const Sim& init, const bool free[8], size_t coarsen,
                     size_t* evals = nullptr) {
    std::vector<Lvl<T>> pref = gauss_levels<T>(rf, w, h), ptgt = gauss_levels<T>(tg, w, h);
    size_t n = std::min(pref.size(), ptgt.size()) + 1;
    std::vector<size_t> free_idx;
    for (size_t k = 0; k < 8; k++)
        if (free[k]) free_idx.push_back(k);
    std::vector<double> lo_f, hi_f;
    for (size_t k : free_idx) {
        lo_f.push_back(init.v[k] - SIM_SPAN[k]);
        hi_f.push_back(init.v[k] + SIM_SPAN[k]);
    }
    Sim cur = init;
    size_t finest = std::min(coarsen, n - 1);
    for (size_t lvl = n; lvl-- > finest;) {
        const T* a_d = lvl == 0 ? rf : pref[lvl - 1].d.data();
        size_t aw = lvl == 0 ? w : pref[lvl - 1].w, ah = lvl == 0 ? h : pref[lvl - 1].h;
        const T* t_d = lvl == 0 ? tg : ptgt[lvl - 1].d.data();
        size_t tw = lvl == 0 ? w : ptgt[lvl - 1].w, th = lvl == 0 ? h : ptgt[lvl - 1].h;
        Sim snap = cur;
        auto cost = [&](const std::vector<double>& xf) {
            Sim v = snap;
            for (size_t k = 0; k < free_idx.size(); k++) v.v[free_idx[k]] = xf[k];
            return warp_cost<T>(a_d, aw, ah, t_d, tw, th, v);
        };
        std::vector<double> x0;
        for (size_t k : free_idx) x0.push_back(cur.v[k]);
        std::vector<double> step, tol;
        level_steps(free_idx, lvl, w, h, step, tol);
        std::vector<double> best = nelder_mead(cost, x0, lo_f, hi_f, step, tol, evals);
        for (size_t k = 0; k < free_idx.size(); k++) cur.v[free_idx[k]] = best[k];
    }
    return cur;
}

struct Rect {
    size_t x = 0, y = 0, w = 0, h = 0;
};

// align.rs:344 `common_area`
inline Rect common_area(const std::vector<Sim>& sims, size_t w, size_t h, int interp) {
    Rect full{0, 0, w, h};
    if (w == 0 || h == 0) return full;
    std::vector<std::array<std::array<double, 3>, 3>> invs;
    for (auto& s : sims) {
        if (s.is_id()) continue;
        Mat3 m, inv;
        sim_matrix(s, w, h, m);
        mat_inverse(m, inv);
        std::array<std::array<double, 3>, 3> a;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) a[i][j] = inv[i][j];
        invs.push_back(a);
    }
    if (invs.empty()) return full;
    double mg = interp_margin(interp);
    double xmax = (double)(w - 1) - mg, ymax = (double)(h - 1) - mg;
    std::vector<std::pair<long, long>> rows;
    for (size_t y = 0; y < h; y++) {
        double lo = 0.0, hi = (double)(w - 1), yf = (double)y;
        for (auto& inv : invs) {
            double g = inv[2][0], d = inv[2][1] * yf + inv[2][2];
            if (d <= 0.0 || g * (double)(w - 1) + d <= 0.0) {
                lo = 1.0;
                hi = 0.0;
                break;
            }
            double A[2] = {inv[0][0], inv[1][0]}, Kk[2] = {inv[0][1] * yf + inv[0][2], inv[1][1] * yf + inv[1][2]};
            double smin[2] = {mg, mg}, smax[2] = {xmax, ymax};
            for (int ax = 0; ax < 2; ax++) {
                double a = A[ax], k = Kk[ax];
                double pq[2][2] = {{a - smin[ax] * g, k - smin[ax] * d}, {smax[ax] * g - a, smax[ax] * d - k}};
                for (int t = 0; t < 2; t++) {
                    double p = pq[t][0], q = pq[t][1];
                    if (std::fabs(p) < 1e-12) {
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
        rows.push_back(lo <= hi ? std::make_pair((long)std::ceil(lo), (long)std::floor(hi)) : std::make_pair(1L, 0L));
    }
    Rect best{0, 0, 0, 0};
    for (size_t y0 = 0; y0 < h; y0++) {
        long lo = rows[y0].first, hi = rows[y0].second;
        for (size_t y1 = y0; y1 < h; y1++) {
            lo = std::max(lo, rows[y1].first);
            hi = std::min(hi, rows[y1].second);
            if (lo > hi) break;
            size_t rw = (size_t)(hi - lo + 1), rh = y1 - y0 + 1;
            if (rw * rh > best.w * best.h) best = Rect{(size_t)lo, y0, rw, rh};
        }
    }
    return best.w * best.h == 0 ? full : best;
}

// ------------------------------------------------------------- brightness.rs

constexpr float GAIN_MIN = 0.25f, GAIN_MAX = 4.0f;
constexpr size_t BSTEP = 4;

// brightness.rs:34 `Reference`: frame 0 on the stride-4 grid.
template <class T>
struct BReference {
    size_t w = 0, h = 0, gw = 0;
    std::vector<T> p[3];
    void init(const Img3<T>& f) {
        w = f.w;
        h = f.h;
        gw = (w + BSTEP - 1) / BSTEP;
        for (int c = 0; c < 3; c++) {
            p[c].clear();
            for (size_t y = 0; y < h; y += BSTEP)
                for (size_t x = 0; x < w; x += BSTEP) p[c].push_back(f.p[c][y * w + x]);
        }
    }
};

// brightness.rs:67 `sums`
template <class T>
void bsums(const Img3<T>& f, const BReference<T>* other, const Sim& sim, double sf[3], double so[3], size_t& n) {
    size_t w = f.w, h = f.h;
    bool use_inv = !sim.is_id();
    Mat3 m, inv;
    if (use_inv) {
        sim_matrix(sim, w, h, m);
        mat_inverse(m, inv);
    }
    for (int c = 0; c < 3; c++) sf[c] = so[c] = 0.0;
    n = 0;
    for (size_t y = 0; y < h; y += BSTEP)
        for (size_t x = 0; x < w; x += BSTEP) {
            if (use_inv) {
                double sx, sy;
                mat_map(inv, (double)x, (double)y, sx, sy);
                if (!(sx >= 0.0 && sx <= (double)(w - 1) && sy >= 0.0 && sy <= (double)(h - 1))) continue;
            }
            size_t i = y * w + x;
            for (int c = 0; c < 3; c++) {
                sf[c] += (double)f.p[c][i];
                if (other) so[c] += (double)other->p[c][(y / BSTEP) * other->gw + x / BSTEP];
            }
            n++;
        }
}

// brightness.rs:93 `ratio`
inline void bratio(const double ref[3], const double frame[3], size_t n, float g[3]) {
    for (int c = 0; c < 3; c++) {
        if (n < 64) {
            g[c] = 1.0f;
            continue;
        }
        float v = frame[c] > 1e-9 ? (float)(ref[c] / frame[c]) : 1.0f;
        g[c] = std::min(std::max(v, GAIN_MIN), GAIN_MAX);
    }
}

// brightness.rs:107 `means`
template <class T>
void bmeans(const Img3<T>& f, double m[3]) {
    double s[3], so[3];
    size_t n;
    bsums<T>(f, nullptr, Sim(), s, so, n);
    for (int c = 0; c < 3; c++) m[c] = n == 0 ? 0.0 : s[c] / (double)n;
}

// brightness.rs:124 `apply`
template <class T>
void bapply(Img3<T>& f, const float g[3]) {
    for (int c = 0; c < 3; c++)
        if (std::fabs(g[c] - 1.0f) > 1e-6f)
            for (auto& v : f.p[c]) v *= (T)g[c];
}

}  // namespace orc
