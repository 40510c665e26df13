// Oracle (test infrastructure only; see orc_core.hpp): depth.rs of
// crates/lapstack-core/src restated — focus measure, block mean, box and
// guided filters, the streamed peak tracker, median, confidence
// normalisation, the edge-aware WLS solve (FGS guess + multigrid-
// preconditioned CG) and the upsampling.
#pragma once
#include "orc_core.hpp"

namespace orc {

enum FocusKind { FOCUS_RDF = 0, FOCUS_SML = 1 };
enum UpsampleKind { UP_BILINEAR = 0, UP_GUIDED = 1 };

// depth.rs:69-109 `DepthParams`
struct DepthParams {
    size_t scale = 1;
    int focus = FOCUS_RDF;
    size_t r_in = 1, r_out = 3, sml_step = 1;
    size_t agg_radius = 3;
    float agg_eps = 1e-4f;
    float lambda = 3.0f, sigma_c = 0.04f;
    size_t cg_iters = 200;
    bool median = true;
    int upsample = UP_GUIDED;
    size_t up_radius = 2;
    float up_eps = 1e-2f;
    float gate = 1.0f, robust = 1.0f;
};

// depth.rs:169 `blocks`
inline size_t blocks(size_t n, size_t k) { return (n + k - 1) / k; }

// depth.rs:160 `luma`
template <class T>
std::vector<T> luma(const Img3<T>& im) {
    std::vector<T> y(im.w * im.h);
    for (size_t i = 0; i < y.size(); i++) y[i] = luma_of<T>(im.p[0][i], im.p[1][i], im.p[2][i]);
    return y;
}

// depth.rs:174 `block_mean`
template <class T>
std::vector<T> block_mean(const T* src, size_t w, size_t h, size_t k, size_t& dw, size_t& dh) {
    dw = blocks(w, k);
    dh = blocks(h, k);
    if (k == 1) return std::vector<T>(src, src + w * h);
    std::vector<T> out(dw * dh, T(0));
#pragma omp parallel for schedule(static) if (dw * dh >= (1u << 14))
    for (long oy = 0; oy < (long)dh; oy++) {
        size_t y0 = (size_t)oy * k, y1 = std::min(y0 + k, h);
        T* row = &out[(size_t)oy * dw];
        for (size_t y = y0; y < y1; y++) {
            const T* s = src + y * w;
            for (size_t ox = 0; ox < dw; ox++) {
                size_t x0 = ox * k, x1 = std::min(x0 + k, w);
                T a = T(0);
                for (size_t x = x0; x < x1; x++) a += s[x];
                row[ox] += a;
            }
        }
        for (size_t ox = 0; ox < dw; ox++) {
            T cnt = (T)((y1 - y0) * (std::min(ox * k + k, w) - ox * k));
            row[ox] /= cnt;
        }
    }
    return out;
}

// depth.rs:201 `upsample_bilinear`
template <class T>
std::vector<T> upsample_bilinear(const T* g, size_t dw, size_t dh, size_t w, size_t h, size_t k) {
    std::vector<T> out(w * h);
    T inv = T(1) / (T)k;
#pragma omp parallel for schedule(static)
    for (long y = 0; y < (long)h; y++) {
        T fy = std::min(std::max(((T)y + LIT(0.5)) * inv - LIT(0.5), T(0)), (T)(dh - 1));
        size_t y0 = (size_t)fy, y1 = std::min(y0 + 1, dh - 1);
        T ty = fy - (T)y0;
        const T *r0 = g + y0 * dw, *r1 = g + y1 * dw;
        for (size_t x = 0; x < w; x++) {
            T fx = std::min(std::max(((T)x + LIT(0.5)) * inv - LIT(0.5), T(0)), (T)(dw - 1));
            size_t x0 = (size_t)fx, x1 = std::min(x0 + 1, dw - 1);
            T tx = fx - (T)x0;
            T top = r0[x0] + (r0[x1] - r0[x0]) * tx;
            T bot = r1[x0] + (r1[x1] - r1[x0]) * tx;
            out[(size_t)y * w + x] = top + (bot - top) * ty;
        }
    }
    return out;
}

// depth.rs:263 `BoxFilter`: border-clipped window mean, f64 moving sums.
template <class T>
struct BoxFilter {
    size_t w, h, r;
    std::vector<T> inv_count, tmp;
    BoxFilter(size_t w_, size_t h_, size_t r_) : w(w_), h(h_), r(r_) {
        auto cnt = [&](size_t n, size_t i) { return (T)(std::min(i + r + 1, n) - (i >= r ? i - r : 0)); };
        inv_count.resize(w * h);
        for (size_t y = 0; y < h; y++) {
            T cy = cnt(h, y);
            for (size_t x = 0; x < w; x++) inv_count[y * w + x] = T(1) / (cy * cnt(w, x));
        }
        tmp.resize(w * h);
    }
    void sum_into(const T* src, T* out) {
#pragma omp parallel for schedule(static)
        for (long y = 0; y < (long)h; y++) {
            const T* s = src + (size_t)y * w;
            T* row = &tmp[(size_t)y * w];
            double acc = 0.0;
            for (size_t x = 0; x < std::min(r + 1, w); x++) acc += (double)s[x];
            for (size_t x = 0; x < w; x++) {
                row[x] = (T)acc;
                if (x + r + 1 < w) acc += (double)s[x + r + 1];
                if (x >= r) acc -= (double)s[x - r];
            }
        }
#pragma omp parallel for schedule(static)
        for (long x = 0; x < (long)w; x++) {
            double acc = 0.0;
            for (size_t y = 0; y < std::min(r + 1, h); y++) acc += (double)tmp[y * w + x];
            for (size_t y = 0; y < h; y++) {
                out[y * w + x] = (T)acc;
                if (y + r + 1 < h) acc += (double)tmp[(y + r + 1) * w + x];
                if (y >= r) acc -= (double)tmp[(y - r) * w + x];
            }
        }
    }
    void mean_into(const T* src, T* out) {
        sum_into(src, out);
        for (size_t i = 0; i < w * h; i++) out[i] *= inv_count[i];
    }
    std::vector<T> mean(const T* src) {
        std::vector<T> o(w * h);
        mean_into(src, o.data());
        return o;
    }
};

// depth.rs:352 `GuidedFilter`
template <class T>
struct GuidedFilter {
    std::vector<T> guide, mean_i, var_i, s0, s1, s2, s3;
    BoxFilter<T> bf;
    T eps;
    size_t n;
    GuidedFilter(const std::vector<T>& g, size_t w, size_t h, size_t r, T eps_) : guide(g), bf(w, h, r), eps(eps_), n(w * h) {
        mean_i.resize(n);
        bf.mean_into(guide.data(), mean_i.data());
        std::vector<T> ii(n);
        for (size_t i = 0; i < n; i++) ii[i] = guide[i] * guide[i];
        var_i.resize(n);
        bf.mean_into(ii.data(), var_i.data());
        for (size_t i = 0; i < n; i++) var_i[i] = std::max(var_i[i] - mean_i[i] * mean_i[i], T(0));
        s0.resize(n);
        s1.resize(n);
        s2.resize(n);
        s3.resize(n);
    }
    // depth.rs:379 `coeffs_into`: a-bar in s1, b-bar in s0
    void coeffs_into(const T* p) {
        bf.mean_into(p, s0.data());
        for (size_t i = 0; i < n; i++) s1[i] = guide[i] * p[i];
        bf.mean_into(s1.data(), s2.data());
        for (size_t k = 0; k < n; k++) {
            T cov = s2[k] - mean_i[k] * s0[k];
            T a = cov / (var_i[k] + eps);
            s2[k] = a;
            s3[k] = s0[k] - a * mean_i[k];
        }
        bf.mean_into(s2.data(), s1.data());
        bf.mean_into(s3.data(), s0.data());
    }
    void filter_into(const T* p, T* out) {
        coeffs_into(p);
        for (size_t k = 0; k < n; k++) out[k] = s1[k] * guide[k] + s0[k];
    }
};

// depth.rs:454 `rdf_taps`: (dy, dx, w), disk then ring, dy-major.
template <class T>
struct Tap {
    long dy, dx;
    T w;
};
template <class T>
std::vector<Tap<T>> rdf_taps(size_t r_in, size_t r_out) {
    long ri2 = (long)(r_in * r_in), ro2 = (long)(r_out * r_out), r = (long)r_out;
    std::vector<std::pair<long, long>> disk, ring;
    for (long dy = -r; dy <= r; dy++)
        for (long dx = -r; dx <= r; dx++) {
            long d2 = dx * dx + dy * dy;
            if (d2 <= ri2) disk.push_back({dy, dx});
            else if (d2 <= ro2) ring.push_back({dy, dx});
        }
    T wd = T(1) / (T)disk.size(), wr = T(-1) / (T)std::max<size_t>(ring.size(), 1);
    std::vector<Tap<T>> t;
    for (auto& p : disk) t.push_back({p.first, p.second, wd});
    for (auto& p : ring) t.push_back({p.first, p.second, wr});
    return t;
}

// depth.rs:417 `conv_sparse`: taps grouped by dy in order of first
// appearance; per pixel, acc += w * s[reflect] in that order.
template <class T>
std::vector<T> conv_sparse(const T* src, size_t w, size_t h, const std::vector<Tap<T>>& taps) {
    std::vector<std::pair<long, std::vector<std::pair<long, T>>>> rows;
    for (auto& t : taps) {
        bool found = false;
        for (auto& r : rows)
            if (r.first == t.dy) {
                r.second.push_back({t.dx, t.w});
                found = true;
                break;
            }
        if (!found) rows.push_back({t.dy, {{t.dx, t.w}}});
    }
    std::vector<T> out(w * h, T(0));
#pragma omp parallel for schedule(static)
    for (long y = 0; y < (long)h; y++) {
        T* acc = &out[(size_t)y * w];
        for (auto& r : rows) {
            const T* s = src + reflect(y + r.first, h) * w;
            for (auto& t : r.second)
                for (size_t x = 0; x < w; x++) acc[x] += t.second * s[reflect((long)x + t.first, w)];
        }
    }
    return out;
}

// depth.rs:474 `focus_measure`
template <class T>
std::vector<T> focus_measure(const T* y, size_t w, size_t h, const DepthParams& p) {
    if (p.focus == FOCUS_RDF) {
        std::vector<T> f = conv_sparse<T>(y, w, h, rdf_taps<T>(p.r_in, p.r_out));
        for (auto& v : f) v = std::fabs(v);
        return f;
    }
    long s = (long)std::max<size_t>(p.sml_step, 1);
    std::vector<T> out(w * h);
#pragma omp parallel for schedule(static)
    for (long yy = 0; yy < (long)h; yy++) {
        size_t up = reflect(yy - s, h), dn = reflect(yy + s, h);
        const T *c = y + (size_t)yy * w, *u = y + up * w, *d = y + dn * w;
        for (size_t x = 0; x < w; x++) {
            T l = c[reflect((long)x - s, w)], r = c[reflect((long)x + s, w)];
            out[(size_t)yy * w + x] = std::fabs(T(2) * c[x] - l - r) + std::fabs(T(2) * c[x] - u[x] - d[x]);
        }
    }
    return out;
}

// depth.rs:1097 `focus_slice`
template <class T>
std::vector<T> focus_slice(const Img3<T>& img, const DepthParams& p, size_t& dw, size_t& dh) {
    std::vector<T> y = luma(img);
    std::vector<T> f = focus_measure<T>(y.data(), img.w, img.h, p);
    return block_mean<T>(f.data(), img.w, img.h, (size_t)1 << p.scale, dw, dh);
}

// depth.rs:500-611 `PeakTracker`
template <class T>
struct Px {
    T c1 = -1, l1 = -1, r1 = -1, c2 = -1, prev = 0, prev2 = 0, sum = 0, cmin = std::numeric_limits<T>::infinity();
    uint32_t i1 = 0;
    void reg(T val, uint32_t idx, T l, T r) {
        if (val > c1) {
            if (c1 >= T(0)) c2 = c1;
            c1 = val;
            i1 = idx;
            l1 = l;
            r1 = r;
        } else if (val > c2) {
            c2 = val;
        }
    }
};

// Rust's f32::min: the smaller, ignoring a NaN operand.
template <class T>
inline T rmin(T a, T b) {
    if (std::isnan(a)) return b;
    if (std::isnan(b)) return a;
    return a < b ? a : b;
}
template <class T>
inline T rmax(T a, T b) {
    if (std::isnan(a)) return b;
    if (std::isnan(b)) return a;
    return a > b ? a : b;
}
template <class T>
inline T rclamp(T v, T lo, T hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

// Rust's `select_nth_unstable_by(total_cmp)`: the k-th smallest value.
template <class T>
T select_nth(std::vector<T> v, size_t k) {
    std::nth_element(v.begin(), v.begin() + k, v.end(), [](T a, T b) { return a < b; });
    return v[k];
}

template <class T>
struct PeakTracker {
    std::vector<Px<T>> px;
    size_t m = 0;
    explicit PeakTracker(size_t n) : px(n) {}
    void push(const T* c) {
        size_t mm = m;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)px.size(); i++) {
            Px<T>& p = px[i];
            T v = c[i];
            if (mm >= 1) {
                bool is_peak = (mm == 1 || p.prev >= p.prev2) && p.prev > v;
                if (is_peak) p.reg(p.prev, (uint32_t)(mm - 1), mm >= 2 ? p.prev2 : T(-1), v);
            }
            p.sum += v;
            p.cmin = rmin(p.cmin, v);
            p.prev2 = p.prev;
            p.prev = v;
        }
        m++;
    }
    // depth.rs:568 `finish`: depth, raw confidence, per-cell profile minimum; floor out.
    void finish(T gate, std::vector<T>& depth, std::vector<T>& conf, std::vector<T>& mins, T& floor_) {
        size_t n = m;
        for (auto& p : px)
            if (n == 1 || p.prev >= p.prev2) p.reg(p.prev, (uint32_t)(n - 1), n >= 2 ? p.prev2 : T(-1), T(-1));
        std::vector<T> sub;
        for (size_t i = 0; i < px.size(); i += 7) sub.push_back(px[i].cmin);
        floor_ = select_nth(sub, sub.size() / 2);
        T inv_n = T(1) / (T)n;
        depth.resize(px.size());
        conf.resize(px.size());
        mins.resize(px.size());
        for (size_t i = 0; i < px.size(); i++) mins[i] = std::isfinite(px[i].cmin) ? px[i].cmin : T(0);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)px.size(); i++) {
            const Px<T>& p = px[i];
            T c1 = p.c1, l = p.l1, r = p.r1;
            T delta = T(0);
            if (l >= T(0) && r >= T(0) && c1 > T(0)) {
                T ll = std::log(rmax(l, LIT(1e-12))), lc = std::log(c1), lr = std::log(rmax(r, LIT(1e-12)));
                T den = ll - T(2) * lc + lr;
                if (den < T(0)) delta = rclamp(LIT(0.5) * (ll - lr) / den, LIT(-0.5), LIT(0.5));
            }
            depth[i] = (T)p.i1 + delta;
            if (c1 > T(0)) {
                T mean = p.sum * inv_n;
                T prom = rclamp(T(1) - mean / c1, T(0), T(1));
                T pkr = p.c2 >= T(0) ? rclamp(T(1) - p.c2 / c1, T(0), T(1)) : T(1);
                T g = (gate > T(0) && floor_ > T(0)) ? rclamp((c1 - floor_) / (gate * floor_), T(0), T(1)) : T(1);
                conf[i] = prom * pkr * g;
            } else {
                conf[i] = T(0);
            }
        }
    }
};

// depth.rs:615 `normalize_conf`
template <class T>
T normalize_conf(std::vector<T>& conf) {
    std::vector<T> sub;
    for (size_t i = 0; i < conf.size(); i += 7) sub.push_back(conf[i]);
    size_t k = std::min(sub.size() * 9 / 10, sub.size() - 1);
    T p90 = select_nth(sub, k);
    if (p90 > LIT(1e-6))
        for (auto& c : conf) c = rmin(c / p90, T(1));
    return p90;
}

// depth.rs:628 `median3`
template <class T>
std::vector<T> median3(const T* src, size_t w, size_t h) {
    std::vector<T> out(w * h);
#pragma omp parallel for schedule(static)
    for (long y = 0; y < (long)h; y++) {
        const T* rows[3];
        for (int k = 0; k < 3; k++) rows[k] = src + reflect(y + k - 1, h) * w;
        for (size_t x = 0; x < w; x++) {
            size_t xs[3] = {reflect((long)x - 1, w), x, reflect((long)x + 1, w)};
            T v[9];
            int k = 0;
            for (int r = 0; r < 3; r++)
                for (int j = 0; j < 3; j++) v[k++] = rows[r][xs[j]];
            std::sort(v, v + 9);
            out[(size_t)y * w + x] = v[4];
        }
    }
    return out;
}

// depth.rs:653 `edge_weights`: exp(-|dI| / sigma) to the right and below
// (edge_mode 0). edge_mode 1 is not in the reference: the Gaussian of the
// guide gradient, exp(-dI^2 / (2 sigma^2)), the large-grid solve's weights.
template <class T>
void edge_weights(const T* g, size_t w, size_t h, T sigma, std::vector<T>& ax, std::vector<T>& ay, int edge_mode = 0) {
    T inv = T(-1) / rmax(sigma, LIT(1e-6));
    T inv2s2 = T(1) / (T(2) * sigma * sigma);
    auto wgt = [&](T a, T b) {
        T d = std::fabs(a - b);
        return edge_mode == 0 ? std::exp(d * inv) : std::exp(-(d * d * inv2s2));
    };
    ax.assign(w * h, T(0));
    ay.assign(w * h, T(0));
    for (size_t y = 0; y < h; y++)
        for (size_t x = 0; x + 1 < w; x++) ax[y * w + x] = wgt(g[y * w + x], g[y * w + x + 1]);
    for (size_t y = 0; y + 1 < h; y++)
        for (size_t x = 0; x < w; x++) ay[y * w + x] = wgt(g[y * w + x], g[(y + 1) * w + x]);
}

// depth.rs:677 `solve_rows` (Thomas algorithm per row) and :707 `solve_cols`,
// written once over a strided line.
template <class T>
void thomas_line(T* u, const T* f, const T* wd, const T* a, size_t n, size_t stride, T lam, T* cp, T* dp) {
    T prev_a = T(0);
    for (size_t i = 0; i < n; i++) {
        size_t k = i * stride;
        T ai = i + 1 < n ? a[k] : T(0);
        T diag = wd[k] + lam * (prev_a + ai);
        T lower = -lam * prev_a;
        T upper = -lam * ai;
        T m = diag - lower * (i > 0 ? cp[i - 1] : T(0));
        if (std::fabs(m) < LIT(1e-12)) m = LIT(1e-12);
        cp[i] = upper / m;
        dp[i] = (wd[k] * f[k] - lower * (i > 0 ? dp[i - 1] : T(0))) / m;
        prev_a = ai;
    }
    u[(n - 1) * stride] = dp[n - 1];
    for (size_t i = n - 1; i-- > 0;) u[i * stride] = dp[i] - cp[i] * u[(i + 1) * stride];
}
// depth.rs:677 `solve_rows`
template <class T>
void solve_rows(T* u, const T* f, const T* wd, const T* a, size_t w, size_t h, T lam) {
#pragma omp parallel for schedule(static)
    for (long y = 0; y < (long)h; y++) {
        std::vector<T> cp(w), dp(w);
        size_t o = (size_t)y * w;
        thomas_line<T>(u + o, f + o, wd + o, a + o, w, 1, lam, cp.data(), dp.data());
    }
}
// depth.rs:707 `solve_cols`
template <class T>
void solve_cols(T* u, const T* f, const T* wd, const T* a, size_t w, size_t h, T lam) {
#pragma omp parallel for schedule(static)
    for (long x = 0; x < (long)w; x++) {
        std::vector<T> cp(h), dp(h);
        thomas_line<T>(u + x, f + x, wd + x, a + x, h, w, lam, cp.data(), dp.data());
    }
}

// depth.rs:770-777
constexpr float MG_OMEGA = 0.8f;
constexpr size_t MG_PRE = 1, MG_POST = 1, MG_COARSE = 32, MG_MIN = 16;

// depth.rs:753 `MgLevel`
template <class T>
struct MgLevel {
    size_t w, h;
    std::vector<T> wd, ax, ay, dinv, x, b, r;
    MgLevel(size_t w_, size_t h_) : w(w_), h(h_) {
        size_t n = w * h;
        wd.assign(n, T(0));
        ax.assign(n, T(0));
        ay.assign(n, T(0));
        dinv.assign(n, T(0));
        x.assign(n, T(0));
        b.assign(n, T(0));
        r.assign(n, T(0));
    }
    inline T ax_at(const T* x_, size_t k, size_t i, size_t y) const {
        T xk = x_[k];
        T v = wd[k] * xk;
        if (i > 0) v += ax[k - 1] * (xk - x_[k - 1]);
        if (i + 1 < w) v += ax[k] * (xk - x_[k + 1]);
        if (y > 0) v += ay[k - w] * (xk - x_[k - w]);
        if (y + 1 < h) v += ay[k] * (xk - x_[k + w]);
        return v;
    }
    // depth.rs:786 `apply`: out_k = f(k, (A x)_k)
    template <class F>
    void apply(const T* x_, T* out, F f) const {
#pragma omp parallel for schedule(static) if (w * h >= (1u << 15))
        for (long y = 0; y < (long)h; y++)
            for (size_t i = 0; i < w; i++) {
                size_t k = (size_t)y * w + i;
                out[k] = f(k, ax_at(x_, k, i, (size_t)y));
            }
    }
    void set_dinv() {
        for (size_t y = 0; y < h; y++)
            for (size_t i = 0; i < w; i++) {
                size_t k = y * w + i;
                T v = wd[k];
                if (i > 0) v += ax[k - 1];
                if (i + 1 < w) v += ax[k];
                if (y > 0) v += ay[k - w];
                if (y + 1 < h) v += ay[k];
                dinv[k] = T(1) / rmax(v, LIT(1e-12));
            }
    }
    // depth.rs:837 `jacobi`
    void jacobi(bool zero_start) {
        const T om = (T)MG_OMEGA;
        if (zero_start) {
            for (size_t k = 0; k < x.size(); k++) x[k] = om * dinv[k] * b[k];
            return;
        }
        const T* xx = x.data();
        apply(xx, r.data(), [&](size_t k, T axk) { return xx[k] + om * dinv[k] * (b[k] - axk); });
        std::swap(x, r);
    }
    // depth.rs:852 `coarsen`
    MgLevel coarsen() const {
        size_t cw = half(w), ch = half(h);
        MgLevel c(cw, ch);
        coarsen_wd_into(c);
        for (size_t yy = 0; yy < ch; yy++)
            for (size_t y = 2 * yy; y < std::min(2 * yy + 2, h); y++)
                for (size_t xx = 0; xx + 1 < cw; xx++) c.ax[yy * cw + xx] += ax[y * w + 2 * xx + 1];
        for (size_t yy = 0; yy + 1 < ch; yy++) {
            size_t y = 2 * yy + 1;
            for (size_t xx = 0; xx < cw; xx++) {
                T a = T(0);
                for (size_t x_ = 2 * xx; x_ < std::min(2 * xx + 2, w); x_++) a += ay[y * w + x_];
                c.ay[yy * cw + xx] = a;
            }
        }
        return c;
    }
    // depth.rs:886 `coarsen_wd_into`
    void coarsen_wd_into(MgLevel& c) const {
        size_t cw = c.w;
        for (size_t yy = 0; yy < c.h; yy++) {
            for (size_t xx = 0; xx < cw; xx++) c.wd[yy * cw + xx] = T(0);
            for (size_t y = 2 * yy; y < std::min(2 * yy + 2, h); y++)
                for (size_t xx = 0; xx < cw; xx++) {
                    T a = T(0);
                    for (size_t x_ = 2 * xx; x_ < std::min(2 * xx + 2, w); x_++) a += wd[y * w + x_];
                    c.wd[yy * cw + xx] += a;
                }
        }
    }
};

// depth.rs:901 `prolong_add`, :911 `restrict`
template <class T>
void prolong_add(T* x, size_t w, size_t h, const T* xc, size_t cw) {
    for (size_t y = 0; y < h; y++)
        for (size_t i = 0; i < w; i++) x[y * w + i] += xc[(y / 2) * cw + i / 2];
}
template <class T>
void restrict_(const T* r, size_t w, size_t h, T* bc, size_t cw, size_t ch) {
    for (size_t yy = 0; yy < ch; yy++) {
        for (size_t xx = 0; xx < cw; xx++) bc[yy * cw + xx] = T(0);
        for (size_t y = 2 * yy; y < std::min(2 * yy + 2, h); y++)
            for (size_t xx = 0; xx < cw; xx++) {
                T a = T(0);
                for (size_t x_ = 2 * xx; x_ < std::min(2 * xx + 2, w); x_++) a += r[y * w + x_];
                bc[yy * cw + xx] += a;
            }
    }
}

// depth.rs:924 `vcycle`
template <class T>
void vcycle(std::vector<MgLevel<T>>& lv, size_t l) {
    MgLevel<T>& top = lv[l];
    if (l + 1 == lv.size()) {
        for (size_t k = 0; k < MG_COARSE; k++) top.jacobi(k == 0);
        return;
    }
    for (size_t k = 0; k < MG_PRE; k++) top.jacobi(k == 0);
    {
        const T* bb = top.b.data();
        top.apply(top.x.data(), top.r.data(), [&](size_t k, T axk) { return bb[k] - axk; });
    }
    restrict_<T>(top.r.data(), top.w, top.h, lv[l + 1].b.data(), lv[l + 1].w, lv[l + 1].h);
    vcycle(lv, l + 1);
    prolong_add<T>(top.x.data(), top.w, top.h, lv[l + 1].x.data(), lv[l + 1].w);
    for (size_t k = 0; k < MG_POST; k++) top.jacobi(false);
}

// depth.rs:1037 the CG's `dot`: f64 products summed (here in index order; the reference's rayon
// split only moves the sum at the 1e-16 level)
template <class T>
double dot(const T* a, const T* b, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += (double)a[i] * (double)b[i];
    return s;
}

// depth.rs:958 `WlsSolver`
template <class T>
struct WlsSolver {
    size_t w, h;
    T lambda;
    std::vector<T> ex, ey;
    std::vector<MgLevel<T>> levels;
    std::vector<T> r, z, p, ap, f;
    WlsSolver(const T* guide, size_t w_, size_t h_, T lambda_, T sigma_c, int edge_mode = 0) : w(w_), h(h_), lambda(lambda_) {
        edge_weights<T>(guide, w, h, sigma_c, ex, ey, edge_mode);
        MgLevel<T> top(w, h);
        for (size_t i = 0; i < w * h; i++) {
            top.ax[i] = lambda * ex[i];
            top.ay[i] = lambda * ey[i];
        }
        levels.push_back(std::move(top));
        while (std::max(levels.back().w, levels.back().h) > MG_MIN) levels.push_back(levels.back().coarsen());
        size_t n = w * h;
        r.assign(n, T(0));
        z.assign(n, T(0));
        p.assign(n, T(0));
        ap.assign(n, T(0));
        f.assign(n, T(0));
    }
    // depth.rs:992 `set_weights`
    void set_weights(const T* conf) {
        for (size_t i = 0; i < w * h; i++) levels[0].wd[i] = rmax(conf[i], T(0)) + LIT(1e-4);
        for (size_t l = 0; l < levels.size(); l++) {
            if (l > 0) levels[l - 1].coarsen_wd_into(levels[l]);
            levels[l].set_dinv();
        }
    }
    // depth.rs:1006 `solve`: returns (rel, iters)
    std::pair<T, size_t> solve(const T* d, size_t max_iters, T* u) {
        const T* wd = levels[0].wd.data();
        size_t n = w * h;
        if (w == 1 || h == 1) {
            if (h == 1) solve_rows<T>(u, d, wd, ex.data(), w, h, lambda);
            else solve_cols<T>(u, d, wd, ey.data(), w, h, lambda);
            return {T(0), 0};
        }
        const size_t TT = 3;
        std::vector<T> ones(n, T(1));
        std::copy(d, d + n, f.begin());
        for (size_t t = 1; t <= TT; t++) {
            T lam_t = LIT(1.5) * lambda * (T)std::pow(4.0, (double)(TT - t)) / ((T)std::pow(4.0, (double)TT) - T(1));
            const T* wt = t == 1 ? wd : ones.data();
            solve_rows<T>(u, f.data(), wt, ex.data(), w, h, lam_t);
            std::copy(u, u + n, f.begin());
            solve_cols<T>(u, f.data(), ones.data(), ey.data(), w, h, lam_t);
            std::copy(u, u + n, f.begin());
        }
        for (size_t i = 0; i < n; i++) f[i] = wd[i] * d[i];
        const T* b = f.data();
        double bnorm = std::max(std::sqrt(dot(b, b, n)), 1e-30);
        levels[0].apply(u, r.data(), [&](size_t k, T au) { return b[k] - au; });
        auto precond = [&]() {
            std::copy(r.begin(), r.end(), levels[0].b.begin());
            vcycle(levels, 0);
            std::copy(levels[0].x.begin(), levels[0].x.end(), z.begin());
        };
        precond();
        p = z;
        double rz = dot(r.data(), z.data(), n);
        T rel = (T)(std::sqrt(dot(r.data(), r.data(), n)) / bnorm);
        size_t iters = 0;
        for (size_t it = 0; it < max_iters; it++) {
            if (rel < LIT(1e-5)) break;
            iters++;
            levels[0].apply(p.data(), ap.data(), [](size_t, T v) { return v; });
            double pap = dot(p.data(), ap.data(), n);
            if (pap <= 0.0) break;
            T alpha = (T)(rz / pap);
            for (size_t i = 0; i < n; i++) u[i] += alpha * p[i];
            for (size_t i = 0; i < n; i++) r[i] -= alpha * ap[i];
            rel = (T)(std::sqrt(dot(r.data(), r.data(), n)) / bnorm);
            if (rel < LIT(1e-5)) break;
            precond();
            double rz_new = dot(r.data(), z.data(), n);
            T beta = (T)(rz_new / rz);
            rz = rz_new;
            for (size_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        }
        return {rel, iters};
    }
};

// depth.rs:141 `DepthMap`
template <class T>
struct DepthMap {
    std::vector<T> depth, conf, floor_cells;
    size_t w = 0, h = 0, dw = 0, dh = 0;
    T floor_ = T(0), p90 = T(0), rel = T(0);
    size_t iters = 0, iters_first = 0;
};

// depth.rs:1119 `depth_from_slices`
template <class T>
DepthMap<T> depth_from_slices(const std::vector<std::vector<T>>& slices, const Img3<T>& fused, const DepthParams& p) {
    DepthMap<T> out;
    size_t w = fused.w, h = fused.h, n = slices.size(), k = (size_t)1 << p.scale;
    std::vector<T> y_full = luma(fused);
    size_t dw, dh;
    std::vector<T> guide = block_mean<T>(y_full.data(), w, h, k, dw, dh);
    PeakTracker<T> tracker(dw * dh);
    {
        GuidedFilter<T> gf(guide, dw, dh, p.agg_radius, (T)p.agg_eps);
        std::vector<T> agg(dw * dh);
        for (size_t m = 0; m < n; m++) {
            if (p.agg_radius > 0) {
                gf.filter_into(slices[m].data(), agg.data());
                for (auto& v : agg) v = rmax(v, T(0));
                tracker.push(agg.data());
            } else {
                tracker.push(slices[m].data());
            }
        }
    }
    std::vector<T> depth_w, conf, mins;
    T floor_;
    tracker.finish((T)p.gate, depth_w, conf, mins, floor_);
    if (p.median) depth_w = median3<T>(depth_w.data(), dw, dh);
    T p90 = normalize_conf(conf);
    if (p.lambda > 0.0f) {
        WlsSolver<T> solver(guide.data(), dw, dh, (T)p.lambda, (T)p.sigma_c);
        solver.set_weights(conf.data());
        std::vector<T> u(dw * dh, T(0));
        auto rs = solver.solve(depth_w.data(), p.cg_iters, u.data());
        out.iters_first = rs.second;
        if (p.robust > 0.0f) {
            std::vector<T> w2(dw * dh);
            for (size_t i = 0; i < w2.size(); i++) w2[i] = conf[i] * rmin((T)p.robust / std::fabs(depth_w[i] - u[i]), T(1));
            solver.set_weights(w2.data());
            rs = solver.solve(depth_w.data(), p.cg_iters, u.data());
        }
        out.rel = rs.first;
        out.iters = rs.second;
        depth_w = u;
    }
    T max_d = (T)(n - 1);
    std::vector<T> depth;
    if (p.upsample == UP_BILINEAR) {
        depth = upsample_bilinear<T>(depth_w.data(), dw, dh, w, h, k);
    } else {
        GuidedFilter<T> g2(guide, dw, dh, p.up_radius, (T)p.up_eps);
        if (k == 1) {
            depth.resize(dw * dh);
            g2.filter_into(depth_w.data(), depth.data());
        } else {
            g2.coeffs_into(depth_w.data());
            std::vector<T> a = upsample_bilinear<T>(g2.s1.data(), dw, dh, w, h, k);
            std::vector<T> b = upsample_bilinear<T>(g2.s0.data(), dw, dh, w, h, k);
            depth.resize(w * h);
            for (size_t i = 0; i < w * h; i++) depth[i] = a[i] * y_full[i] + b[i];
        }
    }
    for (auto& v : depth) v = rclamp(v, T(0), max_d);
    out.conf = k == 1 ? conf : upsample_bilinear<T>(conf.data(), dw, dh, w, h, k);
    out.depth = std::move(depth);
    out.floor_cells = std::move(mins);
    out.w = w;
    out.h = h;
    out.dw = dw;
    out.dh = dh;
    out.floor_ = floor_;
    out.p90 = p90;
    return out;
}

}  // namespace orc
