// Oracle (test infrastructure only; see orc_core.hpp): the weighted average
// of crates/lapstack-core/src/wav.rs. Every frame's pixels are averaged with
// weights that follow its contrast above the depth pass's per-cell noise
// floor: the focus measure block-averaged to the working grid (the depth
// pass's focus slice), box-smoothed, cut at (1 + gate) x floor and raised to
// `power`, smoothed again (guided by the fused luma, or a box mean), taken to
// full resolution bilinearly; then acc += w * frame, wsum += w over the
// frames in order, and acc / wsum clamped to [0, 1].
#pragma once
#include <cmath>
#include <memory>

#include "orc_depth.hpp"

namespace orc {

// wav.rs:52-80 WavParams and its defaults
struct WavParams {
    float power = 2.0f;
    size_t smooth = 3;
    float gate = 0.5f;
    bool edge = true;
};

// wav.rs:84 `weight`: (c - (1 + gate) f).max(0)^power + (1e-2 f)^power + 1e-30
template <class T>
inline T wav_weight(T c, T f, T gate, T power) {
    return std::pow(rmax(c - (T(1) + gate) * f, T(0)), power) + std::pow(LIT(1e-2) * f, power) + LIT(1e-30);
}

// wav.rs:92 `weighted_average` over the frames as folded (aligned, equalized), `floor` the depth
// pass's floor cells on the dw x dh grid, `guide` the fused image (may be null: the box mean)
template <class T>
Img3<T> weighted_average(const std::vector<Img3<T>>& frames, const DepthParams& dp, const WavParams& wp, const std::vector<T>& floor,
                         const Img3<T>* guide) {
    const size_t w = frames[0].w, h = frames[0].h, k = (size_t)1 << dp.scale;
    const size_t dw = blocks(w, k), dh = blocks(h, k), m = dw * dh;
    const T power = rmax((T)wp.power, T(0)), gate = rmax((T)wp.gate, T(0));
    std::unique_ptr<BoxFilter<T>> bf;
    if (wp.smooth > 0) bf.reset(new BoxFilter<T>(dw, dh, wp.smooth));
    std::unique_ptr<GuidedFilter<T>> gf;
    if (wp.edge && wp.smooth > 0 && guide) {
        size_t gw, gh;
        std::vector<T> y = luma(*guide);
        std::vector<T> g = block_mean(y.data(), guide->w, guide->h, k, gw, gh);
        gf.reset(new GuidedFilter<T>(g, dw, dh, wp.smooth, (T)dp.agg_eps));
    }
    Img3<T> acc(w, h);
    std::vector<T> wsum(w * h, T(0));
    for (const Img3<T>& f : frames) {
        size_t gw, gh;
        std::vector<T> g = focus_slice(f, dp, gw, gh);
        if (bf) g = bf->mean(g.data());
        for (size_t i = 0; i < m; i++) g[i] = wav_weight(g[i], floor[i], gate, power);
        if (gf) {
            std::vector<T> o(m);
            gf->filter_into(g.data(), o.data());
            for (size_t i = 0; i < m; i++) o[i] = rmax(o[i], LIT(1e-30));  // the guided filter undershoots at an edge
            g.swap(o);
        } else if (bf) {
            g = bf->mean(g.data());
        }
        std::vector<T> wf = upsample_bilinear(g.data(), dw, dh, w, h, k);
        for (int c = 0; c < 3; c++)
            for (size_t i = 0; i < w * h; i++) acc.p[c][i] += wf[i] * f.p[c][i];
        for (size_t i = 0; i < w * h; i++) wsum[i] += wf[i];
    }
    for (int c = 0; c < 3; c++)
        for (size_t i = 0; i < w * h; i++) acc.p[c][i] = rclamp(acc.p[c][i] / wsum[i], T(0), T(1));
    return acc;
}

}  // namespace orc
