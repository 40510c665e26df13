// Oracle (test infrastructure only; see orc_core.hpp): the frame preparation
// a decoded 16-bit frame goes through before it is aligned and folded.
//
// - dust.rs:478-593 DustMap::apply / apply_rgb16 and pull_push: every dust
//   spot of the map filled from its surroundings (pull-push over a window in
//   which every spot's pixels are weighted out) or divided by its measured
//   attenuation (flat-field);
// - prep.rs:16 rotate and prep.rs:77 reduce on planar f32 frames (stack.rs:309
//   prep_frame);
// - the same three steps on interleaved u16 frames as the browser engine does
//   them (lapstack-web decode.rs:68 rotate, :92 reduce, :125 resize, and
//   lib.rs:766-779 decode: dust, turn, draft reduction, then the run's size).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "orc_core.hpp"
#include "orc_depth.hpp"

namespace orc {

// dust.rs:85 Spot
struct DustSpot {
    size_t x = 0, y = 0, w = 0, h = 0;
    std::vector<uint8_t> mask;  // w*h, 1 = dust
    std::vector<float> gain;    // w*h attenuation (>= 1), read in flat mode
};

// dust.rs:105 DustMap; mode 0 = DustMode::Fill, 1 = DustMode::Flat (dust.rs:42)
struct DustMap {
    size_t w = 0, h = 0;
    int mode = 0;
    std::vector<DustSpot> spots;
};

// dust.rs:591 `pull_push`: v weighted by wt REDUCEd (v*wt and wt) down to one cell; on the way back
// every pixel keeps its own value where it has weight, the coarser level's where it has none,
// blending in between (wc = clamp(d, 0, 1)).
template <class T>
std::vector<T> pull_push(const std::vector<T>& v, const std::vector<T>& wt, size_t w, size_t h) {
    std::vector<std::vector<T>> nums(1), dens(1);
    std::vector<std::pair<size_t, size_t>> dims{{w, h}};
    nums[0].resize(w * h);
    for (size_t i = 0; i < w * h; i++) nums[0][i] = v[i] * wt[i];
    dens[0] = wt;
    while ((dims.back().first > 1 || dims.back().second > 1) && dims.size() < 24) {
        const size_t cw = dims.back().first, ch = dims.back().second;
        std::vector<T> n2, d2;
        size_t ow, oh;
        reduce<T>(nums.back().data(), cw, ch, n2, ow, oh);
        reduce<T>(dens.back().data(), cw, ch, d2, ow, oh);
        nums.push_back(std::move(n2));
        dens.push_back(std::move(d2));
        dims.push_back({ow, oh});
    }
    const size_t top = dims.size() - 1;
    std::vector<T> f(nums[top].size());
    for (size_t i = 0; i < f.size(); i++) f[i] = dens[top][i] > LIT(1e-9) ? nums[top][i] / dens[top][i] : T(0);
    for (size_t l = top; l-- > 0;) {
        const size_t ow = dims[l].first, oh = dims[l].second;
        std::vector<T> up = expand<T>(f.data(), dims[l + 1].first, dims[l + 1].second, ow, oh);
        f.assign(ow * oh, T(0));
        for (size_t i = 0; i < ow * oh; i++) {
            const T n = nums[l][i], d = dens[l][i], u = up[i];
            const T wc = rclamp(d, T(0), T(1));
            f[i] = d > LIT(1e-9) ? wc * (n / d) + (T(1) - wc) * u : u;
        }
    }
    return f;
}

// dust.rs:542-590: one channel of a frame, planar f32 or interleaved u16
struct PlaneF32 {
    float* p;
    size_t w;
    float get(size_t x, size_t y) const { return p[y * w + x]; }
    void set(size_t x, size_t y, float v) { p[y * w + x] = v; }
};
struct PlaneU16 {
    uint16_t* rgb;
    size_t w;
    int c;
    float get(size_t x, size_t y) const { return (float)rgb[3 * (y * w + x) + c] / 65535.0f; }
    void set(size_t x, size_t y, float v) {
        const float q = std::min(std::max(v, 0.0f), 1.0f) * 65535.0f + 0.5f;  // NaN clamps to 0 (as u16 of NaN)
        rgb[3 * (y * w + x) + c] = q != q ? 0 : (uint16_t)std::min(q, 65535.0f);
    }
};

// dust.rs:499 `apply_plane`: every spot in turn, flattened or filled from its window
template <class P>
void dust_apply_plane(const DustMap& m, P& plane) {
    for (const DustSpot& s : m.spots) {
        if (m.mode == 1) {
            for (size_t sy = 0; sy < s.h; sy++)
                for (size_t sx = 0; sx < s.w; sx++)
                    if (s.mask[sy * s.w + sx]) {
                        const size_t x = s.x + sx, y = s.y + sy;
                        plane.set(x, y, plane.get(x, y) * s.gain[sy * s.w + sx]);
                    }
            continue;
        }
        const size_t pad = std::max(std::max(s.w, s.h) / 2, (size_t)6);
        const size_t x0 = s.x >= pad ? s.x - pad : 0, y0 = s.y >= pad ? s.y - pad : 0;
        const size_t x1 = std::min(s.x + s.w + pad, m.w), y1 = std::min(s.y + s.h + pad, m.h);
        const size_t ww = x1 - x0, wh = y1 - y0;
        std::vector<float> v(ww * wh), wt(ww * wh, 1.0f);
        for (size_t y = 0; y < wh; y++)
            for (size_t x = 0; x < ww; x++) v[y * ww + x] = plane.get(x0 + x, y0 + y);
        for (const DustSpot& o : m.spots) {
            if (!(o.x < x1 && o.x + o.w > x0 && o.y < y1 && o.y + o.h > y0)) continue;
            for (size_t sy = 0; sy < o.h; sy++)
                for (size_t sx = 0; sx < o.w; sx++) {
                    const size_t x = o.x + sx, y = o.y + sy;
                    if (o.mask[sy * o.w + sx] && x >= x0 && x < x1 && y >= y0 && y < y1) wt[(y - y0) * ww + (x - x0)] = 0.0f;
                }
        }
        const std::vector<float> filled = pull_push<float>(v, wt, ww, wh);
        for (size_t sy = 0; sy < s.h; sy++)
            for (size_t sx = 0; sx < s.w; sx++)
                if (s.mask[sy * s.w + sx]) {
                    const size_t x = s.x + sx, y = s.y + sy;
                    plane.set(x, y, filled[(y - y0) * ww + (x - x0)]);
                }
    }
}

// dust.rs:478 `apply` (planar f32 frame of the map's size; other sizes are left alone)
inline void dust_apply(const DustMap& m, Img3<float>& f) {
    if (m.spots.empty() || f.w != m.w || f.h != m.h) return;
    for (int c = 0; c < 3; c++) {
        PlaneF32 p{f.p[c].data(), f.w};
        dust_apply_plane(m, p);
    }
}

// dust.rs:487 `apply_rgb16` (interleaved u16, w*h*3 samples)
inline void dust_apply_rgb16(const DustMap& m, uint16_t* rgb, size_t w, size_t h) {
    if (m.spots.empty() || w != m.w || h != m.h) return;
    for (int c = 0; c < 3; c++) {
        PlaneU16 p{rgb, w, c};
        dust_apply_plane(m, p);
    }
}

// ------------------------------------------------------------------ prep.rs
// prep.rs:16 `rotate`: quarter turns clockwise, after a horizontal mirror when flip_h
inline Img3<float> rotate(const Img3<float>& im, int quarters, bool flip_h) {
    const size_t w = im.w, h = im.h;
    const int q = ((quarters % 4) + 4) % 4;
    if (q == 0 && !flip_h) return im;
    const size_t ow = q % 2 ? h : w, oh = q % 2 ? w : h;
    Img3<float> out(ow, oh);
    for (int c = 0; c < 3; c++)
        for (size_t oy = 0; oy < oh; oy++)
            for (size_t ox = 0; ox < ow; ox++) {
                size_t sx, sy;
                switch (q) {
                    case 0: sx = ox, sy = oy; break;
                    case 1: sx = oy, sy = h - 1 - ox; break;
                    case 2: sx = w - 1 - ox, sy = h - 1 - oy; break;
                    default: sx = w - 1 - oy, sy = ox; break;
                }
                if (flip_h) sx = w - 1 - sx;
                out.p[c][oy * ow + ox] = im.p[c][sy * w + sx];
            }
    return out;
}

// prep.rs:77 `reduce`: 2^levels blocks averaged in f64 (the ragged edge averages what is there)
inline Img3<float> draft_reduce(const Img3<float>& im, int levels) {
    if (levels == 0) return im;
    const size_t k = (size_t)1 << levels, w = im.w, h = im.h;
    const size_t ow = std::max((w + k - 1) / k, (size_t)1), oh = std::max((h + k - 1) / k, (size_t)1);
    Img3<float> out(ow, oh);
    for (int c = 0; c < 3; c++)
        for (size_t oy = 0; oy < oh; oy++) {
            const size_t y0 = oy * k, y1 = std::min((oy + 1) * k, h);
            for (size_t ox = 0; ox < ow; ox++) {
                const size_t x0 = ox * k, x1 = std::min((ox + 1) * k, w);
                double s = 0.0;
                for (size_t y = y0; y < y1; y++)
                    for (size_t x = x0; x < x1; x++) s += (double)im.p[c][y * w + x];
                out.p[c][oy * ow + ox] = (float)(s / (double)((y1 - y0) * (x1 - x0)));
            }
        }
    return out;
}

// ------------------------------------------- interleaved u16 (lapstack-web decode.rs)
// decode.rs:68 `rotate` (no mirror)
inline std::vector<uint16_t> rotate_rgb16(const uint16_t* in, size_t w, size_t h, int quarters, size_t& ow, size_t& oh) {
    const int q = ((quarters % 4) + 4) % 4;
    ow = q % 2 ? h : w;
    oh = q % 2 ? w : h;
    std::vector<uint16_t> out(ow * oh * 3);
    for (size_t oy = 0; oy < oh; oy++)
        for (size_t ox = 0; ox < ow; ox++) {
            size_t sx, sy;
            switch (q) {
                case 0: sx = ox, sy = oy; break;
                case 1: sx = oy, sy = h - 1 - ox; break;
                case 2: sx = w - 1 - ox, sy = h - 1 - oy; break;
                default: sx = w - 1 - oy, sy = ox; break;
            }
            for (int c = 0; c < 3; c++) out[3 * (oy * ow + ox) + c] = in[3 * (sy * w + sx) + c];
        }
    return out;
}

// decode.rs:92 `reduce`: integer block sums, (s + n/2) / n
inline std::vector<uint16_t> reduce_rgb16(const uint16_t* in, size_t w, size_t h, int levels, size_t& ow, size_t& oh) {
    const size_t k = (size_t)1 << levels;
    ow = std::max((w + k - 1) / k, (size_t)1);
    oh = std::max((h + k - 1) / k, (size_t)1);
    std::vector<uint16_t> out(ow * oh * 3);
    for (size_t oy = 0; oy < oh; oy++) {
        const size_t y0 = oy * k, y1 = std::min((oy + 1) * k, h);
        for (size_t ox = 0; ox < ow; ox++) {
            const size_t x0 = ox * k, x1 = std::min((ox + 1) * k, w);
            uint64_t s[3] = {0, 0, 0};
            for (size_t y = y0; y < y1; y++)
                for (size_t x = x0; x < x1; x++)
                    for (int c = 0; c < 3; c++) s[c] += in[3 * (y * w + x) + c];
            const uint64_t n = (uint64_t)((y1 - y0) * (x1 - x0));
            for (int c = 0; c < 3; c++) out[3 * (oy * ow + ox) + c] = (uint16_t)((s[c] + n / 2) / n);
        }
    }
    return out;
}

// decode.rs:125 `resize`: bilinear in f64 with centres kept, edge-clamped, + 0.5 truncated
inline std::vector<uint16_t> resize_rgb16(const uint16_t* in, size_t sw, size_t sh, size_t w, size_t h) {
    std::vector<uint16_t> out(w * h * 3);
    const double kx = (double)sw / (double)w, ky = (double)sh / (double)h;
    for (size_t y = 0; y < h; y++) {
        const double fy = std::min(std::max(((double)y + 0.5) * ky - 0.5, 0.0), (double)(sh - 1));
        const size_t y0 = (size_t)std::floor(fy), y1 = std::min(y0 + 1, sh - 1);
        const double ty = fy - std::floor(fy);
        for (size_t x = 0; x < w; x++) {
            const double fx = std::min(std::max(((double)x + 0.5) * kx - 0.5, 0.0), (double)(sw - 1));
            const size_t x0 = (size_t)std::floor(fx), x1 = std::min(x0 + 1, sw - 1);
            const double tx = fx - std::floor(fx);
            const size_t a = 3 * (y0 * sw + x0), b = 3 * (y0 * sw + x1), c = 3 * (y1 * sw + x0), d = 3 * (y1 * sw + x1);
            for (int ch = 0; ch < 3; ch++) {
                const double top = (double)in[a + ch] * (1.0 - tx) + (double)in[b + ch] * tx;
                const double bot = (double)in[c + ch] * (1.0 - tx) + (double)in[d + ch] * tx;
                out[3 * (y * w + x) + ch] = (uint16_t)(top * (1.0 - ty) + bot * ty + 0.5);
            }
        }
    }
    return out;
}

// lapstack-web lib.rs:766-779 `decode` + :784 `decode_for_run`: the dust map (frames of its size only),
// the turn, the draft reduction, then the run's size (rw x rh; 0: as prepared)
inline std::vector<uint16_t> prep_rgb16(const DustMap* dust, int quarters, int draft, std::vector<uint16_t> f, size_t w, size_t h,
                                        size_t rw, size_t rh, size_t& ow, size_t& oh) {
    if (dust) dust_apply_rgb16(*dust, f.data(), w, h);
    if (quarters % 4 != 0) f = rotate_rgb16(f.data(), w, h, quarters, w, h);
    if (draft > 0) f = reduce_rgb16(f.data(), w, h, draft, w, h);
    if (rw && rh && (rw != w || rh != h)) {
        f = resize_rgb16(f.data(), w, h, rw, rh);
        w = rw;
        h = rh;
    }
    ow = w;
    oh = h;
    return f;
}

}  // namespace orc
