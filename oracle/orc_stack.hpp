// Oracle (test infrastructure only; see orc_core.hpp): the per-frame
// sequence of stack.rs for in-memory 16-bit frames — AlignedFrames::get /
// register (stack.rs:513-530, 638-706), LazyFrames brightness (stack.rs:
// 276-437), fuse_range (stack.rs:740-826), fuse_and_depth (stack.rs:833-853)
// and the common-area crop of run_with (stack.rs:1047-1060).
#pragma once
#include "orc_align.hpp"
#include "orc_depth.hpp"
#include "orc_wav.hpp"

namespace orc {

struct StackParams {
    FuseParams fuse;
    bool align = true;
    AlignParams al;
    bool depth = true;
    DepthParams dp;
    bool brightness = true;
    bool crop = true;
    bool wav = false;  // stack.rs:857 `weighted`: the weighted average too (needs the depth pass)
    WavParams wp;
    // the engine's 16-bit storage to emulate (not the reference's): levels >= 1 rounded as stored
    // (orc_core.hpp `stored`), focus slices as IEEE half, aligned frames as u16 after their warp
    int storage = 0;
    // stack.rs:55 `slabs`: (size, overlap) of the slabs fused after the result (size 0: none)
    size_t slab_size = 0, slab_overlap = 0;
};

// stack.rs:76 `slab_ranges`
inline std::vector<std::array<size_t, 2>> slab_ranges(size_t count, size_t size, size_t overlap) {
    std::vector<std::array<size_t, 2>> out;
    if (count == 0) return out;
    size = std::min(std::max(size, (size_t)1), count);
    overlap = std::min(overlap, size - 1);
    size_t lo = 0;
    for (;;) {
        const size_t hi = std::min(lo + size - 1, count - 1);
        out.push_back({lo, hi});
        if (hi + 1 >= count) return out;
        lo = hi + 1 - overlap;
    }
}

// prep.rs:63 `resize_plane`: the plane through the Sim that scales it onto w x h with pixel centres
// corresponding (offset (k - 1)(s + 1) / 2s of the source size on each axis)
template <class T>
std::vector<T> resize_plane(const T* p, size_t pw, size_t ph, size_t w, size_t h, int interp) {
    if (pw == w && ph == h) return std::vector<T>(p, p + w * h);
    const double sw = (double)pw, sh = (double)ph, kx = (double)w / sw, ky = (double)h / sh;
    Sim sim;
    sim.v[0] = (kx - 1.0) * (sw + 1.0) / (2.0 * sw);
    sim.v[1] = (ky - 1.0) * (sh + 1.0) / (2.0 * sh);
    sim.v[2] = kx;
    sim.v[4] = ky / kx;
    std::vector<T> out;
    warp_plane<T>(p, pw, ph, sim, w, h, interp, out, nullptr);
    return out;
}

template <class T>
struct StackOutput {
    Img3<T> image;                 // fused, clamped, full frame (before the crop)
    std::vector<float> winner;     // fuse winner map, upsampled (stack.rs:244 Output::depth when depth is off)
    DepthMap<T> dm;                // depth pass
    std::vector<Sim> sims;
    std::vector<std::array<float, 3>> gains;
    std::vector<float> shares;
    Rect crop;                     // the common area (full frame when nothing is cut)
    size_t levels = 0;
    size_t align_evals = 0;
    Img3<T> wav;                   // the weighted average (wav.rs:92), when asked for
    // stack.rs:872 `fuse_slabs`: each slab's frames and its fused image (full frame, before any cut)
    std::vector<std::array<size_t, 2>> slab_rng;
    std::vector<Img3<T>> slabs;
};

// io.rs:89-94 u16 -> f32 as v * (1/65535) (an f32 multiply by the f32 reciprocal)
template <class T>
Img3<T> img_of_u16(const uint16_t* rgb, size_t w, size_t h) {
    Img3<T> im(w, h);
    const T inv = std::is_same<T, float>::value ? (T)(1.0f / 65535.0f) : (T)(1.0 / 65535.0);
    for (int c = 0; c < 3; c++)
        for (size_t i = 0; i < w * h; i++) im.p[c][i] = (T)rgb[3 * i + c] * inv;
    return im;
}

// io.rs:287 f32 -> u16 as (clamp01 * 65535 + 0.5) as u16
template <class T>
inline uint16_t u16_of(T v) {
    T c = rclamp(v, T(0), T(1));
    return (uint16_t)(c * LIT(65535.0) + LIT(0.5));
}

// stack.rs:1011 `run_with` for frames already decoded, one frame at a time:
// push() registers and gains each frame and folds it (stack.rs:740 `fuse_range`,
// the per-frame body of stack.rs:785-821), finish() takes the shares, the fused
// image, the depth pass (stack.rs:833 `fuse_and_depth`) and the crop.
template <class T>
struct StackRun {
    size_t w, h;
    StackParams sp;
    StackOutput<T> out;
    Fuser<T> fuser;
    std::vector<std::vector<T>> slices;
    bool aligned;
    bool freem[8];
    std::vector<T> prev_ref;
    BReference<T> bref;
    double ref_means[3] = {0, 0, 0};
    size_t i = 0;
    std::vector<Img3<T>> kept;  // the frames as folded, for the weighted average
    StackRun(size_t w_, size_t h_, size_t n, const StackParams& sp_) : w(w_), h(h_), sp(sp_), fuser(w_, h_, sp_.fuse) {
        out.levels = fuser.levels;
        fuser.storage = sp.storage;
        aligned = sp.align && n > 1;
        free_mask(sp.al, freem);
    }
    // `last`: no frame follows (the next frame's reference is not made)
    void push(const uint16_t* frame, bool last) {
        Img3<T> img = img_of_u16<T>(frame, w, h);
        Sim sim;
        std::array<float, 3> gain{1.0f, 1.0f, 1.0f};
        if (aligned) {
            // stack.rs:513 `register`
            std::vector<T> y = luma(img);
            if (i > 0) sim = multiscale_align<T>(prev_ref.data(), y.data(), w, h, out.sims.back(), freem, sp.al.coarsen, &out.align_evals);
            if (!last) {
                if (sim.is_id()) prev_ref = y;
                else warp_plane<T>(y.data(), w, h, sim, w, h, sp.al.interp, prev_ref, nullptr);
            }
            // stack.rs:662-679: warp, the pixel as shot where the source leaves the frame
            if (!sim.is_id()) {
                std::vector<uint8_t> valid;
                Img3<T> warped(w, h);
                warp_plane<T>(img.p[0].data(), w, h, sim, w, h, sp.al.interp, warped.p[0], &valid);
                warp_plane<T>(img.p[1].data(), w, h, sim, w, h, sp.al.interp, warped.p[1], nullptr);
                warp_plane<T>(img.p[2].data(), w, h, sim, w, h, sp.al.interp, warped.p[2], nullptr);
                for (int c = 0; c < 3; c++)
                    for (size_t k = 0; k < w * h; k++)
                        if (!valid[k]) warped.p[c][k] = img.p[c][k];
                img = std::move(warped);
            }
            // 16-bit storage keeps the warped frame as u16 (the brightness sums read the warp itself)
            Img3<T> as_stored;
            if (sp.storage != 0 && !sim.is_id()) {
                as_stored = img;
                const T inv = std::is_same<T, float>::value ? (T)(1.0f / 65535.0f) : (T)(1.0 / 65535.0);
                for (int c = 0; c < 3; c++)
                    for (auto& v : as_stored.p[c]) {
                        const float u = std::min(std::max((float)v * 65535.f + 0.5f, 0.f), 65535.f);
                        v = (T)(uint16_t)u * inv;
                    }
            }
            // stack.rs:680-690 brightness against frame 0 over the covered pixels
            if (sp.brightness) {
                if (i == 0) {
                    bref.init(img);
                } else {
                    double sf[3], so[3];
                    size_t cnt;
                    bsums<T>(img, &bref, sim, sf, so, cnt);
                    bratio(so, sf, cnt, gain.data());
                }
            }
            if (as_stored.w) img = std::move(as_stored);
            if (sp.brightness && i > 0) bapply<T>(img, gain.data());
        } else if (sp.brightness) {
            // stack.rs LazyFrames: frame 0's channel means, gains_to for the others
            if (i == 0) {
                bmeans<T>(img, ref_means);
            } else {
                double m[3];
                bmeans<T>(img, m);
                bratio(ref_means, m, (size_t)-1, gain.data());
                bapply<T>(img, gain.data());
            }
        }
        out.sims.push_back(sim);
        out.gains.push_back(gain);
        fuser.push(img, std::max(gain[0], std::max(gain[1], gain[2])));
        if (sp.depth) {
            size_t dw, dh;
            slices.push_back(focus_slice<T>(img, sp.dp, dw, dh));
            if (sp.storage != 0)
                for (auto& v : slices.back()) v = (T)f16_value(f16_bits((float)v));
        }
        if ((sp.wav && sp.depth) || sp.slab_size > 0) kept.push_back(img);
        i++;
    }
    void finish() {
        out.shares = fuser.shares();
        fuser.finish(out.image, out.winner);
        if (sp.depth) out.dm = depth_from_slices<T>(slices, out.image, sp.dp);
        if (sp.wav && sp.depth && !kept.empty()) out.wav = weighted_average<T>(kept, sp.dp, sp.wp, out.dm.floor_cells, &out.image);
        if (sp.slab_size > 0) {
            // stack.rs:740 `fuse_range` for each slab: a fresh fuser over the slab's frames as folded
            out.slab_rng = slab_ranges(kept.size(), sp.slab_size, sp.slab_overlap);
            for (const auto& r : out.slab_rng) {
                Fuser<T> f(w, h, sp.fuse);
                f.storage = sp.storage;
                for (size_t k = r[0]; k <= r[1]; k++) {
                    const auto& g = out.gains[k];
                    f.push(kept[k], std::max(g[0], std::max(g[1], g[2])));
                }
                Img3<T> im;
                std::vector<float> win;
                f.finish(im, win);
                out.slabs.push_back(std::move(im));
            }
        }
        out.crop = Rect{0, 0, w, h};
        if (aligned && sp.crop) out.crop = common_area(out.sims, w, h, sp.al.interp);
    }
};

template <class T>
StackOutput<T> run_stack(const uint16_t* const* frames, size_t n, size_t w, size_t h, const StackParams& sp) {
    StackRun<T> run(w, h, n, sp);
    for (size_t i = 0; i < n; i++) run.push(frames[i], i + 1 == n);
    run.finish();
    return std::move(run.out);
}

}  // namespace orc
