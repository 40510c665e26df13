"""Pins the oracle to the reference's own known-answer and property tests.

Each test restates one #[test] of crates/lapstack-core/src (cited), so the
CPU restatement is checked against the values the reference asserts before
it is trusted as the checker for the CUDA engine. CPU only.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.fixtures import blur, checker, halves, lcg_plane, rms, xorshift_img


# ------------------------------------------------------------------ pyramid.rs
def test_reflect_101():  # pyramid.rs:253
    assert [O.reflect(-1, 5), O.reflect(-2, 5), O.reflect(5, 5), O.reflect(6, 5), O.reflect(3, 2), O.reflect(-3, 1)] == [
        1, 2, 3, 2, 1, 0]


def test_kernel_sums_to_one():  # pyramid.rs:263
    k = np.array([1, 4, 6, 4, 1], np.float32) / np.float32(16)
    assert abs(float(k.sum()) - 1.0) < 1e-6
    assert abs(float(np.float32(2) * (k[0] + k[2] + k[4])) - 1.0) < 1e-6


def test_reduce_preserves_constant():  # pyramid.rs:271
    im = np.full((22, 37), 0.7, np.float32)
    r = O.reduce(im)
    assert r.shape == (11, 19)
    assert np.all(np.abs(r - 0.7) < 1e-5)
    e = O.expand(r, 37, 22)
    assert np.all(np.abs(e - 0.7) < 1e-5)


@pytest.mark.parametrize("w,h", [(64, 48), (63, 47), (1, 1), (2, 3), (129, 5)])
def test_perfect_reconstruction(w, h):  # pyramid.rs:282
    im = xorshift_img(w, h, 7 + w)
    levels = O.auto_levels(w, h, 1)
    back = O.build_collapse(im, levels)
    assert np.all(np.abs(back - im) < 1e-5)


def test_auto_levels_targets_top_size():  # pyramid.rs:298
    assert O.auto_levels(8280, 5520, 32) == 7
    assert O.auto_levels(16, 16, 32) == 1


# --------------------------------------------------------------------- fuse.rs
def test_binomial_weights():  # fuse.rs:582
    assert list(O.binomial(0)) == [1.0]
    assert list(O.binomial(1)) == [0.25, 0.5, 0.25]
    k = np.array([1, 4, 6, 4, 1], np.float32) / np.float32(16)
    assert np.all(np.abs(O.binomial(2) - k) < 1e-6)


def test_winner_shares_count_detail_cells_only():  # fuse.rs:528
    win = np.array([0, 0, 0, 1, 1, 2], np.uint16)
    best = np.array([0.001, 0.002, 0.001, 1.0, 0.5, 0.2], np.float32)
    s = O.winner_shares(win, best, 3)
    assert list(s) == [0.0, np.float32(2.0) / np.float32(3.0), np.float32(1.0) / np.float32(3.0)]
    assert np.all(O.winner_shares(win, np.zeros(6, np.float32), 3) == 0)
    img = checker(64, 64, 8)
    f = O.Fuser(64, 64)
    for _ in range(3):
        f.push(img)
    s = f.shares()
    assert len(s) == 3 and abs(s[0] - 1.0) < 1e-6 and s[1] == 0.0 and s[2] == 0.0


def test_identical_frames_are_a_fixed_point():  # fuse.rs:592
    im = checker(70, 50, 7)
    f = O.Fuser(70, 50)
    for _ in range(3):
        f.push(im)
    out, depth = f.finish()
    assert rms(out, im) < 1e-5
    assert np.all(depth == 0.0)


@pytest.mark.parametrize("variant", ["base", "r0", "avg"])
def test_picks_the_sharp_half_from_each_frame(variant):  # fuse.rs:604
    w, h = 96, 64
    sharp = checker(w, h, 6)
    soft = blur(sharp, 6, O)
    a, b = halves(sharp, soft, w)
    p = O.FuseParams(depth_level=0)
    if variant == "r0":
        p.energy_radius = 0
    if variant == "avg":
        p.top_rule = "avg"
    f = O.Fuser(w, h, p)
    f.push(a)
    f.push(b)
    out, depth = f.finish()
    assert rms(out, sharp) < 0.6 * rms(a, sharp)
    n = depth.size
    x = np.arange(depth.size) % w
    left = np.count_nonzero((x < w // 2 - 8) & (depth.reshape(-1) == 0.0))
    right = np.count_nonzero((x >= w // 2 + 8) & (depth.reshape(-1) == 1.0))
    assert left > 0.9 * (n / 2 - 8 * h) and right > 0.9 * (n / 2 - 8 * h)


def test_halo_weight_is_monotonic_and_bounded():  # fuse.rs:644
    assert abs(O.halo_weight(1e-4 - 1e-8, 3.0) - 1.0) < 1e-5
    assert O.halo_weight(1e-3, 2.0) > O.halo_weight(1e-4, 2.0)
    assert O.halo_weight(1e-4, 4.0) / O.halo_weight(1e-5, 4.0) > 9e3
    assert O.halo_weight(0.0, 8.0) > 0.0 and math.isfinite(O.halo_weight(0.0, 8.0))
    assert math.isfinite(O.halo_weight(1e3, 8.0))


def test_halo_control_keeps_identical_frames():  # fuse.rs:655
    im = checker(70, 50, 7)
    f = O.Fuser(70, 50, O.FuseParams(halo=2.0, levels=3, depth_level=1))
    for _ in range(3):
        f.push(im)
    out, depth = f.finish()
    assert rms(out, im) < 1e-5
    assert np.all(depth == 0.0)


def test_halo_control_coarse_levels_follow_the_guide():  # fuse.rs:674
    w, h = 192, 144
    a = checker(w, h, 6)
    b = blur(a, 64, O)
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    d2 = (x - np.float32(96.0)) ** 2 + (y - np.float32(72.0)) ** 2
    bump = np.float32(0.35) * np.exp(-d2 / np.float32(2.0 * 20.0 ** 2))
    b = np.minimum(b + bump[None], 1.0).astype(np.float32)

    def fuse(halo, order):
        f = O.Fuser(w, h, O.FuseParams(levels=5, depth_level=2, halo=halo))
        f.push(order[0])
        f.push(order[1])
        return f.finish()[0]

    off = rms(fuse(0.0, [a, b]), a)
    assert off > 0.05
    for halo in [1.0, 2.0, 4.0, 8.0]:
        assert rms(fuse(halo, [a, b]), a) < 0.15 * off
    assert rms(fuse(2.0, [b, a]), a) < 0.15 * off


def test_top_rule_two_frames_matches_eq12():  # fuse.rs:705
    a = checker(40, 40, 4)
    b = np.full_like(a, 0.5)
    # with one band-pass level the residuals are the frames REDUCEd once
    ta = np.stack([O.reduce(a[c]) for c in range(3)])
    tb = np.stack([O.reduce(b[c]) for c in range(3)])
    top = O.fuse_residuals(np.stack([ta, tb]), O.FuseParams(levels=1))
    assert rms(top, ta) < 1e-6


# -------------------------------------------------------------------- align.rs
def test_reduce_burt_keeps_a_constant_plane():  # align.rs:969
    for w, h in [(1, 1), (2, 3), (3, 4), (4, 5), (5, 5), (6, 7), (9, 65), (10, 66), (33, 130)]:
        d = O.reduce_burt(np.full((h, w), 0.75, np.float32))
        assert d.shape == ((h + 1) // 2, (w + 1) // 2)
        assert np.all(np.abs(d - 0.75) < 1e-6)
    lv = O.gauss_levels(np.full((300, 40), 0.25, np.float32))
    assert [(l.shape[1], l.shape[0]) for l in lv] == [(20, 150), (10, 75), (5, 38)]
    assert all(np.all(np.abs(l - 0.25) < 1e-6) for l in lv)


def _two_pass_cost(a, b, sim):
    bw, valid = O.warp_plane(b, sim, "spline4x4")
    v = valid.astype(bool)
    av, bv = a[v].astype(np.float64), bw[v].astype(np.float64)
    return math.sqrt(np.sum(((av - av.mean()) - (bv - bv.mean())) ** 2) / v.sum())


def test_cost_matches_the_two_pass_definition():  # align.rs:987
    w, h = 96, 72
    i = np.arange(w * h)
    a = (((i * 7919) % 1000) / np.float32(1000.0)).astype(np.float32).reshape(h, w)
    b = ((((i * 104729 + 13) % 1000) / np.float32(1000.0)) + np.float32(0.2)).astype(np.float32).reshape(h, w)
    sims = [O.SIM_ID, [0.03, -0.02, 1.02, 0.01, 1.0, 0.0, 0.0, 0.0], [0.0, 0.0, 1.0, 0.0, 1.0, 0.01, 0.03, -0.02]]
    for s in sims:
        want = _two_pass_cost(a, b, s)
        got = O.warp_cost(a, b, s)
        assert abs(got - want) < 1e-5 * want
    assert O.warp_cost(a, a, O.SIM_ID) < 1e-9
    assert O.warp_cost(a, a, [2.0, 0, 1, 0, 1, 0, 0, 0]) == 1e9


def test_level_steps_move_the_edge_by_a_level_pixel():  # align.rs:1016
    w, h = 8000, 6000
    step, tol = O.level_steps(list(range(8)), 3, w, h)
    r = max(w, h) / 2
    gain = [w, h, r, r, h / 2, h / 2, w / 4, h / 4]
    for k in range(8):
        assert abs(step[k] * gain[k] - 8.0) < 1e-9 and abs(tol[k] * gain[k] - 0.8) < 1e-9
    assert step[0] * w == 8.0 and step[2] * w / 2.0 == 8.0
    s2, _ = O.level_steps([0, 3], 0, w, h)
    assert len(s2) == 2 and s2[0] == 1.0 / w


def test_common_area():  # align.rs:1034, 1040
    assert O.common_area([O.SIM_ID, O.SIM_ID], 640, 480) == (0, 0, 640, 480)
    w, h = 640, 480
    s = [10.0 / w, 0, 1, 0, 1, 0, 0, 0]
    assert O.common_area([O.SIM_ID, s], w, h) == (12, 2, w - 12, h - 4)
    assert O.common_area([O.SIM_ID, s], w, h, "lanczos3") == (13, 3, w - 13, h - 6)
    assert O.common_area([O.SIM_ID, s], w, h, "bilinear") == (11, 1, w - 11, h - 2)
    assert O.common_area([O.SIM_ID, s], w, h, "nearest") == (10, 0, w - 10, h)


def test_common_area_rotation_is_inside_every_frame():  # align.rs:1122
    w, h = 640, 480
    sims = [O.SIM_ID, [-0.01, 0.02, 1.03, 0.02, 1, 0, 0, 0], [0.005, -0.01, 0.98, -0.015, 1, 0, 0, 0]]
    x, y, rw, rh = O.common_area(sims, w, h)
    assert rw > w // 2 and rh > h // 2 and (rw, rh) != (w, h)
    for s in sims[1:]:
        inv = O.mat_inverse(O.sim_matrix(s, w, h))
        for px, py in [(x, y), (x + rw - 1, y), (x, y + rh - 1), (x + rw - 1, y + rh - 1)]:
            d = inv[2, 0] * px + inv[2, 1] * py + inv[2, 2]
            sx = (inv[0, 0] * px + inv[0, 1] * py + inv[0, 2]) / d
            sy = (inv[1, 0] * px + inv[1, 1] * py + inv[1, 2]) / d
            assert 2 <= sx <= w - 3 and 2 <= sy <= h - 3


@pytest.mark.parametrize("kind", O.INTERPS)
def test_every_kernel_interpolates(kind):  # align.rs:1056
    w, h = 40, 30
    src = ((np.arange(w * h) * 7919 % 1000) / np.float32(1000.0)).astype(np.float32).reshape(h, w)
    o, _ = O.warp_plane(src, O.SIM_ID, kind)
    assert np.all(np.abs(o - src) < 1e-6)
    o, valid = O.warp_plane(src, [3.0 / w, -2.0 / h, 1, 0, 1, 0, 0, 0], kind)
    assert np.all(valid[6:h - 6, 6:w - 6] == 1)
    assert np.all(np.abs(o[6:h - 6, 6:w - 6] - src[8:h - 4, 3:w - 9]) < 1e-5)


@pytest.mark.parametrize("kind", O.INTERPS)
def test_kernels_reproduce_a_ramp(kind):  # align.rs:1079
    w, h = 48, 40
    i = np.arange(w * h)
    ramp = ((i % w) + 0.5 * (i // w)).astype(np.float32).reshape(h, w)
    o, _ = O.warp_plane(ramp, [2.3 / w, 1.6 / h, 1, 0, 1, 0, 0, 0], kind)
    yy, xx = np.mgrid[8:h - 8, 8:w - 8]
    sx, sy = xx - 2.3, yy - 1.6
    want = (np.round(sx) + 0.5 * np.round(sy)) if kind == "nearest" else (sx + 0.5 * sy)
    tol = 0.03 if kind == "lanczos3" else 1e-3
    assert np.all(np.abs(o[8:h - 8, 8:w - 8] - want) < tol)


@pytest.mark.parametrize("t", [0.0, 0.1, 0.5, 0.9])
def test_kernel_weights(t):  # align.rs:1099
    for kind in ["spline4x4", "bicubic", "spline6x6", "lanczos3"]:
        ws = O.interp_weights(kind, t)
        assert abs(ws.sum() - 1.0) < 1e-6
        if t == 0.0:
            c = len(ws) // 2 - 1
            assert abs(ws[c] - 1.0) < 1e-6 and all(abs(v) < 1e-6 for i, v in enumerate(ws) if i != c)


def test_homography_round_trip():  # align.rs:1154
    w, h = 640, 480
    s = [0.01, -0.02, 1.03, 0.02, 1.02, 0.01, 0.03, -0.02]
    m = O.sim_matrix(s, w, h)
    inv = O.mat_inverse(m)
    assert inv[2, 2] == 1.0
    for x, y in [(0.0, 0.0), (100.0, 37.0), (639.0, 479.0), (320.0, 240.0)]:
        d = m[2] @ [x, y, 1]
        fx, fy = (m[0] @ [x, y, 1]) / d, (m[1] @ [x, y, 1]) / d
        d2 = inv[2] @ [fx, fy, 1]
        bx, by = (inv[0] @ [fx, fy, 1]) / d2, (inv[1] @ [fx, fy, 1]) / d2
        assert abs(bx - x) < 1e-9 and abs(by - y) < 1e-9
    a = O.sim_matrix([0, 0, 1, 0, 1.5, 0.2, 0, 0], w, h)
    assert tuple(a[:2] @ [320, 250, 1]) == (322.0, 255.0)
    assert np.array_equal(O.mat_inverse(O.sim_matrix(O.SIM_ID, w, h)), np.eye(3))


def test_projective_warp_and_common_area():  # align.rs:1187
    w, h = 64, 48
    ramp = np.array([(i % w) + 0.5 * (i // w) for i in range(w * h)], np.float32).reshape(h, w)
    s = [0, 0, 1, 0, 1, 0.01, 0.04, -0.03]  # Sim { px: 0.04, py: -0.03, shear: 0.01, ..id }
    o, valid = O.warp_plane(ramp, s, "bilinear")
    inv = O.mat_inverse(O.sim_matrix(s, w, h))

    def src(x, y):
        d = inv[2] @ [x, y, 1.0]
        return (inv[0] @ [x, y, 1.0]) / d, (inv[1] @ [x, y, 1.0]) / d

    for y in range(4, h - 4):
        for x in range(4, w - 4):
            sx, sy = src(float(x), float(y))
            assert valid[y, x] == 1
            assert abs(float(o[y, x]) - (sx + 0.5 * sy)) < 1e-3, (x, y)
    x0, y0, rw, rh = O.common_area([O.SIM_ID, s], w, h, "bilinear")
    assert (rw, rh) != (w, h) and rw > w // 2 and rh > h // 2
    m = 1.0  # Interp::Bilinear.margin(): half its 2 taps
    for px, py in [(x0, y0), (x0 + rw - 1, y0), (x0, y0 + rh - 1), (x0 + rw - 1, y0 + rh - 1)]:
        sx, sy = src(float(px), float(py))
        assert m <= sx <= w - 1 - m and m <= sy <= h - 1 - m, (px, py, sx, sy)


def test_multiscale_align_recovers_a_shift():
    """The search finds a known sub-pixel similarity on a textured plane."""
    w, h = 256, 192
    rng = np.random.default_rng(3)
    base = rng.random((h, w)).astype(np.float32)
    k = np.array([1, 4, 6, 4, 1], np.float32) / np.float32(16)
    for _ in range(3):
        base = O.window_sum(base, k)
    truth = [1.7 / w, -0.8 / h, 1.004, 0.003, 1, 0, 0, 0]
    tg, _ = O.warp_plane(base, truth)  # tg = base moved by truth; search maps tg back onto base
    got, evals = O.multiscale_align(tg, base)
    assert evals > 20
    inv = O.mat_inverse(O.sim_matrix(got, w, h))
    fwd = O.sim_matrix(truth, w, h)
    # composing the found transform with the truth gives (nearly) the identity at the frame's corners
    for x, y in [(20, 20), (w - 20, 20), (20, h - 20), (w - 20, h - 20)]:
        p = fwd @ [x, y, 1]
        q = inv @ p
        assert abs(q[0] / q[2] - x) < 0.15 and abs(q[1] / q[2] - y) < 0.15


def test_nelder_mead_step_counts_add_up_to_the_evaluations():
    """The oracle's step counters (used to size the device search's batches) account for every
    evaluation: n+1 per search's first simplex, 1 per accepted reflection, 2 per expansion or
    accepted contraction, 2+n per shrink (align.rs:796)."""
    w, h = 256, 192
    rng = np.random.default_rng(5)
    base = rng.random((h, w)).astype(np.float32)
    k = np.array([1, 4, 6, 4, 1], np.float32) / np.float32(16)
    for _ in range(3):
        base = O.window_sum(base, k)
    tg, _ = O.warp_plane(base, [2.3 / w, 1.1 / h, 0.997, -0.002, 1, 0, 0, 0])
    O.nm_step_kinds(reset=True)
    _, evals = O.multiscale_align(tg, base)
    s = O.nm_step_kinds(reset=True)
    n = 4  # similarity: shift x, y, scale, rotation
    assert s["searches"] >= 2
    assert evals == s["searches"] * (n + 1) + s["accepted"] + 2 * (s["expanded"] + s["contracted"]) + (2 + n) * s["shrunk"]
    assert O.nm_step_kinds() == dict(accepted=0, expanded=0, contracted=0, shrunk=0, searches=0)


# --------------------------------------------------------------- brightness.rs
def _bscene(w, h):  # brightness.rs:148 `scene`
    y, x = np.mgrid[0:h, 0:w]
    t = (((x * 7 + y * 3) % 23).astype(np.float32) / np.float32(23.0)).astype(np.float32)
    r = np.float32(0.2) + np.float32(0.5) * t
    g = np.float32(0.3) + np.float32(0.3) * (x.astype(np.float32) / np.float32(w))
    b = np.float32(0.1) + np.float32(0.6) * (y.astype(np.float32) / np.float32(h))
    return np.stack([r, g, b]).astype(np.float32)


def _blur5(im):  # brightness.rs:163 `blur5`: 5x5 box, edge-clamped
    _, h, w = im.shape
    p = np.pad(im.astype(np.float64), ((0, 0), (2, 2), (2, 2)), mode="edge")
    s = sum(p[:, dy:dy + h, dx:dx + w] for dy in range(5) for dx in range(5))
    return (s / 25.0).astype(np.float32)


def test_brightness_gains():  # brightness.rs:185-213
    a = _bscene(160, 120)
    assert np.all(O.brightness_gains(a, a, O.SIM_ID) == 1.0)
    assert np.all(O.brightness_gains(a, a, [0.05, -0.02, 1.01, 0.01, 1, 0, 0, 0]) == 1.0)
    b = _blur5(a) * np.array([0.8, 0.9, 1.1], np.float32)[:, None, None]
    g = O.brightness_gains(a, b, O.SIM_ID)
    for got, want in zip(g, [1.25, 1.0 / 0.9, 1.0 / 1.1]):
        assert abs(got / want - 1.0) < 0.01
    assert np.all(O.brightness_gains_to(a, a) == 1.0)
    tiny = (a * np.float32(0.001)).astype(np.float32)
    assert np.all(O.brightness_gains(a, tiny, O.SIM_ID) == 4.0)


# -------------------------------------------------------------------- depth.rs
def test_box_filter_matches_naive():  # depth.rs:1212
    w, h, r = 23, 17, 3
    src = lcg_plane(w * h, 5).reshape(h, w)
    m = O.box_mean(src, r)
    for y in range(h):
        for x in range(w):
            win = src[max(0, y - r):y + r + 1, max(0, x - r):x + r + 1]
            assert abs(m[y, x] - win.mean()) < 1e-4


def test_guided_filter_flat_guide_is_box_mean():  # depth.rs:1233
    w, h = 40, 30
    p = lcg_plane(w * h, 9).reshape(h, w)
    q = O.guided_filter(np.full((h, w), 0.5, np.float32), p, 2, 1e-3)
    m = O.box_mean(O.box_mean(p, 2), 2)
    assert np.all(np.abs(q - m) < 1e-4)


def test_rdf_taps_are_zero_mean():  # depth.rs:1248
    t = O.rdf_taps(1, 3)
    assert abs(float(t[:, 2].sum())) < 1e-6
    assert int((t[:, 2] > 0).sum()) == 5
    assert np.all(np.abs(O.focus_measure(np.full((20, 20), 0.3, np.float32))) < 1e-6)


def _track(profile):
    d, c, _, _ = O.peak_track(np.asarray(profile, np.float32).reshape(-1, 1), gate=2.0)
    return float(d[0]), float(c[0])


def test_peak_tracker_profiles():  # depth.rs:1267
    d, c = _track([0.1, 0.5, 1.0, 0.5, 0.1])
    assert abs(d - 2.0) < 1e-5 and c > 0.5
    d, _ = _track([0.1, 0.4, 1.0, 0.8, 0.1])
    assert 2.0 < d < 2.5
    assert abs(_track([1.0, 0.5, 0.1])[0]) < 1e-6
    assert abs(_track([0.1, 0.5, 1.0])[0] - 2.0) < 1e-6
    assert abs(_track([0.1, 1.0, 1.0, 0.1])[0] - 1.5) < 1e-5
    _, c2 = _track([0.1, 1.0, 0.1, 0.95, 0.1])
    _, c1 = _track([0.1, 1.0, 0.1, 0.1, 0.1])
    assert c2 < 0.2 and c1 > 0.5
    assert _track([0.3, 0.3, 0.3, 0.3])[1] < 1e-6
    assert _track([0.7])[0] == 0.0


def test_wls_keeps_confident_data_and_fills_holes():  # depth.rs:1291
    w, h = 32, 24
    y, x = np.mgrid[0:h, 0:w]
    d = x.astype(np.float32)
    conf = np.ones((h, w), np.float32)
    hole = (x >= 10) & (x < 22) & (y >= 6) & (y < 18)
    conf[hole] = 0.0
    d[hole] = 100.0
    guide = np.full((h, w), 0.5, np.float32)
    u, rel, _ = O.wls_solve(d, conf, guide, 5.0, 0.05, 500)
    assert rel < 1e-4
    assert np.all(np.abs(u[4:h - 4, 4:w - 4] - x[4:h - 4, 4:w - 4]) < 0.6)
    u0, _, _ = O.wls_solve(d, np.ones((h, w), np.float32), guide, 0.0, 0.05, 10)
    assert np.all(np.abs(u0 - d) < 1e-3)


def test_wls_respects_guide_edges():  # depth.rs:1324
    w, h = 40, 20
    x = np.arange(w)[None, :].repeat(h, 0)
    d = np.where(x >= w // 2, 10.0, 0.0).astype(np.float32)
    guide = np.where(x >= w // 2, 0.9, 0.1).astype(np.float32)
    u, _, _ = O.wls_solve(d, np.full((h, w), 0.2, np.float32), guide, 50.0, 0.02, 300)
    assert u[10, w // 2 - 1] < 0.5 and u[10, w // 2] > 9.5
    v, _, _ = O.wls_solve(d, np.full((h, w), 0.2, np.float32), np.full((h, w), 0.5, np.float32), 50.0, 0.02, 300)
    assert v[10, w // 2 - 1] > 2.0 and v[10, w // 2] < 8.0


def test_end_to_end_two_frames():  # depth.rs:1367
    w, h = 128, 96
    sharp = checker(w, h, 5, tint=(1.0, 1.0, 1.0))
    soft = blur(sharp, 6, O)
    a, b = halves(sharp, soft, w)
    p = O.DepthParams(lam=5.0)
    slices = np.stack([O.focus_slice(a, p), O.focus_slice(b, p)])
    depth, conf, _, _ = O.depth_from_slices(slices, sharp, p)
    x = np.arange(w)[None, :].repeat(h, 0)
    want = np.where(x < w // 2, 0.0, 1.0)
    mask = np.abs(x - w // 2) >= 6
    bad = np.count_nonzero((np.abs(depth - want) > 0.25) & mask)
    assert bad < w * h / 100
    assert conf.mean() > 0.2


def test_fp64_oracle_agrees_with_fp32_path():
    """The double instantiation runs the same algorithm: on a small stack the
    fused images agree to f32 rounding."""
    w, h = 70, 50
    a = checker(w, h, 7)
    b = blur(a, 3, O)
    f32, f64 = O.Fuser(w, h), O.Fuser(w, h, fp64=True)
    for im in (a, b):
        f32.push(im)
        f64.push(im.astype(np.float64))
    i32, _ = f32.finish()
    i64, _ = f64.finish()
    assert np.max(np.abs(i32 - i64)) < 1e-5
