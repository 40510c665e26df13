"""The oracle's frame preparation (oracle/orc_dust.hpp) against the reference's
own tests: dust.rs:716-778 (fill and flat take the dust out; the u16 path
agrees with the planar one; pull-push interpolates a hole) and prep.rs:135-182
(quarter turns compose and undo; the draft block mean with its ragged edge),
and the interleaved u16 steps of lapstack-web decode.rs:68-150."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.prep_cases import dust_frame, random_map, scene, spot_map, u16_of


def test_pull_push_interpolates_a_hole():
    """dust.rs:770-782."""
    w, h = 32, 24
    y, x = np.mgrid[0:h, 0:w]
    v = (np.float32(0.2) + np.float32(0.5) * (x.astype(np.float32) / np.float32(w))).astype(np.float32)
    wt = np.where((x >= 10) & (x < 16) & (y >= 8) & (y < 14), 0.0, 1.0).astype(np.float32)
    f = O.pull_push(v, wt)
    assert np.max(np.abs(f - v)[wt > 0]) < 1e-5
    assert np.max(np.abs(f - v)[wt == 0]) < 0.02


def test_fill_and_flat_take_the_dust_out():
    """dust.rs:716-759 on a map outlined like `detect` would: the fill within 0.07 and a third of the dust's
    darkening, the flat-field within 0.02, and the u16 path within 2/65535 of the planar one."""
    w, h = 400, 300
    bowls = [(100.0, 80.0, 12.0, 0.4), (300.0, 200.0, 20.0, 0.15)]
    m = spot_map(O, w, h, bowls)
    clean = scene(w, h)
    dusty = (clean * (dust_frame(w, h, bowls) / dust_frame(w, h, []))).astype(np.float32)
    err = lambda a, b: float(np.max(np.abs(a - b)))
    before = err(dusty, clean)
    assert before > 0.1
    filled = O.dust_apply(m, dusty)
    after = err(filled, clean)
    assert after < 0.07 and after < before / 3, (after, before)
    flat = O.dust_apply(O.DustMap(w, h, m.spots, "flat"), dusty)
    assert err(flat, clean) < 0.02
    rgb = u16_of(dusty)
    out = O.dust_apply_rgb16(m, rgb)
    worst = np.max(np.abs(np.transpose(out, (2, 0, 1)).astype(np.float32) / np.float32(65535.0) - filled))
    assert worst < 2.0 / 65535.0, worst
    # a frame of another size is left alone
    other = scene(200, 100)
    assert np.array_equal(O.dust_apply(m, other), other)


def test_overlapping_spots_keep_their_order():
    """Where two masks overlap, the later spot's value stays (fill) and the gains compound (flat)."""
    from oracle import oracle as M
    w, h = 64, 48
    mk = np.ones((10, 10), np.uint8)
    a = M.DustSpot(10, 10, mk, np.full((10, 10), 1.5, np.float32))
    b = M.DustSpot(15, 15, mk, np.full((10, 10), 1.25, np.float32))
    rgb = u16_of(scene(w, h) * np.float32(0.5))
    flat = M.dust_apply_rgb16(M.DustMap(w, h, [a, b], "flat"), rgb)
    once = M.dust_apply_rgb16(M.DustMap(w, h, [a], "flat"), rgb)
    twice = M.dust_apply_rgb16(M.DustMap(w, h, [b], "flat"), once)
    assert np.array_equal(flat, twice)
    fa = M.dust_apply_rgb16(M.DustMap(w, h, [a, b]), rgb)
    fb = M.dust_apply_rgb16(M.DustMap(w, h, [b, a]), rgb)
    assert not np.array_equal(fa[15:20, 15:20], fb[15:20, 15:20])


def ramp(w, h):
    y, x = np.mgrid[0:h, 0:w]
    return np.stack([(x + 10 * y + 100 * c).astype(np.float32) for c in range(3)])


def test_quarter_turns_compose_and_undo():
    """prep.rs:135-149."""
    im = ramp(5, 3)
    r1 = O.rotate(im, 1)
    assert r1.shape == (3, 5, 3)
    assert r1[0, 0, 2] == im[0, 0, 0] and r1[0, 0, 0] == im[0, 2, 0]
    assert np.array_equal(O.rotate(r1, 1), O.rotate(im, 2))
    assert np.array_equal(O.rotate(O.rotate(O.rotate(r1, 1), 1), 1), im)
    assert np.array_equal(O.rotate(r1, 3), im)
    assert O.rotate(im, 0, flip=True)[1, 0, 0] == im[1, 0, 4]


def test_draft_reduce_averages_blocks_and_the_ragged_edge():
    """prep.rs:169-181."""
    im = ramp(5, 3)
    r = O.draft_reduce(im, 1)
    assert r.shape == (3, 2, 3)
    assert abs(r[0, 0, 0] - 5.5) < 1e-6 and abs(r[0, 0, 2] - 9.0) < 1e-6 and abs(r[0, 1, 0] - 20.5) < 1e-6
    assert np.array_equal(O.draft_reduce(im, 0), im)


def test_u16_turn_draft_and_resize():
    """lapstack-web decode.rs:68, 92, 125 on interleaved u16: the turn as prep.rs's, the block mean rounded
    (s + n/2) / n, the resize keeping a constant and the frame's size."""
    im = ramp(5, 3)
    rgb = np.transpose(im, (1, 2, 0)).astype(np.uint16)
    for q in range(4):
        got = O.prep_rgb16(rgb, rotate=q)
        assert np.array_equal(np.transpose(got, (2, 0, 1)), O.rotate(im, q).astype(np.uint16))
    d = O.prep_rgb16(rgb, draft=1)
    assert d.shape == (2, 3, 3)
    assert d[0, 0, 0] == (0 + 1 + 10 + 11 + 2) // 4 and d[0, 2, 0] == (4 + 14 + 1) // 2 and d[1, 0, 0] == (20 + 21 + 1) // 2
    const = np.full((7, 9, 3), 1234, np.uint16)
    assert np.all(O.prep_rgb16(const, size=(13, 5)) == 1234)
    assert np.array_equal(O.prep_rgb16(rgb, size=(5, 3)), rgb)
    # the steps compose in decode's order: dust, turn, draft, size
    w, h = 96, 64
    m = random_map(O, w, h, 8, seed=3)
    f = u16_of(scene(w, h))
    step = O.dust_apply_rgb16(m, f)
    step = O.prep_rgb16(step, rotate=1)
    step = O.prep_rgb16(step, draft=2)
    step = O.prep_rgb16(step, size=(30, 40))
    assert np.array_equal(O.prep_rgb16(f, dust=m, rotate=1, draft=2, size=(30, 40)), step)


@pytest.mark.parametrize("mode", ["fill", "flat"])
def test_u16_dust_on_random_maps_stays_in_range(mode):
    w, h = 128, 96
    m = random_map(O, w, h, 20, seed=7, mode=mode)
    f = u16_of(scene(w, h))
    out = O.dust_apply_rgb16(m, f)
    changed = np.any(out != f, axis=2)
    covered = np.zeros((h, w), bool)
    for s in m.spots:
        hh, ww = s.mask.shape
        covered[s.y:s.y + hh, s.x:s.x + ww] |= s.mask.astype(bool)
    assert not np.any(changed & ~covered)  # only the spots' pixels change
    assert np.count_nonzero(changed) > 0.5 * np.count_nonzero(covered)
