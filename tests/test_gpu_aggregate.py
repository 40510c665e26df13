"""The depth pass's guided-filter aggregation (depth.rs:352-406 GuidedFilter,
depth.rs:285 BoxFilter) fed to the peak tracker (depth.rs:547), in its two
forms on the device: moving f64 window sums at radii 3 and 8 (the default)
and direct window sums of 2R+1 taps (LSB_FLAG_DIRECT_WINDOW_SUMS). Both are
the reference's sums whenever its f64 sums are exact, so the two engines'
depth maps must agree bit for bit, and each must agree with the oracle as
the other depth tests ask.

Cases: FP32 slices (lsb_depth_from_slices) and FP16 slices (a stack with
16-bit storage); grid widths that are and are not a multiple of the 16-byte
copy (the slice window is then staged by plain loads); grids smaller than
one tile, so every tile is a border tile.
"""
import numpy as np
import pytest

import lapstack_b200 as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def assert_same(a, b, what):
    bad = np.count_nonzero(a != b)
    assert bad == 0, f"{what}: {bad} of {a.size} differ (max |d| {np.max(np.abs(a.astype(np.float64) - b))})"


@pytest.fixture(scope="module")
def engines():
    run, direct = L.Engine(), L.Engine(direct_window_sums=True)
    yield run, direct
    run.close()
    direct.close()


def slices_of(w, h, n, seed):
    """Focus slices with a peak per cell at a smooth, cell-varying depth, values over several decades."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    z = (n - 1) * (0.5 + 0.4 * np.sin(x / 23.0) * np.cos(y / 17.0))
    k = np.arange(n, dtype=np.float32)[:, None, None]
    amp = np.exp(rng.normal(0.0, 1.5, (h, w))).astype(np.float32)
    s = amp * np.exp(-0.5 * ((k - z) / 1.3) ** 2) + rng.random((n, h, w)).astype(np.float32) * 1e-3
    return s.astype(np.float32)


def guide_image(w, h, seed):
    rng = np.random.default_rng(seed + 100)
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    g = 0.5 + 0.3 * np.sin(x / 11.0) * np.cos(y / 7.0) + 0.05 * rng.random((h, w))
    return np.stack([g, g * 0.9, g * 1.1]).astype(np.float32)


@pytest.mark.parametrize("radius", [3, 8])
@pytest.mark.parametrize("w,h", [(256, 160), (203, 131), (40, 24)])
def test_fp32_slices_moving_sums_equal_direct_sums_and_the_oracle(engines, radius, w, h):
    n = 9
    sl = slices_of(w, h, n, seed=w + radius)
    fused = guide_image(w, h, seed=h)
    p = L.DepthParams(agg_radius=radius, lam=2.0, scale=0)  # the depth grid is the slices' grid
    run = L.depth_from_slices(sl, fused, p, engine=engines[0])
    direct = L.depth_from_slices(sl, fused, p, engine=engines[1])
    assert_same(direct.depth, run.depth, "depth")
    assert_same(direct.conf, run.conf, "confidence")
    assert run.floor_value == direct.floor_value and run.p90 == direct.p90
    rd, rc, _, st = O.depth_from_slices(sl, fused, O.DepthParams(agg_radius=radius, lam=2.0, scale=0))
    d = np.abs(rd.astype(np.float64) - run.depth)
    assert np.mean(d > 1e-3 * (n - 1)) <= 1e-3
    assert np.mean(np.abs(rc - run.conf) > 1e-3) <= 1e-3
    assert run.floor_value == np.float32(st["floor"])


@pytest.mark.parametrize("radius", [3, 8])
@pytest.mark.parametrize("w,h", [(512, 320), (472, 300)])
def test_fp16_slices_of_a_stack_moving_sums_equal_direct_sums(radius, w, h):
    """A 16-bit stack keeps its focus slices as FP16 on the depth grid (here w/2 x h/2: 256 and 236
    cells wide, the second not a multiple of the 8-half copy)."""
    frames = L.synth_stack(L.SynthSpec(w, h, 6, seed=31 + radius))[0]
    dp = L.DepthParams(agg_radius=radius, scale=1)
    outs = []
    for direct in (False, True):
        e = L.Engine(storage="unorm16", direct_window_sums=direct)
        st = e.stack(w, h, len(frames), L.FuseParams(), None, dp)
        try:
            for f in frames:
                st.push_u16(f)
            outs.append(st.finish())
        finally:
            st.close()
            e.close()
    run, direct = outs
    assert_same(direct.depth.depth, run.depth.depth, "depth")
    assert_same(direct.depth.conf, run.depth.conf, "confidence")
    assert_same(direct.depth.floor, run.depth.floor, "floor cells")
    assert run.depth.floor_value == direct.depth.floor_value and run.depth.p90 == direct.depth.p90
