"""The slabs on the device (stack.rs:740 fuse_range, stack.rs:872 fuse_slabs)
and the resize (prep.rs:46 resize, :63 resize_plane; stack.rs:951
restretched) against the oracle.

- every slab of an aligned stack, FP32 and 16-bit storage, bit-exact with the
  oracle's slabs (a fresh fuser over the slab's frames as folded);
- with halo control on (to 1e-5: its weights go through ln and exp);
- cut to the common area and resized back to the frame (Spline4x4), bit-exact
  with the oracle's resize of the oracle's cut slab;
- Engine.resize bit-exact with the oracle for every interpolation kernel;
- the stack's own results untouched, and the whole-stack slab equal to them.
"""
import numpy as np
import pytest

import lapstack_b200 as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu

INTERPS = ["nearest", "bilinear", "bicubic", "spline4x4", "spline6x6", "lanczos3"]


def assert_same(a, b, what):
    bad = np.count_nonzero(a != b)
    assert bad == 0, f"{what}: {bad} of {a.size} differ (max |d| {np.max(np.abs(a.astype(np.float64) - b))})"


def synth(w, h, n, **kw):
    return L.synth_stack(L.SynthSpec(w, h, n, **kw))[0]


def gpu_stack(fr, fuse, al, storage="f32"):
    n, h, w, _ = fr.shape
    eng = L.Engine(storage=storage)
    st = eng.stack(w, h, n, fuse, al, None)
    for f in fr:
        st.push_u16(f)
    return eng, st


def oracle_params(fuse, al, storage, slabs):
    f = O.FuseParams(levels=fuse.levels, halo=fuse.halo)
    a = None if al is None else O.AlignParams(coarsen=al.coarsen)
    return O.StackParams(fuse=f, align=a, depth=None, storage=storage, slabs=slabs)


@pytest.mark.parametrize("storage,halo", [("f32", 0.0), ("unorm16", 0.0), ("f16", 0.0), ("f32", 2.0)])
def test_slabs_match_oracle(storage, halo):
    fr = synth(416, 288, 7, warp=True, mag_step=0.002, noise_std=0.002, seed=0x5AB)
    fuse, al = L.FuseParams(halo=halo), L.AlignParams(coarsen=1)
    ref = O.run_stack(fr, oracle_params(fuse, al, storage, (3, 1)))

    # halo control's weights go through the f32 ln and exp (the platform libm in the oracle, CUDA's on the
    # device): its images are held to 1e-5, as the fuser's halo test holds them
    def close(want, got, what):
        if halo > 0.0:
            assert np.max(np.abs(want.astype(np.float64) - got)) <= 1e-5, what
        else:
            assert_same(want.astype(np.float32), got, what)

    eng, st = gpu_stack(fr, fuse, al, storage)
    try:
        out = st.finish()
        close(ref.image, out.image, "the stack's fused image")
        assert ref.slab_ranges == L.slab_ranges(7, 3, 1)
        got = list(st.slabs(3, 1))
        assert [(k, c, lo, hi) for k, c, lo, hi, _ in got] == [(k, len(ref.slab_ranges), lo, hi)
                                                              for k, (lo, hi) in enumerate(ref.slab_ranges)]
        for (k, _, lo, hi, img), want in zip(got, ref.slabs):
            close(want, img, f"slab {k} ({lo}..{hi})")
        # the stack's own results stay as they were, and the whole-stack slab is the fused image
        assert_same(out.shares, st.shares(), "shares after the slabs")
        assert_same(out.image, st.fuse_range(0, 6), "whole-stack slab")
    finally:
        st.close()
        eng.close()


def test_slab_cut_and_restretched_matches_oracle():
    """stack.rs:886-889: the slab cut to the common area and brought back to the frame's size."""
    fr = synth(384, 256, 5, warp=True, mag_step=0.0, noise_std=0.002, seed=0x5AC, warp_shift=10.0)
    fuse, al = L.FuseParams(), L.AlignParams(coarsen=1)
    ref = O.run_stack(fr, oracle_params(fuse, al, "f32", (2, 0)))
    eng, st = gpu_stack(fr, fuse, al)
    try:
        out = st.finish()
        x, y, w, h = out.crop
        assert (w, h) != (384, 256), out.crop  # the warps cut something
        for (lo, hi), want in zip(ref.slab_ranges, ref.slabs):
            cut = want[:, y:y + h, x:x + w].astype(np.float32)
            got = st.fuse_range(lo, hi, rect=out.crop)
            assert_same(cut, got, f"cut slab {lo}..{hi}")
            back = O.resize(cut, 384, 256, interp=3)
            got = st.fuse_range(lo, hi, rect=out.crop, size=(384, 256))
            assert got.shape == (3, 256, 384)
            assert_same(back, got, f"restretched slab {lo}..{hi}")
    finally:
        st.close()
        eng.close()


@pytest.mark.parametrize("interp", range(6))
def test_resize_matches_oracle(interp):
    rng = np.random.default_rng(40 + interp)
    a = rng.random((3, 77, 101), dtype=np.float32)
    eng = L.Engine()
    try:
        for w, h in [(130, 90), (64, 50), (101, 77), (33, 120)]:
            assert_same(O.resize(a, w, h, interp), eng.resize(a, w, h, interp), f"{INTERPS[interp]} {w}x{h}")
        one = eng.resize(a[0], 40, 30, interp)
        assert one.shape == (30, 40)
    finally:
        eng.close()


def test_fuse_range_refuses_bad_arguments():
    fr = synth(128, 96, 3, seed=3)
    eng, st = gpu_stack(fr, L.FuseParams(), None)
    try:
        with pytest.raises(L.LsbError, match="finished"):
            st.fuse_range(0, 1)
        st.finish()
        for kw in [dict(lo=2, hi=1), dict(lo=0, hi=3), dict(lo=0, hi=1, rect=(100, 0, 40, 10)),
                   dict(lo=0, hi=1, rect=(0, 0, 0, 10)), dict(lo=0, hi=1, interp=6)]:
            lo, hi = kw.pop("lo"), kw.pop("hi")
            with pytest.raises(L.LsbError):
                st.fuse_range(lo, hi, **kw)
        assert st.fuse_range(1, 1).shape == (3, 96, 128)
    finally:
        st.close()
        eng.close()
