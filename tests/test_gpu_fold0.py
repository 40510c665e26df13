"""The fused level-0 fold kernel (one read of every frame: REDUCE, focus
slice and selection together) against the two-kernel path it replaces on the
interior tiles, bit for bit, and through it against the oracle.

The two-kernel path (LSB_FLAG_TWO_KERNEL_FOLD0) is itself held bit-exact to
the oracle by the other parity tests; here every output of a stack -- the
fused 16-bit and f32 images, the winner map, the shares, the focus slices
(through the noise-floor cells) and the depth -- must be identical with and
without the fused kernel, over the three storage types, the three energy
radii, chroma energies, uneven gains, aligned frames and frame sizes whose
tiles are partly interior.
"""
import numpy as np
import pytest

import lapstack_b200 as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def run(frames, storage, fused, fuse, align=None, depth=None):
    n, h, w, _ = frames.shape
    eng = L.Engine(storage=storage, fused_fold0=fused)
    st = eng.stack(w, h, n, fuse, align, depth, brightness=True)
    for f in frames:
        st.push_u16(f)
    st.set_count(n)  # fold from device memory in one pass (the whole stack per level)
    out = st.finish()
    st.close()
    eng.close()
    return out


def same(a, b):
    assert np.array_equal(a.image_u16, b.image_u16)
    assert np.array_equal(a.image, b.image)
    assert np.array_equal(a.winner, b.winner)
    assert np.array_equal(a.shares, b.shares)
    if a.depth is not None:
        assert np.array_equal(a.depth.floor, b.depth.floor)
        assert np.array_equal(a.depth.depth, b.depth.depth)


def uneven(frames):
    """Per-frame brightness changes, so that the gains (and the 16-bit storage scales) differ."""
    return np.stack([np.clip(f.astype(np.float64) * (1.0 - 0.04 * (k % 4)), 0, 65535).astype(np.uint16) for k, f in enumerate(frames)])


@pytest.mark.parametrize("storage", ["f32", "unorm16", "f16"])
@pytest.mark.parametrize("radius,chroma", [(1, False), (0, False), (2, False), (1, True)])
def test_fused_level0_is_the_two_kernel_fold(storage, radius, chroma):
    fr = uneven(L.synth_stack(L.SynthSpec(512, 384, 5, mag_step=0.003, seed=41))[0])
    fuse = L.FuseParams(energy_radius=radius, use_chroma=chroma, depth_level=0 if chroma else 2)
    depth = L.DepthParams() if radius == 1 else None
    same(run(fr, storage, True, fuse, depth=depth), run(fr, storage, False, fuse, depth=depth))


@pytest.mark.parametrize("w,h", [(1001, 333), (141, 81), (650, 130)])
def test_fused_level0_odd_sizes(w, h):
    """Sizes whose interior tiles meet rows and columns of border tiles of every kind, u16 rows that
    start half way into a 4-byte word (odd widths), and frames with a single interior tile."""
    fr = uneven(L.synth_stack(L.SynthSpec(w, h, 4, seed=43))[0])
    for storage in ("f32", "unorm16"):
        same(run(fr, storage, True, L.FuseParams(), depth=L.DepthParams()),
             run(fr, storage, False, L.FuseParams(), depth=L.DepthParams()))


@pytest.mark.parametrize("n,top", [(1, "avg"), (2, "de"), (3, "avg")])
def test_fused_level0_few_frames_f32_planes_match_oracle(n, top):
    """Few frames, gains of exactly 1 and a 1- or 2-level pyramid: the fused image's f32 planes equal
    the oracle's bit for bit, so every rounding of the level-0 Laplacian is the reference's (a fused
    multiply-add anywhere would move some of them by an ulp)."""
    fr = L.synth_stack(L.SynthSpec(1024, 768, n, mag_step=0.0, noise_std=0.003, seed=5))[0]
    for levels in (1, 2):
        fuse = L.FuseParams(levels=levels, top_rule=top)
        ref = O.run_stack(fr, O.StackParams(fuse=O.FuseParams(levels=levels, top_rule=top), align=None, depth=None, brightness=False))
        eng = L.Engine(storage="f32")
        st = eng.stack(1024, 768, n, fuse, None, None, brightness=False)
        for f in fr:
            st.push_u16(f)
        out = st.finish()
        assert np.array_equal(ref.image.astype(np.float32), out.image), (levels, np.count_nonzero(ref.image.astype(np.float32) != out.image))
        assert np.array_equal(ref.winner, out.winner)


def test_fused_level0_aligned_16bit_frames():
    """Aligned stacks with 16-bit storage fold their warped u16 frames through the fused kernel."""
    fr = L.synth_stack(L.SynthSpec(640, 480, 4, warp=True, mag_step=0.0, seed=47))[0]
    al = L.AlignParams(coarsen=1)
    same(run(fr, "unorm16", True, L.FuseParams(), align=al, depth=L.DepthParams()),
         run(fr, "unorm16", False, L.FuseParams(), align=al, depth=L.DepthParams()))


def test_fused_level0_matches_oracle():
    """FP32 storage, u16 frames with uneven gains: the fused path against the oracle directly."""
    fr = uneven(L.synth_stack(L.SynthSpec(768, 512, 5, mag_step=0.002, seed=53))[0])
    ref = O.run_stack(fr, O.StackParams(align=None, depth=O.DepthParams()))
    out = run(fr, "f32", True, L.FuseParams(), depth=L.DepthParams())
    assert np.array_equal(ref.gains, out.gains)
    assert np.array_equal(ref.image_u16, out.image_u16)
    assert np.array_equal(ref.image.astype(np.float32), out.image)
    assert np.array_equal(ref.winner, out.winner)
    assert np.array_equal(ref.floor_cells.astype(np.float32), out.depth.floor)
