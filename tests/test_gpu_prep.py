"""Frame preparation on the device (lsb_prep.cu) against the oracle
(oracle/orc_dust.hpp), bit for bit:

- dust.rs:487 apply_rgb16, fill (pull-push) and flat, on maps outlined as
  dust.rs:315 detect would and on random maps with spots at the frame's edges
  and spots whose masks overlap (run in layers, in order), one large spot;
- the quarter turns and draft block means of lapstack-web decode.rs:68/92,
  and the resize of a frame of another size (decode.rs:125), alone and
  composed in decode's order;
- a stack whose frames are prepared as they are pushed (dust, a turn, a
  draft level; and frames of other sizes), aligned, against the oracle's run
  over the oracle's prepared frames: transforms, gains and the fused image.
"""
import numpy as np
import pytest

import lapstack_b200 as L
from oracle import oracle as O
from tests.prep_cases import dust_frame, random_map, scene, spot_map, u16_of

pytestmark = pytest.mark.gpu


def assert_same(a, b, what):
    bad = np.count_nonzero(a != b)
    assert bad == 0, f"{what}: {bad} of {a.size} differ (max |d| {np.max(np.abs(a.astype(np.int64) - b.astype(np.int64)))})"


def both_maps(make):
    return make(O), make(L)


@pytest.fixture(scope="module")
def eng():
    e = L.Engine()
    yield e
    e.close()


@pytest.mark.parametrize("mode", ["fill", "flat"])
def test_dust_outlined_spots_match_oracle(eng, mode):
    w, h = 400, 300
    bowls = [(100.0, 80.0, 12.0, 0.4), (300.0, 200.0, 20.0, 0.15), (40.0, 220.0, 8.0, 0.25)]
    mo, ml = both_maps(lambda M: spot_map(M, w, h, bowls, mode=mode))
    dusty = u16_of(scene(w, h) * (dust_frame(w, h, bowls) / dust_frame(w, h, [])))
    want = O.prep_rgb16(dusty, dust=mo)
    got = eng.prep_frame(dusty, L.FramePrep(dust=ml))
    assert np.count_nonzero(want != dusty) > 100
    assert_same(want, got, f"{mode} dust")


@pytest.mark.parametrize("mode,seed", [("fill", 1), ("fill", 2), ("flat", 3)])
def test_dust_random_maps_with_edges_and_overlaps_match_oracle(eng, mode, seed):
    w, h = 257, 193
    mo, ml = both_maps(lambda M: random_map(M, w, h, 40, seed=seed, mode=mode))
    f = u16_of(scene(w, h))
    assert_same(O.prep_rgb16(f, dust=mo), eng.prep_frame(f, L.FramePrep(dust=ml)), f"{mode} random map {seed}")
    # twice in a row: the scratch of one call leaves nothing behind for the next
    assert_same(O.prep_rgb16(f, dust=mo), eng.prep_frame(f, L.FramePrep(dust=ml)), "second call")


def test_dust_large_spot_matches_oracle(eng):
    """A spot 150 px across: a 300 px window, a pull-push pyramid of 9 levels in the CTA's scratch."""
    w, h = 640, 480
    mo, ml = both_maps(lambda M: spot_map(M, w, h, [(320.0, 240.0, 75.0, 0.3)]))
    f = u16_of(scene(w, h) * (dust_frame(w, h, [(320.0, 240.0, 75.0, 0.3)]) / dust_frame(w, h, [])))
    assert_same(O.prep_rgb16(f, dust=mo), eng.prep_frame(f, L.FramePrep(dust=ml)), "large spot")


@pytest.mark.parametrize("rotate,draft,size", [(1, 0, None), (2, 0, None), (3, 0, None), (0, 1, None), (1, 2, None), (0, 3, None),
                                               (0, 0, (150, 90)), (3, 1, (70, 100)), (0, 0, (61, 47))])
def test_turn_draft_resize_match_oracle(eng, rotate, draft, size):
    w, h = 203, 131
    rng = np.random.default_rng(rotate * 10 + draft)
    f = rng.integers(0, 65536, (h, w, 3), dtype=np.uint16)
    assert_same(O.prep_rgb16(f, rotate=rotate, draft=draft, size=size), eng.prep_frame(f, L.FramePrep(rotate=rotate, draft=draft), size),
                f"rotate {rotate} draft {draft} size {size}")


def test_prepared_stack_matches_oracle():
    """Frames as decoded (sensor orientation, full size, dusty) pushed into a stack that takes the dust out,
    turns them a quarter and halves them on the device; one frame comes at another size and is brought to
    the stack's. The oracle prepares the same frames on the host and runs the same aligned stack."""
    n, w, h = 5, 480, 320
    raw = L.synth_stack(L.SynthSpec(w, h, n, warp=True, mag_step=0.0, noise_std=0.002, seed=0x9A))[0]
    bowls = [(120.0, 90.0, 10.0, 0.35), (350.0, 250.0, 16.0, 0.2)]
    shade = dust_frame(w, h, bowls) / dust_frame(w, h, [])
    frames = [np.clip(f.astype(np.float32) * np.transpose(shade, (1, 2, 0)) + np.float32(0.5), 0, 65535).astype(np.uint16) for f in raw]
    frames[3] = O.prep_rgb16(frames[3], size=(500, 300))  # a frame of another size slips in
    mo, ml = both_maps(lambda M: spot_map(M, w, h, bowls))
    sw, sh = 160, 240  # turned a quarter, halved
    prepped = np.stack([O.prep_rgb16(f, dust=mo, rotate=1, draft=1, size=(sw, sh)) for f in frames])
    fuse, al = L.FuseParams(), L.AlignParams(coarsen=1)
    ref = O.run_stack(prepped, O.StackParams(fuse=O.FuseParams(), align=O.AlignParams(coarsen=1), depth=None))
    eng = L.Engine()
    st = eng.stack(sw, sh, n, fuse, al, None)
    try:
        st.set_prep(L.FramePrep(dust=ml, rotate=1, draft=1))
        for f in frames:
            st.push_u16(f)
        out = st.finish()
        # the frames the device prepared are the oracle's
        dev = _device_frames(st.frames_device(), (n, sh, sw, 3))
        assert_same(prepped, dev, "prepared frames")
        assert np.max(np.abs(out.align - ref.sims)) < 1e-9
        assert_same(ref.gains, out.gains, "gains")
        assert_same(ref.image_u16, out.image_u16, "fused u16")
    finally:
        st.close()
        eng.close()


def _device_frames(ptr, shape):
    """The stack's frame store (u16, device) read back through torch's CUDA array interface."""
    import torch

    class _Cuda:
        def __init__(self):
            self.__cuda_array_interface__ = {"data": (ptr, False), "shape": shape, "typestr": "<i2", "version": 3}
    torch.cuda.synchronize()
    return torch.as_tensor(_Cuda(), device="cuda").cpu().numpy().view(np.uint16)
