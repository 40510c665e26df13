"""The oracle's host twin of the seeded generator, and its one-frame-at-a-time
stack (CPU; the checks the CPU baseline relies on).

- The twin makes the engine's host generator's frames byte for byte, so that
  the CPU baseline gets the benchmark's inputs without the CUDA library.
- StackRun (push per frame, then finish) gives run_stack's result exactly.
"""
import numpy as np
import pytest

import lapstack_b200 as L
from oracle import oracle as O


@pytest.mark.parametrize("kw", [dict(w=97, h=61, n=3, warp=True, mag_step=0.0, seed=5),
                                dict(w=128, h=96, n=4, mag_step=0.002, noise_std=0.003, seed=0x1A957ACC),
                                dict(w=64, h=40, n=2, blur_px=2.0, warp=True, warp_shift=3.0, seed=(1 << 40) + 7)])
def test_twin_generator_matches_the_engine_host_generator(kw):
    lib_frames, lib_truth = L.synth_stack(L.SynthSpec(**kw))
    orc_frames, orc_truth = O.synth_stack(**kw)
    assert np.array_equal(lib_frames, orc_frames)
    assert np.array_equal(lib_truth, orc_truth)
    # a subset of the stack's frames is those frames
    sub, _ = O.synth_stack(**kw, frames=(1, kw["n"] - 1))
    assert np.array_equal(sub, orc_frames[1:])


@pytest.mark.parametrize("align,depth", [(True, True), (False, True), (True, False)])
def test_stack_run_by_frames_matches_run_stack(align, depth):
    fr, _ = O.synth_stack(160, 120, 4, warp=align, mag_step=0.0 if align else 0.002, seed=11)
    sp = O.StackParams(align=O.AlignParams(coarsen=1) if align else None, depth=O.DepthParams() if depth else None)
    whole = O.run_stack(fr, sp)
    run = O.StackRun(len(fr), 160, 120, sp)
    for f in fr:
        run.push(f)
    part = run.finish()
    assert np.array_equal(whole.image_u16, part.image_u16)
    assert np.array_equal(whole.sims, part.sims) and np.array_equal(whole.gains, part.gains)
    assert np.array_equal(whole.shares, part.shares)
    if depth:
        assert np.array_equal(whole.depth, part.depth)


def test_cycled_slices_run_the_depth_pass_over_a_whole_stack():
    """cycle_slices (a timing aid) makes the depth pass see n_total slices: the peaks of the last
    pushed frame then have a neighbour after them, so the depth map changes."""
    fr, _ = O.synth_stack(96, 64, 3, seed=13)
    outs = []
    for total in (3, 9):
        run = O.StackRun(3, 96, 64, O.StackParams(align=None))
        for f in fr:
            run.push(f)
        run.cycle_slices(total)
        outs.append(run.finish())
    assert np.array_equal(outs[0].image_u16, outs[1].image_u16)
    assert not np.array_equal(outs[0].depth, outs[1].depth)


def test_thread_count_is_set():
    try:
        assert O.set_threads(1) == 1
    finally:
        O.set_threads(0)
