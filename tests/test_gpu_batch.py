"""Several stacks at once through lsb_batch_run: stacks of uneven sizes and frame
counts, some registered and some not, on two engines that each take half the
SMs (lsb_config.grid_limit), run side by side. Each stack's output equals, bit
for bit, the same stack run alone on an engine with the same grid limit (the
grid limit bounds the registration search's CTAs, whose partial sums it
orders), and an aligned stack of the batch agrees with the oracle as the
single-stack tests ask (transforms within 1e-9, gains and the fused u16 image
exact)."""
import numpy as np
import pytest

import lapstack_b200 as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = [  # w, h, frames, aligned
    (320, 240, 5, True),
    (400, 300, 4, True),
    (256, 192, 6, False),
    (360, 272, 3, True),
    (288, 208, 7, False),
]


def frames_of(w, h, n, aligned, seed):
    return L.synth_stack(L.SynthSpec(w, h, n, warp=aligned, mag_step=0.0 if aligned else 0.002, noise_std=0.002, seed=seed))[0]


def make(eng, w, h, n, aligned, frames):
    st = eng.stack(w, h, n, L.FuseParams(), L.AlignParams(coarsen=1) if aligned else None, L.DepthParams())
    for f in frames:
        st.push_u16(f)
    return st


def assert_same(a, b, what):
    bad = np.count_nonzero(a != b)
    assert bad == 0, f"{what}: {bad} of {a.size} differ"


def test_two_engines_side_by_side_match_single_runs_and_the_oracle():
    import torch
    half = torch.cuda.get_device_properties(0).multi_processor_count
    frames = [frames_of(w, h, n, al, 0xB0 + i) for i, (w, h, n, al) in enumerate(CASES)]
    alone = L.Engine(grid_limit=half)
    singles = []
    for (w, h, n, al), fr in zip(CASES, frames):
        st = make(alone, w, h, n, al, fr)
        singles.append(st.finish())
        st.close()
    alone.close()
    engines = [L.Engine(grid_limit=half), L.Engine(grid_limit=half)]
    stacks = [make(engines[i % 2], w, h, n, al, fr) for i, ((w, h, n, al), fr) in enumerate(zip(CASES, frames))]
    try:
        outs = L.batch_run(stacks)
        for i, (o, s) in enumerate(zip(outs, singles)):
            assert_same(s.image_u16, o.image_u16, f"stack {i}: fused u16")
            assert_same(s.winner, o.winner, f"stack {i}: winner map")
            assert_same(s.align, o.align, f"stack {i}: transforms")
            assert_same(s.gains, o.gains, f"stack {i}: gains")
            assert_same(s.depth.depth, o.depth.depth, f"stack {i}: depth")
            assert_same(s.depth.conf, o.depth.conf, f"stack {i}: confidence")
        w, h, n, _ = CASES[0]
        ref = O.run_stack(np.stack(frames[0]), O.StackParams(fuse=O.FuseParams(), align=O.AlignParams(coarsen=1), depth=None))
        assert np.max(np.abs(outs[0].align - ref.sims)) < 1e-9
        assert_same(ref.gains, outs[0].gains, "gains vs the oracle")
        assert_same(ref.image_u16, outs[0].image_u16, "fused u16 vs the oracle")
    finally:
        for st in stacks:
            st.close()
        for e in engines:
            e.close()


def test_stacks_of_two_engines_must_share_the_focus_measure():
    e1, e2 = L.Engine(), L.Engine()
    a = e1.stack(64, 48, 2, L.FuseParams(), None, L.DepthParams(r_in=1))
    b = e2.stack(64, 48, 2, L.FuseParams(), None, L.DepthParams(r_in=2))
    try:
        fr = frames_of(64, 48, 2, False, 7)
        for st in (a, b):
            for f in fr:
                st.push_u16(f)
        with pytest.raises(RuntimeError, match="focus measure"):
            L.batch_run([a, b])
    finally:
        a.close()
        b.close()
        e1.close()
        e2.close()
