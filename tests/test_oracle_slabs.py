"""The slabs (stack.rs:76 slab_ranges, stack.rs:740 fuse_range, stack.rs:872
fuse_slabs) and the resize of prep.rs:46/63, on the CPU.

- slab_ranges, in the oracle and through the C ABI (a host-only entry point),
  against the known answers and properties of stack.rs:1126-1141.
- the oracle's resize against prep.rs:153-166 (a constant stays constant and
  lands on the size asked; a ramp resampled onto its own line keeps its
  centre), and equal sizes copy.
- the oracle's slabs: a slab that spans the stack is the stack's own fused
  image, bit for bit; without brightness gains each slab is the stack of its
  frames alone; a one-frame slab returns that frame up to the pyramid's
  round-off.
"""
import numpy as np
import pytest

from oracle import oracle as O

# stack.rs:1127-1132
KNOWN = [((8, 3, 1), [(0, 2), (2, 4), (4, 6), (6, 7)]),
         ((20, 10, 2), [(0, 9), (8, 17), (16, 19)]),
         ((8, 8, 0), [(0, 7)]),
         ((8, 20, 5), [(0, 7)]),
         ((5, 2, 7), [(0, 1), (1, 2), (2, 3), (3, 4)]),
         ((0, 3, 1), [])]


def check_cover(r, count):
    """stack.rs:1133-1140: starts at 0, ends at the last frame, advances and leaves no gap."""
    assert r[0][0] == 0 and r[-1][1] == count - 1
    for a, b in zip(r, r[1:]):
        assert a[0] < b[0] <= a[1] + 1, r


@pytest.mark.parametrize("args,want", KNOWN)
def test_oracle_slab_ranges_known_answers(args, want):
    assert O.slab_ranges(*args) == want


def test_oracle_slab_ranges_cover():
    for count, size, overlap in [(100, 10, 2), (7, 3, 2), (9, 4, 0), (1, 5, 3)]:
        check_cover(O.slab_ranges(count, size, overlap), count)


def test_abi_slab_ranges_match_oracle():
    """lsb_slab_ranges needs no device: the reference's cases and a sweep, against the oracle."""
    import lapstack_b200 as L
    for args, want in KNOWN:
        assert L.slab_ranges(*args) == want
    for count in range(0, 30):
        for size in range(0, 12):
            for overlap in range(0, 12):
                got = L.slab_ranges(count, size, overlap)
                assert got == O.slab_ranges(count, size, overlap), (count, size, overlap)
                if count:
                    check_cover(got, count)


def test_oracle_resize_keeps_a_constant_and_a_ramp():
    """prep.rs:153-166."""
    im = np.stack([np.full((5, 7), 0.25 * (c + 1), np.float32) for c in range(3)])
    out = O.resize(im, 13, 9, interp=3)
    assert out.shape == (3, 9, 13)
    for c in range(3):
        assert np.all(np.abs(out[c] - 0.25 * (c + 1)) < 1e-5)
    ramp = np.zeros((3, 21), np.float32)
    ramp[:] = np.arange(21, dtype=np.float32) / 20.0
    r = O.resize(ramp, 41, 3, interp=1)
    assert abs(r[0, 20] - 0.5) < 1e-3, r[0, 20]
    assert r[0, 0] < 0.05 and r[0, 40] > 0.95
    a = np.random.default_rng(3).random((2, 11, 17), dtype=np.float32)
    assert np.array_equal(O.resize(a, 17, 11), a)


def small_stack(n=5, w=96, h=64, seed=5):
    return O.synth_stack(w, h, n, seed=seed)[0]


@pytest.mark.parametrize("storage", ["f32", "unorm16"])
def test_oracle_whole_stack_slab_is_the_result(storage):
    fr = small_stack()
    sp = O.StackParams(align=None, depth=None, slabs=(fr.shape[0], 0), storage=storage)
    r = O.run_stack(fr, sp)
    assert r.slab_ranges == [(0, fr.shape[0] - 1)]
    assert np.array_equal(r.slabs[0], r.image)


def test_oracle_slabs_follow_the_ranges():
    """Without the brightness gains (each slab would otherwise keep the whole stack's frame-0 reference),
    every slab is the fused image of a stack of its frames alone, bit for bit."""
    fr = small_stack(n=7)
    sp = O.StackParams(align=None, depth=None, brightness=False, slabs=(3, 1))
    r = O.run_stack(fr, sp)
    assert r.slab_ranges == O.slab_ranges(7, 3, 1)
    for (lo, hi), img in zip(r.slab_ranges, r.slabs):
        alone = O.run_stack(fr[lo:hi + 1], O.StackParams(align=None, depth=None, brightness=False))
        assert np.array_equal(img, alone.image), (lo, hi)
    # with the gains, the first slab shares frame 0 as its reference: the same again
    r = O.run_stack(fr, O.StackParams(align=None, depth=None, slabs=(3, 1)))
    assert np.array_equal(r.slabs[0], O.run_stack(fr[:3], O.StackParams(align=None, depth=None)).image)


def test_oracle_one_frame_slab_is_the_frame():
    fr = small_stack(n=3)
    sp = O.StackParams(align=None, depth=None, brightness=False, slabs=(1, 0))
    r = O.run_stack(fr, sp)
    assert len(r.slabs) == 3
    for k in range(3):
        want = np.transpose(fr[k], (2, 0, 1)).astype(np.float64) / 65535.0
        assert np.max(np.abs(r.slabs[k] - want)) < 1e-5
