"""The oracle's weighted average (wav.rs:92), pinned by the reference's own
unit tests (wav.rs:169-266), restated here on the CPU:

- takes_the_sharper_frame: two frames, each sharp on one half; the average
  keeps each half's sharp checkerboard;
- noise_floor_keeps_the_sharp_frame: twelve noisy frames, a faint texture
  sharp in one; with the depth pass's noise floor the texture survives and a
  flat area's noise drops, without it the texture drowns.
"""
import numpy as np

from oracle import oracle as O
from tests.fixtures import lcg_plane


def test_takes_the_sharper_frame():
    w, h = 64, 64
    y, x = np.mgrid[0:h, 0:w]
    fine = np.where(((x // 2) + (y // 2)) % 2 == 0, np.float32(0.8), np.float32(0.2)).astype(np.float32)
    va = np.where(x < 32, fine, np.float32(0.5)).astype(np.float32)
    vb = np.where(x < 32, np.float32(0.5), fine).astype(np.float32)
    a, b = np.stack([va] * 3), np.stack([vb] * 3)
    dp = O.DepthParams(scale=1)
    out = O.weighted_average(np.stack([a, b]), dp, O.WavParams(power=2.0, smooth=0, gate=0.5, edge=False))
    i, j = (16, 8), (16, 56)
    assert abs(out[0][i] - a[0][i]) < 0.05
    assert abs(out[0][j] - b[0][j]) < 0.05


def test_noise_floor_keeps_the_sharp_frame():
    w, h, n = 96, 64, 12
    # the reference draws every frame's three planes from one LCG stream, frame by frame
    vals = lcg_plane(n * 3 * w * h, 7).reshape(n, 3, h, w)
    frames = (np.float32(0.5) + np.float32(0.06) * (vals - np.float32(0.5))).astype(np.float32)
    y, x = np.mgrid[0:h, 0:w // 2]
    t = np.where(((x // 2) + (y // 2)) % 2 == 0, np.float32(0.05), np.float32(-0.05)).astype(np.float32)
    for c in range(3):
        frames[5, c, :, :w // 2] += t
    dp = O.DepthParams(scale=1)
    fused = frames[5].copy()
    slices = np.stack([O.focus_slice(f, dp) for f in frames])
    _, _, floor, _ = O.depth_from_slices(slices, fused, dp)
    wp = O.WavParams(power=2.0, smooth=2, gate=0.5, edge=True)
    out = O.weighted_average(frames, dp, wp, floor=floor, guide=fused)

    def corr(img):
        yy, xx = np.mgrid[8:h - 8, 8:w // 2 - 8]
        tt = np.where(((xx // 2) + (yy // 2)) % 2 == 0, 1.0, -1.0)
        return float(np.mean(tt * (img[0][8:h - 8, 8:w // 2 - 8] - 0.5)))

    assert corr(out) / corr(frames[5]) > 0.8
    sd = lambda img: float(np.std(img[0][8:h - 8, w // 2 + 8:w - 8]))
    assert sd(out) / sd(frames[0]) < 0.5
    plain = O.weighted_average(frames, dp, wp, floor=np.zeros_like(floor), guide=fused)
    assert corr(plain) / corr(frames[5]) < 0.5


def test_stack_weighted_average_is_the_direct_one():
    """run_stack's weighted average (stack.rs:857) is wav.rs:92 over the frames as folded, with the
    depth pass's floor cells and the fused image as guide."""
    fr, _ = O.synth_stack(160, 120, 5, seed=3)
    sp = O.StackParams(align=None, depth=O.DepthParams(), wav=O.WavParams())
    res = O.run_stack(fr, sp)
    planes = np.stack([np.transpose(f, (2, 0, 1)).astype(np.float32) * (np.float32(1) / np.float32(65535)) for f in fr])
    g = res.gains.astype(np.float32)
    for k in range(1, len(fr)):  # the no-align path's gains (stack.rs LazyFrames), as applied
        for c in range(3):
            if abs(g[k, c] - 1.0) > 0:
                planes[k, c] = planes[k, c] * g[k, c]
    direct = O.weighted_average(planes, O.DepthParams(), O.WavParams(), floor=res.floor_cells, guide=res.image.astype(np.float32))
    assert res.wav is not None
    assert np.array_equal(res.wav.astype(np.float32), direct)
