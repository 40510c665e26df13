"""Small synthetic inputs of the kinds the reference's unit tests build
(xorshift / LCG noise, checkerboards, binomial blur, two-frame
sharp-left / sharp-right stacks); see crates/lapstack-core/src/pyramid.rs:235,
fuse.rs:547-569, depth.rs:1206-1209 and 1343-1364."""
import numpy as np


def xorshift_img(w, h, seed):
    """pyramid.rs:235 `noise_img`: three planes of xorshift32 values in [0, 1)."""
    s = np.uint32(seed)
    out = np.empty((3, h, w), np.float32)
    flat = out.reshape(-1)
    with np.errstate(over="ignore"):
        for i in range(flat.size):
            s ^= np.uint32(s << np.uint32(13))
            s ^= np.uint32(s >> np.uint32(17))
            s ^= np.uint32(s << np.uint32(5))
            flat[i] = np.float32(int(s) % 10000) / np.float32(10000.0)
    return out


def lcg_plane(n, seed):
    """depth.rs:1206 `lcg`: values ((s >> 33) % 10000) / 10000."""
    s = seed
    out = np.empty(n, np.float32)
    for i in range(n):
        s = (s * 6364136223846793005 + 1442695040888963407) & ((1 << 64) - 1)
        out[i] = np.float32((s >> 33) % 10000) / np.float32(10000.0)
    return out


def checker(w, h, cell, tint=(1.0, 0.9, 0.5)):
    """fuse.rs:547 `checker` (tint (1, .9, .5)); depth.rs:1343 uses (1, 1, 1)."""
    y, x = np.mgrid[0:h, 0:w]
    v = np.where(((x // cell) + (y // cell)) % 2 == 0, np.float32(0.2), np.float32(0.8)).astype(np.float32)
    return np.stack([v * np.float32(t) for t in tint]).astype(np.float32)


def blur(planes, passes, oracle):
    """fuse.rs:561 `blur`: the 5-tap window `passes` times, no decimation."""
    k = np.array([1, 4, 6, 4, 1], np.float32) / np.float32(16)
    o = planes.copy()
    for _ in range(passes):
        o = np.stack([oracle.window_sum(o[c], k) for c in range(3)])
    return o


def halves(sharp, soft, w):
    """Frame A sharp on the left, blurred on the right; frame B the opposite."""
    a, b = sharp.copy(), sharp.copy()
    a[:, :, w // 2:] = soft[:, :, w // 2:]
    b[:, :, :w // 2] = soft[:, :, :w // 2]
    return a, b


def rms(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)))
