"""Frames and dust maps for the frame-preparation tests (dust.rs:616-650's
test frames, restated), shared by the CPU and GPU tests."""
import numpy as np


def dust_frame(w, h, spots):
    """dust.rs:620 `dust_frame`: a softly lit white frame (0.9 in the middle, 0.85 in the corners) with soft
    dark bowls at (cx, cy) of radius r and depth d; planar (3, h, w) f32."""
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    u, v = x / np.float32(w) - np.float32(0.5), y / np.float32(h) - np.float32(0.5)
    lum = np.float32(0.9) - np.float32(0.1) * (u * u + v * v)
    for cx, cy, r, depth in spots:
        d = np.sqrt((x - np.float32(cx)) ** 2 + (y - np.float32(cy)) ** 2) / np.float32(r)
        bowl = np.float32(1.0) - np.float32(depth) * (np.float32(1.0) - d * d) ** 2
        lum = np.where(d < 1.0, lum * bowl, lum).astype(np.float32)
    return np.stack([lum * np.float32(k) for k in (1.0, 0.98, 0.95)]).astype(np.float32)


def scene(w, h):
    """dust.rs:640 `scene`: a smooth, slightly textured scene; planar (3, h, w) f32."""
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    r = np.float32(0.3) + np.float32(0.3) * (np.sin(x / np.float32(23.0)) * np.float32(0.5) + np.float32(0.5))
    g = np.float32(0.2) + np.float32(0.4) * (y / np.float32(h))
    b = np.float32(0.5) + np.float32(0.2) * np.cos((x + y) / np.float32(37.0))
    return np.stack([r, g, b]).astype(np.float32)


def dilate(mask, r):
    """A square dilation by r pixels."""
    out = mask.copy()
    h, w = mask.shape
    for dy in range(-r, r + 1):
        for dx in range(-r, r + 1):
            sh = np.zeros_like(mask)
            ys, yd = (slice(max(dy, 0), h), slice(0, h - max(dy, 0))) if dy >= 0 else (slice(0, h + dy), slice(-dy, h))
            xs, xd = (slice(max(dx, 0), w), slice(0, w - max(dx, 0))) if dx >= 0 else (slice(0, w + dx), slice(-dx, w))
            sh[yd, xd] = mask[ys, xs]
            out |= sh
    return out


def spot_map(M, w, h, spots, threshold=0.03, margin=3, mode="fill"):
    """A dust map of the given bowls as dust.rs:315 `detect` would outline them: the pixels darker than
    the clean frame by more than `threshold`, grown by `margin`, one spot per bowl with its window cut to
    the frame, and the attenuation clean / dusty as each spot's gain. M is the module with DustSpot /
    DustMap (the oracle's or the engine's)."""
    shadow, flat = dust_frame(w, h, spots)[1], dust_frame(w, h, [])[1]
    dark = (np.float32(1.0) - shadow / flat) > threshold
    gain = (flat / shadow).astype(np.float32)
    out = []
    for cx, cy, r, _ in spots:
        x0, y0 = max(int(cx - r) - margin - 1, 0), max(int(cy - r) - margin - 1, 0)
        x1, y1 = min(int(cx + r) + margin + 2, w), min(int(cy + r) + margin + 2, h)
        own = np.zeros((h, w), bool)
        yy, xx = np.mgrid[0:h, 0:w]
        own[(xx - cx) ** 2 + (yy - cy) ** 2 < r * r] = True
        m = dilate(dark & own, margin)[y0:y1, x0:x1]
        out.append(M.DustSpot(x0, y0, m.astype(np.uint8), gain[y0:y1, x0:x1].copy()))
    return M.DustMap(w, h, out, mode)


def random_map(M, w, h, n, seed, mode="fill", overlap=True):
    """n seeded random blob spots (some overlapping when asked, some at the frame's edges)."""
    rng = np.random.default_rng(seed)
    spots = []
    for k in range(n):
        sw, sh = int(rng.integers(3, 40)), int(rng.integers(3, 40))
        if k % 5 == 0:  # at an edge
            x, y = (0 if k % 2 == 0 else w - sw), int(rng.integers(0, h - sh))
        else:
            x, y = int(rng.integers(0, w - sw)), int(rng.integers(0, h - sh))
        if overlap and k % 4 == 3 and spots:  # on top of the spot before
            p = spots[-1]
            x, y = min(p.x + 2, w - sw), min(p.y + 2, h - sh)
        m = (rng.random((sh, sw)) < 0.7).astype(np.uint8)
        g = (np.float32(1.0) + rng.random((sh, sw), dtype=np.float32) * np.float32(0.5)).astype(np.float32)
        spots.append(M.DustSpot(x, y, m, g))
    return M.DustMap(w, h, spots, mode)


def u16_of(planes):
    """Planar f32 in [0, 1] to interleaved u16 (io.rs:287's v * 65535 + 0.5)."""
    return (np.transpose(np.clip(planes, 0, 1), (1, 2, 0)) * np.float32(65535.0) + np.float32(0.5)).astype(np.uint16)
