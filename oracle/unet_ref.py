"""CPU oracle of the learned warm start's network (test infrastructure only).

The network has no counterpart in the reference; this file restates the
library's U-Net (lapstack_b200/csrc/lsb_unet.cu) in numpy so its forward and
backward kernels can be checked: the same 15 layers, the same tensor layout
(NHWC, weights [tap][cout][cin]), and bf16 rounding (round to nearest even)
at the same points as the kernels: the bf16 copy of the weights, every
stored activation, the 2x2 pooled input of an encoder layer, and the dZ
operand of the backward convolutions. Sums are f64. With bf16_round=False every
rounding is skipped, which the finite-difference test of the backward pass
uses.
"""
from __future__ import annotations

import numpy as np

SAME, UP, POOL = 0, 1, 2
# (src1, mode1, c1, src2, mode2, c2, cout, level, relu) -- tensor 0 is the input, i + 1 the output of layer i
LAYERS = [
    (0, SAME, 32, -1, 0, 0, 32, 0, 1),
    (1, SAME, 32, -1, 0, 0, 32, 0, 1),
    (2, POOL, 32, -1, 0, 0, 64, 1, 1),
    (3, SAME, 64, -1, 0, 0, 64, 1, 1),
    (4, POOL, 64, -1, 0, 0, 128, 2, 1),
    (5, SAME, 128, -1, 0, 0, 128, 2, 1),
    (6, POOL, 128, -1, 0, 0, 256, 3, 1),
    (7, SAME, 256, -1, 0, 0, 256, 3, 1),
    (8, UP, 256, 6, SAME, 128, 128, 2, 1),
    (9, SAME, 128, -1, 0, 0, 128, 2, 1),
    (10, UP, 128, 4, SAME, 64, 64, 1, 1),
    (11, SAME, 64, -1, 0, 0, 64, 1, 1),
    (12, UP, 64, 2, SAME, 32, 32, 0, 1),
    (13, SAME, 32, -1, 0, 0, 32, 0, 1),
    (14, SAME, 32, -1, 0, 0, 32, 0, 0),
]


def offsets():
    wo, bo, out = 0, 0, []
    for (_, _, c1, _, _, c2, co, _, _) in LAYERS:
        out.append((wo, bo))
        wo += 9 * co * (c1 + c2)
        bo += co
    return out, wo, bo


def bf16(x):
    """Round to bfloat16 (nearest even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def _src(act, t, mode, rnd, ft):
    x = act[t]
    if mode == SAME:
        return x
    if mode == UP:
        return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)
    b, h, w, c = x.shape
    q = x.reshape(b, h // 2, 2, w // 2, 2, c).astype(ft)
    p = (((q[:, :, 0, :, 0] + q[:, :, 0, :, 1]) + q[:, :, 1, :, 0]) + q[:, :, 1, :, 1]) * ft(0.25)
    return rnd(p)


def _conv(x, w, bias=None):
    """x [B][H][W][Ci] (f64), w [9][Co][Ci] -> [B][H][W][Co] f64, zero padding 1."""
    b, h, wd, ci = x.shape
    xp = np.zeros((b, h + 2, wd + 2, ci))
    xp[:, 1:-1, 1:-1] = x
    out = np.zeros((b, h, wd, w.shape[1]))
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        out += xp[:, ky:ky + h, kx:kx + wd] @ w[tap].T
    if bias is not None:
        out += bias
    return out


def _layer_input(act, L, rnd, ft):
    s1, m1, c1, s2, m2, c2 = L[:6]
    x = _src(act, s1, m1, rnd, ft)[..., :c1]
    if s2 >= 0:
        x = np.concatenate([x, _src(act, s2, m2, rnd, ft)[..., :c2]], axis=-1)
    return x.astype(np.float64)


def _modes(bf16_round):
    """(rounding of stored tensors, storage float type): bf16 over f32, or exact f64."""
    if bf16_round:
        return bf16, np.float32
    return (lambda a: np.asarray(a, np.float64)), np.float64


def forward(inp, w, b, bf16_round=True):
    """inp [B][H][W][32]; w, b the flat master arrays. Returns (activations, out0 [B][H][W])."""
    rnd, ft = _modes(bf16_round)
    offs, _, _ = offsets()
    act = [rnd(inp)]
    out0 = None
    for i, L in enumerate(LAYERS):
        s1, m1, c1, s2, m2, c2, co, lv, relu = L
        ci = c1 + c2
        wo, bo = offs[i]
        wl = rnd(w[wo:wo + 9 * co * ci].reshape(9, co, ci)).astype(np.float64)
        z = _conv(_layer_input(act, L, rnd, ft), wl, b[bo:bo + co].astype(np.float64))
        if relu:
            z = np.maximum(z, 0.0)
        if i == len(LAYERS) - 1:
            out0 = z[..., 0].astype(ft)
        act.append(rnd(z.astype(ft)))
    return act, out0


def backward(act, out0, d_in, target, w, bf16_round=True):
    """MSE of d_in + out0 against target; returns (loss, gw, gb) as the kernels compute them."""
    rnd, ft = _modes(bf16_round)
    offs, nw, nb = offsets()
    gw, gb = np.zeros(nw), np.zeros(nb)
    n = out0.size
    e = (d_in.astype(np.float64) + out0) - target
    loss = float(np.mean(e * e))
    grad = [np.zeros(a.shape) for a in act]
    grad[-1][..., 0] = (2.0 * e / n).astype(ft)
    for i in range(len(LAYERS) - 1, -1, -1):
        s1, m1, c1, s2, m2, c2, co, lv, relu = LAYERS[i]
        ci = c1 + c2
        wo, bo = offs[i]
        g = grad[i + 1]
        if relu:
            g = np.where(act[i + 1] > 0, g, 0.0)
        if i == len(LAYERS) - 1:
            g = np.where(np.arange(co) == 0, g, 0.0)
        dz = rnd(g.astype(ft)).astype(np.float64)
        x = _layer_input(act, LAYERS[i], rnd, ft)
        bsz, h, wd, _ = x.shape
        xp = np.zeros((bsz, h + 2, wd + 2, ci))
        xp[:, 1:-1, 1:-1] = x
        dw = np.zeros((9, co, ci))
        for tap in range(9):
            ky, kx = divmod(tap, 3)
            dw[tap] = np.einsum("bhwo,bhwi->oi", dz, xp[:, ky:ky + h, kx:kx + wd])
        gw[wo:wo + 9 * co * ci] = dw.ravel()
        gb[bo:bo + co] = dz.sum(axis=(0, 1, 2))
        if i == 0:
            continue
        wl = rnd(w[wo:wo + 9 * co * ci].reshape(9, co, ci)).astype(np.float64)
        wt = wl[::-1].transpose(0, 2, 1)  # wt[8 - tap][ci][co]
        dx = _conv(dz, wt).astype(ft).astype(np.float64)
        for (src, mode, c0, cn) in ((s1, m1, 0, c1), (s2, m2, c1, c2)):
            if src < 0:
                continue
            part = dx[..., c0:c0 + cn]
            if mode == SAME:
                grad[src][..., :cn] += part
            elif mode == UP:
                bb, hh, ww, cc = part.shape
                grad[src][..., :cn] += part.reshape(bb, hh // 2, 2, ww // 2, 2, cc).sum(axis=(2, 4))
            else:
                grad[src][..., :cn] += 0.25 * np.repeat(np.repeat(part, 2, axis=1), 2, axis=2)
    return loss, gw, gb


def init_params(seed=0):
    """Small random parameters with the library's live/dead pattern (tests only)."""
    rng = np.random.default_rng(seed)
    offs, nw, nb = offsets()
    w, b = np.zeros(nw, np.float32), np.zeros(nb, np.float32)
    for i, (s1, m1, c1, s2, m2, c2, co, lv, relu) in enumerate(LAYERS):
        ci = c1 + c2
        wo, bo = offs[i]
        wl = rng.standard_normal((9, co, ci)).astype(np.float32) * np.float32(np.sqrt(2.0 / (9 * ci)))
        if i == 0:
            wl[..., 3:] = 0
        if i == len(LAYERS) - 1:
            wl[:, 1:] = 0
        w[wo:wo + 9 * co * ci] = wl.ravel()
        b[bo:bo + co] = rng.standard_normal(co).astype(np.float32) * np.float32(0.05)
        if i == len(LAYERS) - 1:
            b[bo + 1:bo + co] = 0
    return w, b
