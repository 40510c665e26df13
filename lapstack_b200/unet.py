"""The learned warm start of the WLS depth solve (no counterpart in the reference).

`UNet` wraps the library's network (lapstack_b200/csrc/lsb_unet.cu): a
4-level U-Net, 32 base channels, BF16 weights and activations with FP32
accumulation, trained by the library's own forward, backward and Adam
kernels. Its prediction is the x0 of MG-PCG (`Stack.set_warm_start`), which
then runs to the same relative residual as the plain solve.

Training data comes from the plain method itself: seeded synthetic stacks
go through the whole pipeline, and each stack's depth-grid planes (guide,
raw depth, confidence) and its WLS solution become one (input, target)
pair on the network's quarter-resolution grid.

torch is used only for device buffers and streams here.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from ._lib import check, load
from .engine import DepthParams, Engine, FuseParams, SynthSpec, default_engine, synth_stack_device

CH = 32  # channels of the network's input tensor (3 live)
# the 15 convolutions as lsb_unet.cu runs them: (input channels, output channels, level)
CONVS = [(32, 32, 0), (32, 32, 0), (32, 64, 1), (64, 64, 1), (64, 128, 2), (128, 128, 2), (128, 256, 3), (256, 256, 3),
         (384, 128, 2), (128, 128, 2), (192, 64, 1), (64, 64, 1), (96, 32, 0), (32, 32, 0), (32, 32, 0)]


def forward_flops(H, W, B=1):
    """Tensor-core FLOPs of one forward pass on a B x H x W grid (as executed: padded channels included)."""
    return 2 * sum(9 * ci * co * B * (H >> lv) * (W >> lv) for ci, co, lv in CONVS)


def grid_of(dw, dh):
    """The network grid of a dw x dh depth grid."""
    H, W = C.c_uint32(), C.c_uint32()
    load().lsb_unet_grid(dw, dh, C.byref(H), C.byref(W))
    return H.value, W.value


class UNet:
    def __init__(self, device: int = 0, seed: int = 0):
        self._L = load()
        h = C.c_void_p()
        check(self._L.lsb_unet_create(device, seed, C.byref(h)))
        self._h = h
        nw, nb = C.c_uint64(), C.c_uint64()
        self._L.lsb_unet_sizes(self._h, C.byref(nw), C.byref(nb))
        self.n_weights, self.n_biases = nw.value, nb.value

    def close(self):
        if getattr(self, "_h", None):
            self._L.lsb_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------- parameters
    def params(self):
        w = np.zeros(self.n_weights, np.float32)
        b = np.zeros(self.n_biases, np.float32)
        check(self._L.lsb_unet_get_params(self._h, C.c_void_p(w.ctypes.data), C.c_void_p(b.ctypes.data), None, None))
        return w, b

    def grads(self):
        gw = np.zeros(self.n_weights, np.float32)
        gb = np.zeros(self.n_biases, np.float32)
        check(self._L.lsb_unet_get_params(self._h, None, None, C.c_void_p(gw.ctypes.data), C.c_void_p(gb.ctypes.data)))
        return gw, gb

    def set_params(self, w, b):
        w = np.ascontiguousarray(w, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        assert w.size == self.n_weights and b.size == self.n_biases
        check(self._L.lsb_unet_set_params(self._h, C.c_void_p(w.ctypes.data), C.c_void_p(b.ctypes.data)))

    def set_conv(self, path: str = "tcgen05"):
        """The 3x3 convolutions' tensor-core path: "tcgen05" (the default; TMEM accumulators) or
        "mma.sync" (the same products summed in another order, for comparison)."""
        check(self._L.lsb_unet_set_conv(self._h, {"tcgen05": 0, "mma.sync": 1}[path]))

    def save(self, path):
        w, b = self.params()
        np.savez(path, w=w, b=b)

    def load(self, path):
        z = np.load(path)
        self.set_params(z["w"], z["b"])

    # ---------------------------------------------------------- compute
    def forward(self, inp, d_in):
        """inp: CUDA bf16 [B][H][W][32]; d_in: CUDA f32 [B][H][W]. Returns out0 (f32 [B][H][W])."""
        import torch
        torch.cuda.current_stream().synchronize()  # the network runs on its own stream
        B, H, W = d_in.shape
        out = torch.empty((B, H, W), dtype=torch.float32, device=d_in.device)
        check(self._L.lsb_unet_forward(self._h, C.c_void_p(inp.data_ptr()), C.c_void_p(d_in.data_ptr()), B, H, W,
                                       C.c_void_p(out.data_ptr())))
        return out

    def forward_ms(self):
        """The last forward pass's device time (CUDA events around its layers)."""
        ms = C.c_float()
        check(self._L.lsb_unet_forward_ms(self._h, C.byref(ms)))
        return ms.value

    def train_step(self, inp, d_in, target, lr):
        """One step on a batch; lr = 0 computes the gradients only. Returns the batch MSE."""
        import torch
        torch.cuda.current_stream().synchronize()  # the network runs on its own stream
        B, H, W = d_in.shape
        loss = C.c_double()
        check(self._L.lsb_unet_train_step(self._h, C.c_void_p(inp.data_ptr()), C.c_void_p(d_in.data_ptr()),
                                          C.c_void_p(target.data_ptr()), B, H, W, float(lr), C.byref(loss)))
        return loss.value


def prepare(guide_ptr, d_ptr, conf_ptr, dw, dh, dmax, inp, d_in, b, stream=None):
    """Depth-grid device planes -> batch entry b of the network input (inp, d_in)."""
    check(load().lsb_unet_prepare(C.c_void_p(guide_ptr), C.c_void_p(d_ptr), C.c_void_p(conf_ptr), dw, dh, float(dmax),
                                  C.c_void_p(inp.data_ptr()), C.c_void_p(d_in.data_ptr()), b, C.c_void_p(stream)))


# ------------------------------------------------------------------- data
def solver_pairs(n_stacks, w, h, frames=(8, 16), seed=0x1A957ACC, engine: Engine | None = None, depth: DepthParams | None = None):
    """(input, d_in, target) on the network grid for n seeded synthetic stacks
    solved by the plain method, as CUDA tensors [n][H][W][32] bf16, [n][H][W],
    [n][H][W]; plus the per-stack (dmax, dw, dh)."""
    import torch
    eng = engine or default_engine()
    dp = depth or DepthParams()
    rng = np.random.default_rng(seed)
    items = []
    for s in range(n_stacks):
        n = int(rng.integers(frames[0], frames[1] + 1))
        st = eng.stack(w, h, n, FuseParams(), None, dp)
        synth_stack_device(SynthSpec(w, h, n, seed=seed ^ s, mag_step=0.002, noise_std=0.003), st.frames_device(), eng.stream)
        st.set_count(n)
        st.run()
        (g, d, cf, u), (dw, dh) = st.depth_planes()
        H, W = grid_of(dw, dh)
        inp = torch.empty((1, H, W, CH), dtype=torch.bfloat16, device="cuda")
        d_in = torch.empty((1, H, W), dtype=torch.float32, device="cuda")
        tgt_in = torch.empty_like(inp)
        tgt = torch.empty_like(d_in)
        prepare(g, d, cf, dw, dh, n - 1, inp, d_in, 0, eng.stream)
        prepare(g, u, cf, dw, dh, n - 1, tgt_in, tgt, 0, eng.stream)
        torch.cuda.synchronize()
        items.append((inp, d_in, tgt, n - 1, dw, dh))
        st.close()
    inp = torch.cat([i[0] for i in items])
    d_in = torch.cat([i[1] for i in items])
    tgt = torch.cat([i[2] for i in items])
    return inp, d_in, tgt, [(i[3], i[4], i[5]) for i in items]


def train(net: UNet, inp, d_in, tgt, steps=300, batch=8, crop=128, lr=1e-3, seed=1, log=None):
    """Adam on random crops of the solver pairs; returns the loss per step."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    n, H, W = d_in.shape
    ch, cw = min(crop, H), min(crop, W)
    ch, cw = ch - ch % 8, cw - cw % 8
    losses = []
    t0 = time.perf_counter()
    for it in range(steps):
        k = torch.randint(0, n, (batch,), generator=g)
        y0 = torch.randint(0, H - ch + 1, (batch,), generator=g)
        x0 = torch.randint(0, W - cw + 1, (batch,), generator=g)
        bi = torch.stack([inp[k[j], y0[j]:y0[j] + ch, x0[j]:x0[j] + cw] for j in range(batch)]).contiguous()
        bd = torch.stack([d_in[k[j], y0[j]:y0[j] + ch, x0[j]:x0[j] + cw] for j in range(batch)]).contiguous()
        bt = torch.stack([tgt[k[j], y0[j]:y0[j] + ch, x0[j]:x0[j] + cw] for j in range(batch)]).contiguous()
        # cosine decay
        lr_t = lr * 0.5 * (1 + math.cos(math.pi * it / max(steps, 1)))
        losses.append(net.train_step(bi, bd, bt, lr_t))
        if log and (it % 50 == 0 or it == steps - 1):
            log(f"step {it} loss {losses[-1]:.3e} ({time.perf_counter() - t0:.1f} s)")
    return losses


def compare_warm_start(net: UNet, w, h, n, seeds, engine: Engine | None = None, depth: DepthParams | None = None, repeats=2):
    """Plain (the reference's FGS start) against learned (the network's x0)
    WLS solves on seeded stacks: per seed, per mode, the iterations of both
    solves, the solve time (device ms, warm start included), the final
    relative residual and the depth map."""
    eng = engine or default_engine()
    dp = depth or DepthParams()
    out = []
    for seed in seeds:
        st = eng.stack(w, h, n, FuseParams(), None, dp)
        synth_stack_device(SynthSpec(w, h, n, seed=seed, mag_step=0.002, noise_std=0.003), st.frames_device(), eng.stream)
        st.set_count(n)
        row = {}
        for mode in ("plain", "learned") * repeats:
            st.set_warm_start(net if mode == "learned" else None)
            o = st.finish()
            row[mode] = dict(iters_first=o.depth.wls_iters_first, iters=o.depth.wls_iters, ms=o.ms["wls_solve"],
                             rel=o.depth.wls_rel64, depth=o.depth.depth)
        st.close()
        out.append(row)
    return out
