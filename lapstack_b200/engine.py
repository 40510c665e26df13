"""Host-side mirror of lapstack-core's stacking interface over the C ABI.

Names and argument meaning follow the reference (crates/lapstack-core/src):
FuseParams / AlignParams / DepthParams carry its defaults (fuse.rs:94-107,
align.rs:66-70, depth.rs:93-109); `GpuFuser` has the new / push / shares /
finish contract of gpu.rs:326 (and stack.rs:123 AnyFuser); `depth_from_slices`
is gpu.rs:1327; `Stack` runs stack.rs:1011 `run_with` for in-memory 16-bit
frames. Errors are raised as LsbError with the library's message, the way
the reference returns Result<_, String>.

Inputs may be numpy arrays (host memory) or CUDA tensors (device memory).
"""
from __future__ import annotations

import atexit
import ctypes as C
import sys
import weakref
from dataclasses import dataclass, field

import numpy as np

from ._lib import (AlignParamsC, Config, DepthParamsC, DustMapC, DustSpotC, FramePrepC, FuseParamsC, LOG_FN, LsbError, Result,
                   SynthDesc, WavParamsC, check, load)

TOP_RULES = {"de": 0, "dev": 1, "avg": 2}
INTERPS = ["nearest", "bilinear", "bicubic", "spline4x4", "spline6x6", "lanczos3"]
MODELS = ["similarity", "affine", "projective"]
FOCUS = ["rdf", "sml"]
UPSAMPLE = ["bilinear", "guided"]
# the other spellings the reference's parsers accept, by canonical name
TOP_RULE_ALIASES = {"dev-entropy": "de", "deviation": "dev", "average": "avg"}  # fuse.rs:59
MODEL_ALIASES = {"sim": "similarity", "perspective": "projective", "homography": "projective"}  # align.rs:95
INTERP_ALIASES = {"nn": "nearest", "linear": "bilinear", "cubic": "bicubic", "spline16": "spline4x4",
                  "spline36": "spline6x6", "lanczos": "lanczos3"}  # align.rs:148


def _canon(name, names, what, aliases=None, fold=False):
    """The canonical spelling of a named option. The reference's parsers (fuse.rs:59, align.rs:95 and
    :148, which also trim and lower-case, depth.rs:112 and :127) return None for an unknown name: here
    that is an LsbError naming the choices."""
    key = name.strip().lower() if fold and isinstance(name, str) else name
    key = (aliases or {}).get(key, key)
    if key in names:
        return key
    raise LsbError(f"unknown {what} {name!r}: one of {', '.join(names)}")


def _pick(name, names, what, aliases=None, fold=False):
    """The C-ABI code of a named option (its index in `names`, or its value when `names` is a dict)."""
    key = _canon(name, names, what, aliases, fold)
    return names[key] if isinstance(names, dict) else names.index(key)


@dataclass
class FuseParams:  # fuse.rs:70-107
    levels: int = 0
    energy_radius: int = 1
    top_rule: str = "de"
    top_radius: int = 2
    entropy_bins: int = 256
    use_chroma: bool = False
    depth_level: int = 2
    halo: float = 0.0

    def c(self):
        return FuseParamsC(self.levels, self.energy_radius, _pick(self.top_rule, TOP_RULES, "top rule", TOP_RULE_ALIASES),
                           self.top_radius, self.entropy_bins,
                           int(self.use_chroma), self.depth_level, self.halo)


@dataclass
class AlignParams:  # align.rs:52-70
    shift: bool = True
    scale: bool = True
    rotation: bool = True
    model: str = "similarity"
    coarsen: int = 0
    interp: str = "spline4x4"
    host_search: bool = False  # True: the host drives Nelder-Mead, one launch per simplex step

    def c(self, enabled=True):
        return AlignParamsC(int(enabled), int(self.shift), int(self.scale), int(self.rotation),
                            _pick(self.model, MODELS, "alignment model", MODEL_ALIASES, fold=True), self.coarsen,
                            _pick(self.interp, INTERPS, "interpolation", INTERP_ALIASES, fold=True), int(self.host_search))

    def free(self):
        model = _canon(self.model, MODELS, "alignment model", MODEL_ALIASES, fold=True)
        a, p = model != "similarity", model == "projective"
        return [self.shift, self.shift, self.scale, self.rotation, a, a, p, p]


@dataclass
class DepthParams:  # depth.rs:69-109
    scale: int = 1
    focus: str = "rdf"
    r_in: int = 1
    r_out: int = 3
    sml_step: int = 1
    agg_radius: int = 3
    agg_eps: float = 1e-4
    lam: float = 3.0
    sigma_c: float = 0.04
    cg_iters: int = 200
    median: bool = True
    upsample: str = "guided"
    up_radius: int = 2
    up_eps: float = 1e-2
    gate: float = 1.0
    robust: float = 1.0
    edge_mode: int = 0  # 0: exp(-|dI|/sigma_c) as the reference; 1: exp(-dI^2/(2 sigma_c^2))
    vcycle_mode: int = 0  # 0: FP32 V-cycle as the reference; 1: BF16 smoother and restriction

    def c(self, enabled=True):
        return DepthParamsC(int(enabled), self.scale, _pick(self.focus, FOCUS, "focus measure"), self.r_in, self.r_out,
                            self.sml_step, self.agg_radius, self.agg_eps, self.lam, self.sigma_c, self.cg_iters,
                            int(self.median), _pick(self.upsample, UPSAMPLE, "upsampling"), self.up_radius, self.up_eps,
                            self.gate, self.robust, self.edge_mode, self.vcycle_mode)


@dataclass
class WavParams:  # wav.rs:52-80
    power: float = 2.0
    smooth: int = 3
    gate: float = 0.5
    edge: bool = True

    def c(self):
        return WavParamsC(self.power, self.smooth, self.gate, int(self.edge))


@dataclass
class DustSpot:  # dust.rs:85 Spot: its window at (x, y), mask (h, w) nonzero = dust, gain (h, w) for flat mode
    x: int
    y: int
    mask: np.ndarray
    gain: np.ndarray | None = None


DUST_MODES = ("fill", "flat")


@dataclass
class DustMap:  # dust.rs:105 DustMap; mode dust.rs:42 ("fill": pull-push, "flat": times the attenuation)
    w: int
    h: int
    spots: list
    mode: str = "fill"


@dataclass
class FramePrep:  # stack.rs:52-58 Params::dust, rotate, reduce
    dust: DustMap | None = None
    rotate: int = 0
    draft: int = 0

    def c(self):
        """The C struct and the arrays it points into (keep both alive while it is used)."""
        keep = []
        dm = None
        if self.dust is not None:
            d = self.dust
            spots = (DustSpotC * max(len(d.spots), 1))()
            for k, sp in enumerate(d.spots):
                m = np.ascontiguousarray(sp.mask, dtype=np.uint8)
                g = None if sp.gain is None else np.ascontiguousarray(sp.gain, dtype=np.float32)
                keep += [m, g]
                spots[k] = DustSpotC(sp.x, sp.y, m.shape[1], m.shape[0], m.ctypes.data, None if g is None else g.ctypes.data)
            mode = _pick(d.mode, DUST_MODES, "dust mode") if isinstance(d.mode, str) else int(d.mode)
            dm = DustMapC(d.w, d.h, mode, len(d.spots), spots)
            keep += [spots, dm]
        p = FramePrepC(C.pointer(dm) if dm is not None else None, self.rotate, self.draft)
        keep.append(p)
        return p, keep


@dataclass
class DepthMap:  # depth.rs:141
    depth: np.ndarray
    conf: np.ndarray
    w: int
    h: int
    dw: int
    dh: int
    floor: np.ndarray
    floor_value: float = 0.0
    p90: float = 0.0
    wls_rel: float = 0.0
    wls_rel64: float = 0.0
    wls_iters: int = 0
    wls_iters_first: int = 0


@dataclass
class Output:  # stack.rs:244 Output (the hot-path part)
    image: np.ndarray  # (3, h, w) float32 in [0, 1]
    image_u16: np.ndarray  # (h, w, 3) uint16
    winner: np.ndarray  # (h, w) float32
    depth: DepthMap | None
    align: np.ndarray  # (n, 8) Sim vectors
    gains: np.ndarray  # (n, 3)
    shares: np.ndarray
    levels: int
    crop: tuple
    align_evals: int = 0
    ms: dict = field(default_factory=dict)


STAGES = ["align", "gains", "fold", "collapse", "aggregate", "wls", "upsample", "total", "fold_level0", "select_level0",
          "reduce_level0", "wls_solve"]

# Live handles, released stacks-first at interpreter exit while the CUDA
# runtime is still up (a finaliser run during shutdown does nothing).
_live_stacks: "weakref.WeakSet" = weakref.WeakSet()
_live_engines: "weakref.WeakSet" = weakref.WeakSet()


@atexit.register
def _release_all():
    for s in list(_live_stacks):
        s.close()
    for e in list(_live_engines):
        e.close()


def _ptr(a):
    """A host numpy array or a CUDA tensor -> (void*, keep-alive)."""
    if isinstance(a, np.ndarray):
        a = np.ascontiguousarray(a)
        return C.c_void_p(a.ctypes.data), a
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            a = a.contiguous()
        return C.c_void_p(a.data_ptr()), a
    raise TypeError(f"expected a numpy array or a tensor, got {type(a)}")


class Engine:
    """lsb_engine: one CUDA device, one stream (gpu.rs:308-324's set-up, once)."""

    STORAGE = {"f32": 0, "unorm16": 1, "f16": 2}

    def __init__(self, device: int = 0, storage: str = "f32", grid_limit: int = 0, log=None, fused_fold0: bool = True,
                 fold_beside_chain: bool = False, direct_window_sums: bool = False):
        """storage: "f32" (bit-exact with the reference FP32 path), "unorm16" (16-bit
        Gaussian levels, FP16 slices) or "f16" (IEEE half levels and slices).
        fused_fold0=False folds level 0 with the separate REDUCE and select kernels on
        every tile (LSB_FLAG_TWO_KERNEL_FOLD0); fold_beside_chain=True folds an aligned
        stack in device memory chunk by chunk beside its registration chain instead of
        after it (LSB_FLAG_FOLD_BESIDE_CHAIN); direct_window_sums=True forms the depth
        pass's guided-filter window sums tap by tap instead of as moving sums
        (LSB_FLAG_DIRECT_WINDOW_SUMS). None changes a result."""
        self._L = load()
        self._logcb = LOG_FN(lambda line, _u: log(line.decode())) if log else LOG_FN()
        flags = (0 if fused_fold0 else 1) | (2 if fold_beside_chain else 0) | (4 if direct_window_sums else 0)
        cfg = Config(device, self.STORAGE[storage], grid_limit, flags, self._logcb, None)
        h = C.c_void_p()
        check(self._L.lsb_engine_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.storage = storage
        _live_engines.add(self)

    @property
    def stream(self):
        return self._L.lsb_engine_stream(self._h)

    def close(self):
        if getattr(self, "_h", None):
            self._L.lsb_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        if sys.is_finalizing():
            return
        try:
            self.close()
        except Exception:
            pass

    def stack(self, w, h, n, fuse=None, align=None, depth=None, brightness=True, crop=True):
        return Stack(self, w, h, n, fuse, align, depth, brightness, crop)

    def prep_frame(self, rgb, prep: FramePrep, size=None) -> np.ndarray:
        """lapstack-web lib.rs:766-784 on one (h, w, 3) uint16 frame on the device: the dust map (frames of
        its size only), the quarter turns, the draft block mean and, with size = (w, h), the run's size."""
        a = np.ascontiguousarray(rgb, dtype=np.uint16)
        p, keep = prep.c()
        rw, rh = (int(size[0]), int(size[1])) if size is not None else (0, 0)
        wh = (C.c_uint32 * 2)()
        check(self._L.lsb_prep_frame_u16(self._h, C.byref(p), C.c_void_p(a.ctypes.data), a.shape[1], a.shape[0], rw, rh, None, wh))
        out = np.empty((wh[1], wh[0], 3), np.uint16)
        check(self._L.lsb_prep_frame_u16(self._h, C.byref(p), C.c_void_p(a.ctypes.data), a.shape[1], a.shape[0], rw, rh,
                                         C.c_void_p(out.ctypes.data), wh))
        return out

    def resize(self, planes, w: int, h: int, interp: int = 3) -> np.ndarray:
        """prep.rs:46 `resize` / :63 `resize_plane` on the device: (p, ph, pw) or (ph, pw) float32 planes
        resampled to (..., h, w) with pixel centres kept (interp: align.rs:148 code, 3 = Spline4x4)."""
        a = np.ascontiguousarray(planes, dtype=np.float32)
        one = a.ndim == 2
        if one:
            a = a[None]
        out = np.empty((a.shape[0], h, w), np.float32)
        check(self._L.lsb_resize(self._h, C.c_void_p(a.ctypes.data), a.shape[0], a.shape[2], a.shape[1], w, h, interp,
                                 C.c_void_p(out.ctypes.data)))
        return out[0] if one else out


def slab_ranges(count: int, size: int, overlap: int = 0) -> list:
    """stack.rs:76 `slab_ranges`: (lo, hi) inclusive frame ranges of `size` frames (clamped to
    [1, count]), consecutive ones overlapping by `overlap` (at most size - 1), the last cut short."""
    L = load()
    k = L.lsb_slab_ranges(count, size, overlap, None, 0)
    buf = (C.c_uint32 * (2 * max(k, 1)))()
    L.lsb_slab_ranges(count, size, overlap, buf, k)
    return [(buf[2 * i], buf[2 * i + 1]) for i in range(k)]


def check_params(fuse=None, align=None, depth=None):
    """Raises LsbError for settings a stack would refuse (lsb_check_params); needs no device.
    None stands for the defaults (fuse) or for the pass being off (align, depth), as in Engine.stack."""
    L = load()
    fp = (fuse or FuseParams()).c()
    ap = (align or AlignParams()).c(enabled=align is not None)
    dp = (depth or DepthParams()).c(enabled=depth is not None)
    check(L.lsb_check_params(C.byref(fp), C.byref(ap), C.byref(dp)))


_default = None


def default_engine() -> Engine:
    global _default
    if _default is None:
        _default = Engine()
    return _default


def _arr(ptr, n, dt):
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True)


class _ResultOwner:
    """Frees an lsb_result once no array viewing its buffers is left."""

    def __init__(self, lib, r):
        self._lib, self._r = lib, r

    def __del__(self):
        try:
            self._lib.lsb_result_free(C.byref(self._r))
        except Exception:
            pass


def _view(owner, ptr, n, dt):
    """A numpy view of a result buffer (no copy) that keeps the result alive."""
    ct = np.ctypeslib.as_ctypes_type(np.dtype(dt))
    buf = (ct * n).from_address(C.cast(ptr, C.c_void_p).value)
    buf._owner = owner
    return np.frombuffer(buf, dtype=dt)


class Stack:
    """One stack: push frames (host or device), then finish (stack.rs:1011 run_with)."""

    def __init__(self, engine: Engine, w, h, n, fuse=None, align=None, depth=None, brightness=True, crop=True):
        self.e, self.w, self.h, self.n = engine, w, h, n
        self._L = engine._L
        self.fuse = fuse or FuseParams()
        self.align = align
        self.depth = depth
        fp = self.fuse.c()
        ap = (align or AlignParams()).c(enabled=align is not None)
        dp = (depth or DepthParams()).c(enabled=depth is not None)
        hnd = C.c_void_p()
        check(self._L.lsb_stack_begin(engine._h, w, h, n, C.byref(fp), C.byref(ap), C.byref(dp), int(brightness), int(crop),
                                      C.byref(hnd)))
        self._h = hnd
        self._keep = []
        self.count = 0  # frames pushed (or declared with set_count)
        self._prep = None
        _live_stacks.add(self)

    def close(self):
        if getattr(self, "_h", None):
            self._L.lsb_stack_destroy(self._h)
            self._h = None

    def __del__(self):
        if sys.is_finalizing():
            return
        try:
            self.close()
        except Exception:
            pass

    def push_u16(self, rgb, stride_px: int = 0):
        """One decoded frame, (h, w, 3) uint16 (numpy or CUDA tensor). A frame of another size than the
        stack's (or any frame, with a preparation set) goes through the preparation and is brought to
        the stack's size (lsb_stack_push_u16_sized)."""
        p, keep = _ptr(rgb)
        h, w = int(rgb.shape[0]), int(rgb.shape[1])
        if stride_px == 0 and (self._prep is not None or (w, h) != (self.w, self.h)):
            check(self._L.lsb_stack_push_u16_sized(self._h, p, w, h))
        else:
            check(self._L.lsb_stack_push_u16(self._h, p, stride_px))
        self.count += 1
        self._keep.append(keep)  # async copies from host memory complete before the next sync

    def set_prep(self, prep: FramePrep | None):
        """stack.rs:52-58 the dust map, quarter turns and draft level every decoded frame goes through
        (lapstack-web lib.rs:766-784), on the device as each frame lands; before the first push."""
        if prep is None:
            check(self._L.lsb_stack_set_prep(self._h, None))
        else:
            p, keep = prep.c()
            check(self._L.lsb_stack_set_prep(self._h, C.byref(p)))
        self._prep = prep

    def push_f32(self, planes):
        """AnyFuser::push(&Img3): (3, h, w) float32 planes in [0, 1]."""
        ps = []
        for c in range(3):
            p, keep = _ptr(planes[c])
            ps.append(p)
            self._keep.append(keep)
        arr = (C.c_void_p * 3)(*ps)
        check(self._L.lsb_stack_push_f32(self._h, arr))
        self.count += 1

    push = push_f32

    def weighted_average(self, wav: WavParams | None = None) -> np.ndarray:
        """stack.rs:857 / wav.rs:92 the weighted average of the frames of the last finish (or run), with
        its depth pass's noise floor: (3, h, w) float32 in [0, 1]."""
        out = np.empty((3, self.h, self.w), np.float32)
        p = (wav or WavParams()).c()
        check(self._L.lsb_stack_weighted_average(self._h, C.byref(p), C.c_void_p(out.ctypes.data)))
        return out

    def fuse_range(self, lo: int, hi: int, rect=None, size=None, interp: int = 3) -> np.ndarray:
        """stack.rs:740 `fuse_range` over frames lo..hi (inclusive) of the last finish (or run), fused on
        their own, cut to rect = (x, y, w, h) and resized to size = (w, h) as stack.rs:872 `fuse_slabs`
        does (Spline4x4 by default): (3, oh, ow) float32. The stack's own results stay as they were."""
        r = None
        if rect is not None:
            r = (C.c_uint32 * 4)(*[int(v) for v in rect])
        ow, oh = (int(size[0]), int(size[1])) if size is not None else (0, 0)
        w, h = (ow, oh) if size is not None else ((int(rect[2]), int(rect[3])) if rect is not None else (self.w, self.h))
        out = np.empty((3, h, w), np.float32)
        check(self._L.lsb_stack_fuse_range(self._h, lo, hi, r, ow, oh, interp, C.c_void_p(out.ctypes.data)))
        return out

    def slabs(self, size: int, overlap: int = 0, rect=None, restretch=None, interp: int = 3):
        """stack.rs:872 `fuse_slabs` after a finish: (index, count, lo, hi, image) for each slab of
        slab_ranges(count, size, overlap), each fused on its own, cut to rect and, with restretch = (w, h),
        resized to that size; one at a time, none kept."""
        ranges = slab_ranges(self.count, size, overlap)
        for k, (lo, hi) in enumerate(ranges):
            yield k, len(ranges), lo, hi, self.fuse_range(lo, hi, rect, restretch, interp)

    def set_warm_start(self, net):
        """Start this stack's WLS solves from the U-Net's prediction (None: the reference's FGS start)."""
        check(self._L.lsb_stack_set_warm_start(self._h, net._h if net is not None else None))
        self._net = net  # the stack does not own the network; keep it alive

    def autotune(self):
        """Time the persistent kernels' grid sizes on this stack's frames; the engine keeps the fastest."""
        from ._lib import Tuning
        t = Tuning()
        check(self._L.lsb_stack_autotune(self._h, C.byref(t)))
        self._keep.clear()
        return dict(candidates=list(t.candidates), fold_ms=list(t.fold_ms), aggregate_ms=list(t.aggregate_ms),
                    grid_select=t.grid_select, grid_aggregate=t.grid_aggregate)

    def depth_planes(self):
        """Device pointers of the last run's depth-grid planes: guide, d, conf, u, and (dw, dh)."""
        ps = [C.c_void_p() for _ in range(4)]
        dw, dh = C.c_uint32(), C.c_uint32()
        check(self._L.lsb_stack_depth_planes(self._h, *[C.byref(p) for p in ps], C.byref(dw), C.byref(dh)))
        return [p.value for p in ps], (dw.value, dh.value)

    def frames_device(self):
        p = C.c_void_p()
        check(self._L.lsb_stack_frames_device(self._h, C.byref(p)))
        return p.value

    def set_count(self, count):
        check(self._L.lsb_stack_set_count(self._h, count))
        self.count = count

    def shares(self):
        out = np.zeros(self.n, np.float32)
        check(self._L.lsb_stack_shares(self._h, C.c_void_p(out.ctypes.data)))
        self._keep.clear()
        return out

    def run(self):
        """The whole pipeline, results left on the device; per-stage device ms."""
        ms = np.zeros(12, np.float64)
        check(self._L.lsb_stack_run(self._h, C.c_void_p(ms.ctypes.data)))
        self._keep.clear()
        return dict(zip(STAGES, ms.tolist()))

    def finish(self) -> Output:
        r = Result()
        check(self._L.lsb_stack_finish(self._h, C.byref(r)))
        self._keep.clear()
        return _output_of(self._L, r)


def _output_of(lib, r) -> Output:
    """An Output over an lsb_result; the large planes are views of the library's buffers."""
    own = _ResultOwner(lib, r)
    w, h, n = r.w, r.h, r.n_frames
    img = _view(own, r.image_f32, 3 * w * h, np.float32).reshape(3, h, w)
    u16 = _view(own, r.image_u16, 3 * w * h, np.uint16).reshape(h, w, 3)
    win = _view(own, r.winner, w * h, np.float32).reshape(h, w)
    dm = None
    if r.depth:
        dm = DepthMap(_view(own, r.depth, w * h, np.float32).reshape(h, w), _view(own, r.conf, w * h, np.float32).reshape(h, w),
                      w, h, r.dw, r.dh, _arr(r.floor_cells, r.dw * r.dh, np.float32).reshape(r.dh, r.dw), r.floor_value,
                      r.p90, r.wls_rel, r.wls_rel64, r.wls_iters, r.wls_iters_first)
    return Output(img, u16, win, dm, _arr(r.sims, 8 * n, np.float64).reshape(n, 8),
                  _arr(r.gains, 3 * n, np.float32).reshape(n, 3), _arr(r.shares, n, np.float32), r.levels,
                  tuple(r.crop), r.align_evals, dict(zip(STAGES, list(r.ms))))


def batch_run(stacks) -> list:
    """Several pushed stacks of uneven sizes, one Output each (lsb_batch_run). Stacks of one
    engine run back to back; stacks of different engines on the device run side by side (give
    each engine a share of the SMs through grid_limit)."""
    if not stacks:
        return []
    lib = stacks[0]._L
    n = len(stacks)
    hs = (C.c_void_p * n)(*[st._h.value for st in stacks])
    rs = (Result * n)()
    check(lib.lsb_batch_run(hs, n, rs))
    outs = []
    for i, st in enumerate(stacks):
        st._keep.clear()
        outs.append(_output_of(lib, rs[i]))
    return outs


class GpuFuser:
    """gpu.rs:326 `GpuFuser` (the AnyFuser contract of stack.rs:123): push
    aligned, equalised RGB frames as (3, h, w) float32 planes, then shares /
    finish. finish returns the fused image (clamped) and the winner map of
    depth_level upsampled to full resolution, as fuse.rs:499 `finish`."""

    def __init__(self, w, h, params: FuseParams | None = None, n_max: int = 64, engine: Engine | None = None):
        self.w, self.h = w, h
        self.params = params or FuseParams()
        self._s = Stack(engine or default_engine(), w, h, n_max, self.params, None, None, brightness=False, crop=False)
        self.count = 0

    @property
    def levels(self):
        return _levels_of(self.w, self.h, self.params)

    def push(self, planes):
        self._s.push_f32(planes)
        self.count += 1

    def shares(self):
        return self._s.shares()[:self.count]

    def finish(self):
        o = self._s.finish()
        return o.image, o.winner


def _levels_of(w, h, p: FuseParams):
    if p.levels:
        return p.levels
    cw, ch, k = w, h, 0
    while (cw > 1 or ch > 1) and min((cw + 1) // 2, (ch + 1) // 2) >= 32:
        cw, ch, k = (cw + 1) // 2, (ch + 1) // 2, k + 1
    return max(k, 1)


def depth_from_slices(slices, fused, params: DepthParams | None = None, engine: Engine | None = None) -> DepthMap:
    """gpu.rs:1327: slices (n, dh, dw) float32, fused (3, h, w) float32 -> DepthMap."""
    e = engine or default_engine()
    p = params or DepthParams()
    sl = np.ascontiguousarray(slices, dtype=np.float32)
    fu = np.ascontiguousarray(fused, dtype=np.float32)
    _, h, w = fu.shape
    dp = p.c()
    r = Result()
    check(e._L.lsb_depth_from_slices(e._h, C.c_void_p(sl.ctypes.data), sl.shape[0], C.c_void_p(fu.ctypes.data), w, h,
                                     C.byref(dp), C.byref(r)))
    try:
        return DepthMap(_arr(r.depth, w * h, np.float32).reshape(h, w), _arr(r.conf, w * h, np.float32).reshape(h, w), w, h, r.dw,
                        r.dh, _arr(r.floor_cells, r.dw * r.dh, np.float32).reshape(r.dh, r.dw), r.floor_value, r.p90, r.wls_rel,
                        r.wls_rel64, r.wls_iters, r.wls_iters_first)
    finally:
        e._L.lsb_result_free(C.byref(r))


def wls_solve(d, conf, guide, lam, sigma_c, max_iters=200, edge_mode=0, vcycle_mode=0, engine: Engine | None = None):
    """depth.rs:1081 `wls_solve`: (u, rel, iters, device ms)."""
    e = engine or default_engine()
    d, conf, guide = (np.ascontiguousarray(x, dtype=np.float32) for x in (d, conf, guide))
    h, w = d.shape
    u = np.empty_like(d)
    rel, it, ms = C.c_float(0), C.c_uint32(0), C.c_double(0)
    check(e._L.lsb_wls_solve(e._h, C.c_void_p(d.ctypes.data), C.c_void_p(conf.ctypes.data), C.c_void_p(guide.ctypes.data), w, h,
                             lam, sigma_c, max_iters, edge_mode, vcycle_mode, C.c_void_p(u.ctypes.data), C.byref(rel),
                             C.byref(it), C.byref(ms)))
    return u, rel.value, it.value, ms.value


def multiscale_align(rf, tg, init=None, free=None, coarsen=0, engine: Engine | None = None):
    """align.rs:896 `multiscale_align` of luma plane tg onto rf: (Sim vector, evaluations)."""
    e = engine or default_engine()
    rf, tg = (np.ascontiguousarray(x, dtype=np.float32) for x in (rf, tg))
    h, w = rf.shape
    init = np.asarray(init if init is not None else [0, 0, 1, 0, 1, 0, 0, 0], np.float64)
    fr = np.asarray(free if free is not None else AlignParams().free(), np.uint8)
    out = np.empty(8, np.float64)
    ev = C.c_uint32(0)
    check(e._L.lsb_align_pair(e._h, C.c_void_p(rf.ctypes.data), C.c_void_p(tg.ctypes.data), w, h, C.c_void_p(init.ctypes.data),
                              C.c_void_p(fr.ctypes.data), coarsen, C.c_void_p(out.ctypes.data), C.byref(ev)))
    return out, ev.value


def warp_cost(rf, tgt, sim, engine: Engine | None = None):
    """align.rs:581 `warp_cost` on the device."""
    e = engine or default_engine()
    rf, tgt = (np.ascontiguousarray(x, dtype=np.float32) for x in (rf, tgt))
    s = np.asarray(sim, np.float64)
    out = C.c_double(0)
    check(e._L.lsb_warp_cost(e._h, C.c_void_p(rf.ctypes.data), rf.shape[1], rf.shape[0], C.c_void_p(tgt.ctypes.data), tgt.shape[1],
                             tgt.shape[0], C.c_void_p(s.ctypes.data), C.byref(out)))
    return out.value


# ---------------------------------------------------------------- synthetic
@dataclass
class SynthSpec:
    """A seeded synthetic focus stack (the benchmark inputs)."""
    w: int
    h: int
    n: int
    seed: int = 0x1A957ACC
    mag_step: float = 0.002
    noise_std: float = 0.003
    blur_px: float = 6.0
    warp: bool = False
    warp_scale: float = 0.004
    warp_rot_deg: float = 0.2
    warp_shift: float = 8.0

    def c(self):
        return SynthDesc(self.w, self.h, self.n, int(self.warp), self.seed, self.mag_step, self.noise_std, self.blur_px,
                         self.warp_scale, self.warp_rot_deg, self.warp_shift)


def synth_stack(spec: SynthSpec):
    """(n, h, w, 3) uint16 frames made on the host (OpenMP) and the applied transforms (n, 4)."""
    L = load()
    out = np.empty((spec.n, spec.h, spec.w, 3), np.uint16)
    truth = np.empty((spec.n, 4), np.float64)
    d = spec.c()
    err = L.lsb_synth_stack_host(C.byref(d), C.c_void_p(out.ctypes.data), C.c_void_p(truth.ctypes.data))
    if err:
        raise LsbError(err.decode())
    return out, truth


def synth_stack_device(spec: SynthSpec, dst_ptr: int, stream=None):
    """Generate the stack straight into device memory at dst_ptr ([n][h][w][3] u16)."""
    L = load()
    truth = np.empty((spec.n, 4), np.float64)
    d = spec.c()
    err = L.lsb_synth_stack_device(C.byref(d), C.c_void_p(dst_ptr), C.c_void_p(truth.ctypes.data), C.c_void_p(stream or 0))
    if err:
        raise LsbError(err.decode())
    return truth
