"""ctypes binding of the oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the CPU restatement of ragtux/LAPSTACK's stacking path
(crates/lapstack-core/src/{pyramid,fuse,align,brightness,depth,stack}.rs),
built from oracle/*.hpp into oracle/_build/liblsb_oracle.so. It is the
checker the CUDA engine is compared against. Only tests/, smoke() and
bench.py's CPU legs may import this module; the engine never does.

Parameter blocks follow the reference's defaults (fuse.rs:94-107,
align.rs:66-70, depth.rs:93-109, stack.rs:106-120).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblsb_oracle.so")

_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, no GPU needed)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


P = C.c_void_p
F32 = np.float32
F64 = np.float64


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _declare(L):
    sz = C.c_size_t
    for name, res, args in [
        ("orc_reflect", sz, [C.c_long, sz]),
        ("orc_auto_levels", sz, [sz, sz, sz]),
        ("orc_reduce_f", None, [P, sz, sz, P]),
        ("orc_expand_f", None, [P, sz, sz, sz, sz, P]),
        ("orc_build_collapse_f", None, [P, sz, sz, sz, P]),
        ("orc_binomial_f", None, [sz, P]),
        ("orc_window_sum_f", None, [P, sz, sz, P, sz, P]),
        ("orc_region_energy_f", None, [P, sz, sz, sz, C.c_int, P]),
        ("orc_halo_weight", C.c_float, [C.c_float, C.c_float]),
        ("orc_winner_shares", None, [P, P, sz, sz, P]),
        ("orc_deviation_entropy_f", None, [P, sz, sz, sz, sz, P, P]),
        ("orc_fuse_residuals_f", None, [P, sz, sz, sz, P, P]),
        ("orc_sim_matrix", None, [P, sz, sz, P]),
        ("orc_mat_inverse", None, [P, P]),
        ("orc_interp_weights", C.c_int, [C.c_int, C.c_double, P]),
        ("orc_spline4f", None, [C.c_float, P]),
        ("orc_warp_plane_f", None, [P, sz, sz, P, sz, sz, C.c_int, P, P]),
        ("orc_warp_cost_f", C.c_double, [P, sz, sz, P, sz, sz, P]),
        ("orc_reduce_burt_f", None, [P, sz, sz, P]),
        ("orc_gauss_levels_f", sz, [P, sz, sz, P, P]),
        ("orc_level_steps", None, [P, sz, sz, sz, sz, P, P]),
        ("orc_multiscale_align_f", None, [P, P, sz, sz, P, P, sz, P, P]),
        ("orc_nm_step_kinds", None, [P, C.c_int]),
        ("orc_common_area", None, [P, sz, sz, sz, C.c_int, P]),
        ("orc_brightness_gains_f", None, [P, P, sz, sz, P, P]),
        ("orc_brightness_gains_to_f", None, [P, P, sz, sz, P]),
        ("orc_box_mean_f", None, [P, sz, sz, sz, P]),
        ("orc_guided_filter_f", None, [P, P, sz, sz, sz, C.c_float, P]),
        ("orc_rdf_taps_f", sz, [sz, sz, P]),
        ("orc_focus_measure_f", None, [P, sz, sz, P, P]),
        ("orc_focus_slice_f", None, [P, sz, sz, P, P]),
        ("orc_block_mean_f", None, [P, sz, sz, sz, P]),
        ("orc_upsample_bilinear_f", None, [P, sz, sz, sz, sz, sz, P]),
        ("orc_peak_track_f", None, [P, sz, sz, C.c_float, P, P, P, P]),
        ("orc_normalize_conf_f", C.c_float, [P, sz]),
        ("orc_median3_f", None, [P, sz, sz, P]),
        ("orc_wls_solve_f", None, [P, P, P, sz, sz, C.c_float, C.c_float, sz, P, P, P, C.c_int]),
        ("orc_wls_solve_d", None, [P, P, P, sz, sz, C.c_double, C.c_double, sz, P, P, P, C.c_int]),
        ("orc_wls_levels_f", sz, [P, sz, sz]),
        ("orc_depth_from_slices_f", None, [P, sz, sz, P, sz, sz, P, P, P, P, P]),
        ("orc_depth_from_slices_d", None, [P, sz, sz, P, sz, sz, P, P, P, P, P]),
        ("orc_run_stack", P, [P, sz, sz, sz, P, C.c_int]),
        ("orc_stack_free", None, [P]),
        ("orc_stack_image", None, [P, P, P]),
        ("orc_stack_winner", None, [P, P]),
        ("orc_stack_depth", None, [P, P, P, P]),
        ("orc_stack_stats", None, [P, P]),
        ("orc_stack_sims", None, [P, P, P, P]),
        ("orc_stack_begin", P, [sz, sz, sz, P, C.c_int]),
        ("orc_stack_push", None, [P, P, C.c_int]),
        ("orc_stack_cycle_slices", None, [P, sz]),
        ("orc_stack_end", P, [P]),
        ("orc_stack_abort", None, [P]),
        ("orc_set_threads", None, [C.c_int]),
        ("orc_threads", C.c_int, []),
        ("orc_synth_stack", C.c_int, [P, P, P, C.c_uint32, C.c_uint32]),
        ("orc_stack_wav", C.c_int, [P, P]),
        ("orc_weighted_average_f", None, [P, sz, sz, sz, P, P, P, P, P]),
        ("orc_stack_slabs", sz, [P, P, P]),
        ("orc_dust_apply_rgb16", None, [P, sz, P, P, sz, sz, C.c_int, P, sz, sz]),
        ("orc_dust_apply_f", None, [P, sz, P, P, sz, sz, C.c_int, P, sz, sz]),
        ("orc_pull_push_f", None, [P, P, sz, sz, P]),
        ("orc_rotate_f", None, [P, sz, sz, C.c_int, C.c_int, P]),
        ("orc_draft_reduce_f", None, [P, sz, sz, C.c_int, P]),
        ("orc_prep_rgb16", None, [P, sz, P, P, sz, sz, C.c_int, C.c_int, C.c_int, P, sz, sz, sz, sz, P, P]),
        ("orc_slab_ranges", sz, [sz, sz, sz, P, sz]),
        ("orc_resize_f", None, [P, sz, sz, sz, sz, sz, C.c_int, P]),
    ]:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    for s in ("f", "d"):
        getattr(L, f"orc_fuser_new_{s}").restype = P
        getattr(L, f"orc_fuser_new_{s}").argtypes = [sz, sz, P]
        getattr(L, f"orc_fuser_levels_{s}").restype = sz
        getattr(L, f"orc_fuser_levels_{s}").argtypes = [P]
        getattr(L, f"orc_fuser_push_{s}").argtypes = [P, P]
        getattr(L, f"orc_fuser_shares_{s}").restype = sz
        getattr(L, f"orc_fuser_shares_{s}").argtypes = [P, P]
        getattr(L, f"orc_fuser_winner_{s}").argtypes = [P, P]
        getattr(L, f"orc_fuser_finish_{s}").argtypes = [P, P, P]
        getattr(L, f"orc_fuser_free_{s}").argtypes = [P]


# ----------------------------------------------------------------- parameters
TOP_RULES = {"de": 0, "dev": 1, "avg": 2}
INTERPS = ["nearest", "bilinear", "bicubic", "spline4x4", "spline6x6", "lanczos3"]
MODELS = ["similarity", "affine", "projective"]


@dataclass
class FuseParams:  # fuse.rs:70-107
    levels: int = 0  # 0 = auto (residual short side >= 32)
    energy_radius: int = 1
    top_rule: str = "de"
    top_radius: int = 2
    entropy_bins: int = 256
    use_chroma: bool = False
    depth_level: int = 2
    halo: float = 0.0

    def arr(self):
        return [self.levels, self.energy_radius, TOP_RULES[self.top_rule], self.top_radius, self.entropy_bins,
                float(self.use_chroma), self.depth_level, self.halo]


@dataclass
class AlignParams:  # align.rs:52-70
    shift: bool = True
    scale: bool = True
    rotation: bool = True
    model: str = "similarity"
    coarsen: int = 0
    interp: str = "spline4x4"

    def arr(self):
        return [float(self.shift), float(self.scale), float(self.rotation), MODELS.index(self.model), self.coarsen,
                INTERPS.index(self.interp)]

    def free(self):
        a, p = self.model != "similarity", self.model == "projective"
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

    def arr(self):
        # a misspelt mode must not silently select the other one
        assert self.focus in ("rdf", "sml") and self.upsample in ("bilinear", "guided"), (self.focus, self.upsample)
        return [self.scale, 0 if self.focus == "rdf" else 1, self.r_in, self.r_out, self.sml_step, self.agg_radius,
                self.agg_eps, self.lam, self.sigma_c, self.cg_iters, float(self.median),
                0 if self.upsample == "bilinear" else 1, self.up_radius, self.up_eps, self.gate, self.robust]


@dataclass
class WavParams:  # wav.rs:52-80
    power: float = 2.0
    smooth: int = 3
    gate: float = 0.5
    edge: bool = True


@dataclass
class StackParams:  # stack.rs:27-71 (the hot-path subset)
    fuse: FuseParams = field(default_factory=FuseParams)
    align: AlignParams | None = field(default_factory=AlignParams)
    depth: DepthParams | None = field(default_factory=DepthParams)
    brightness: bool = True
    crop: bool = True
    wav: WavParams | None = None  # stack.rs:857 the weighted average too (needs depth)
    # the engine's 16-bit level storage to emulate ("f32": the reference itself; "unorm16", "f16")
    storage: str = "f32"
    # stack.rs:55 `slabs`: (size, overlap), each slab fused on its own after the result
    slabs: tuple | None = None

    def arr(self):
        a = self.fuse.arr() + (self.align or AlignParams()).arr() + (self.depth or DepthParams()).arr()
        a += [float(self.align is not None), float(self.depth is not None), float(self.brightness), float(self.crop)]
        w = self.wav or WavParams()
        a += [float(self.wav is not None), w.power, w.smooth, w.gate, float(w.edge)]
        a += [float(["f32", "unorm16", "f16"].index(self.storage))]
        a += [float(self.slabs[0]), float(self.slabs[1])] if self.slabs else [0.0, 0.0]
        return np.asarray(a, dtype=F64)


def _arr(v):
    return np.ascontiguousarray(np.asarray(v, dtype=F64))


def c32(a):
    return np.ascontiguousarray(a, dtype=F32)


# ------------------------------------------------------------------- pyramid
def reflect(i, n):
    return lib().orc_reflect(i, n)


def auto_levels(w, h, min_top=32):
    return lib().orc_auto_levels(w, h, min_top)


def half(n):
    return (n + 1) // 2


def reduce(src):
    src = c32(src)
    h, w = src.shape
    out = np.empty((half(h), half(w)), F32)
    lib().orc_reduce_f(_ptr(src), w, h, _ptr(out))
    return out


def expand(coarse, ow, oh):
    coarse = c32(coarse)
    ch, cw = coarse.shape
    out = np.empty((oh, ow), F32)
    lib().orc_expand_f(_ptr(coarse), cw, ch, ow, oh, _ptr(out))
    return out


def build_collapse(planes, levels):
    planes = c32(planes)
    _, h, w = planes.shape
    out = np.empty_like(planes)
    lib().orc_build_collapse_f(_ptr(planes), w, h, levels, _ptr(out))
    return out


# ---------------------------------------------------------------------- fuse
def binomial(r):
    out = np.empty(2 * r + 1, F32)
    lib().orc_binomial_f(r, _ptr(out))
    return out


def window_sum(src, wt):
    src, wt = c32(src), c32(wt)
    h, w = src.shape
    out = np.empty_like(src)
    lib().orc_window_sum_f(_ptr(src), w, h, _ptr(wt), len(wt), _ptr(out))
    return out


def region_energy(planes, radius=1, use_chroma=False):
    planes = c32(planes)
    _, h, w = planes.shape
    out = np.empty((h, w), F32)
    lib().orc_region_energy_f(_ptr(planes), w, h, radius, int(use_chroma), _ptr(out))
    return out


def halo_weight(re, p):
    return lib().orc_halo_weight(re, p)


def winner_shares(win, best, frames):
    win = np.ascontiguousarray(win, dtype=np.uint16)
    best = c32(best)
    out = np.empty(frames, F32)
    lib().orc_winner_shares(_ptr(win), _ptr(best), win.size, frames, _ptr(out))
    return out


def deviation_entropy(y, radius=2, bins=256):
    y = c32(y)
    h, w = y.shape
    d, e = np.empty_like(y), np.empty_like(y)
    lib().orc_deviation_entropy_f(_ptr(y), w, h, radius, bins, _ptr(d), _ptr(e))
    return d, e


def fuse_residuals(tops, params: FuseParams):
    tops = c32(tops)
    n, _, h, w = tops.shape
    out = np.empty((3, h, w), F32)
    lib().orc_fuse_residuals_f(_ptr(tops), n, w, h, _ptr(_arr(params.arr())), _ptr(out))
    return out


class Fuser:
    """fuse.rs:349 `Fuser`: push planar RGB frames, then shares / finish."""

    def __init__(self, w, h, params: FuseParams | None = None, fp64=False):
        self.w, self.h, self.s = w, h, ("d" if fp64 else "f")
        self.dt = F64 if fp64 else F32
        self._p = _arr((params or FuseParams()).arr())
        self._h = getattr(lib(), f"orc_fuser_new_{self.s}")(w, h, _ptr(self._p))
        self.levels = getattr(lib(), f"orc_fuser_levels_{self.s}")(self._h)
        self.count = 0

    def push(self, planes):
        planes = np.ascontiguousarray(planes, dtype=self.dt)
        assert planes.shape == (3, self.h, self.w)
        getattr(lib(), f"orc_fuser_push_{self.s}")(self._h, _ptr(planes))
        self.count += 1

    def shares(self):
        out = np.empty(max(self.count, 1), F32)
        n = getattr(lib(), f"orc_fuser_shares_{self.s}")(self._h, _ptr(out))
        return out[:n]

    def winner(self, dw, dh):
        out = np.empty((dh, dw), np.uint16)
        getattr(lib(), f"orc_fuser_winner_{self.s}")(self._h, _ptr(out))
        return out

    def finish(self):
        img = np.empty((3, self.h, self.w), self.dt)
        depth = np.empty((self.h, self.w), F32)
        getattr(lib(), f"orc_fuser_finish_{self.s}")(self._h, _ptr(img), _ptr(depth))
        return img, depth

    def __del__(self):
        try:
            getattr(lib(), f"orc_fuser_free_{self.s}")(self._h)
        except Exception:
            pass


# --------------------------------------------------------------------- align
SIM_ID = [0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 0.0]


def sim_matrix(sim, w, h):
    m = np.empty(9, F64)
    lib().orc_sim_matrix(_ptr(_arr(sim)), w, h, _ptr(m))
    return m.reshape(3, 3)


def mat_inverse(m):
    inv = np.empty(9, F64)
    lib().orc_mat_inverse(_ptr(_arr(m).reshape(9)), _ptr(inv))
    return inv.reshape(3, 3)


def interp_weights(kind, t):
    w = np.zeros(6, F64)
    n = lib().orc_interp_weights(INTERPS.index(kind), t, _ptr(w))
    return w[:n]


def warp_plane(src, sim, interp="spline4x4", ow=None, oh=None):
    src = c32(src)
    h, w = src.shape
    ow, oh = ow or w, oh or h
    out = np.empty((oh, ow), F32)
    valid = np.empty((oh, ow), np.uint8)
    lib().orc_warp_plane_f(_ptr(src), w, h, _ptr(_arr(sim)), ow, oh, INTERPS.index(interp), _ptr(out), _ptr(valid))
    return out, valid


def warp_cost(rf, tgt, sim):
    rf, tgt = c32(rf), c32(tgt)
    ah, aw = rf.shape
    th, tw = tgt.shape
    return lib().orc_warp_cost_f(_ptr(rf), aw, ah, _ptr(tgt), tw, th, _ptr(_arr(sim)))


def reduce_burt(src):
    src = c32(src)
    h, w = src.shape
    out = np.empty((half(h), half(w)), F32)
    lib().orc_reduce_burt_f(_ptr(src), w, h, _ptr(out))
    return out


def gauss_levels(y):
    y = c32(y)
    h, w = y.shape
    dims = np.zeros(128, np.uint64)
    n = lib().orc_gauss_levels_f(_ptr(y), w, h, _ptr(dims), None)
    total = sum(int(dims[2 * l]) * int(dims[2 * l + 1]) for l in range(n))
    buf = np.empty(total, F32)
    lib().orc_gauss_levels_f(_ptr(y), w, h, _ptr(dims), _ptr(buf))
    out, o = [], 0
    for l in range(n):
        lw, lh = int(dims[2 * l]), int(dims[2 * l + 1])
        out.append(buf[o:o + lw * lh].reshape(lh, lw))
        o += lw * lh
    return out


def level_steps(free_idx, lvl, w, h):
    fi = np.asarray(free_idx, np.uint64)
    step, tol = np.empty(len(fi), F64), np.empty(len(fi), F64)
    lib().orc_level_steps(_ptr(fi), len(fi), lvl, w, h, _ptr(step), _ptr(tol))
    return step, tol


def multiscale_align(rf, tg, init=None, free=None, coarsen=0):
    rf, tg = c32(rf), c32(tg)
    h, w = rf.shape
    out = np.empty(8, F64)
    ev = C.c_size_t(0)
    fr = np.asarray(free if free is not None else AlignParams().free(), np.uint8)
    lib().orc_multiscale_align_f(_ptr(rf), _ptr(tg), w, h, _ptr(_arr(init or SIM_ID)), _ptr(fr), coarsen, _ptr(out),
                                 C.byref(ev))
    return out, ev.value


def nm_step_kinds(reset=False):
    """Nelder-Mead steps of every search since the last reset, by kind (the oracle's own counters):
    accepted reflections, expansions evaluated, accepted contractions, shrinks, and searches run."""
    k = np.zeros(5, np.uint64)
    lib().orc_nm_step_kinds(_ptr(k), int(reset))
    return dict(zip(("accepted", "expanded", "contracted", "shrunk", "searches"), (int(v) for v in k)))


def common_area(sims, w, h, interp="spline4x4"):
    s = _arr(sims).reshape(-1, 8)
    r = np.empty(4, np.uint64)
    lib().orc_common_area(_ptr(s), len(s), w, h, INTERPS.index(interp), _ptr(r))
    return tuple(int(v) for v in r)


def brightness_gains(ref3, frame3, sim):
    ref3, frame3 = c32(ref3), c32(frame3)
    _, h, w = ref3.shape
    g = np.empty(3, F32)
    lib().orc_brightness_gains_f(_ptr(ref3), _ptr(frame3), w, h, _ptr(_arr(sim)), _ptr(g))
    return g


def brightness_gains_to(ref3, frame3):
    ref3, frame3 = c32(ref3), c32(frame3)
    _, h, w = ref3.shape
    g = np.empty(3, F32)
    lib().orc_brightness_gains_to_f(_ptr(ref3), _ptr(frame3), w, h, _ptr(g))
    return g


# --------------------------------------------------------------------- depth
def box_mean(src, r):
    src = c32(src)
    h, w = src.shape
    out = np.empty_like(src)
    lib().orc_box_mean_f(_ptr(src), w, h, r, _ptr(out))
    return out


def guided_filter(guide, p, r, eps):
    guide, p = c32(guide), c32(p)
    h, w = guide.shape
    out = np.empty_like(p)
    lib().orc_guided_filter_f(_ptr(guide), _ptr(p), w, h, r, eps, _ptr(out))
    return out


def rdf_taps(r_in=1, r_out=3):
    buf = np.empty(3 * (2 * r_out + 1) ** 2, F32)
    n = lib().orc_rdf_taps_f(r_in, r_out, _ptr(buf))
    return buf[:3 * n].reshape(n, 3)


def focus_measure(y, params: DepthParams | None = None):
    y = c32(y)
    h, w = y.shape
    out = np.empty_like(y)
    lib().orc_focus_measure_f(_ptr(y), w, h, _ptr(_arr((params or DepthParams()).arr())), _ptr(out))
    return out


def blocks(n, k):
    return (n + k - 1) // k


def focus_slice(planes, params: DepthParams | None = None):
    p = params or DepthParams()
    planes = c32(planes)
    _, h, w = planes.shape
    k = 1 << p.scale
    out = np.empty((blocks(h, k), blocks(w, k)), F32)
    lib().orc_focus_slice_f(_ptr(planes), w, h, _ptr(_arr(p.arr())), _ptr(out))
    return out


def block_mean(src, k):
    src = c32(src)
    h, w = src.shape
    out = np.empty((blocks(h, k), blocks(w, k)), F32)
    lib().orc_block_mean_f(_ptr(src), w, h, k, _ptr(out))
    return out


def upsample_bilinear(g, w, h, k):
    g = c32(g)
    dh, dw = g.shape
    out = np.empty((h, w), F32)
    lib().orc_upsample_bilinear_f(_ptr(g), dw, dh, w, h, k, _ptr(out))
    return out


def peak_track(slices, gate=1.0):
    s = c32(slices)
    n = s.shape[0]
    m = s[0].size
    d, c, mins = np.empty(m, F32), np.empty(m, F32), np.empty(m, F32)
    fl = C.c_float(0)
    lib().orc_peak_track_f(_ptr(s), n, m, gate, _ptr(d), _ptr(c), _ptr(mins), C.byref(fl))
    shp = s.shape[1:]
    return d.reshape(shp), c.reshape(shp), mins.reshape(shp), fl.value


def normalize_conf(conf):
    c = c32(conf).copy()
    p = lib().orc_normalize_conf_f(_ptr(c), c.size)
    return c, p


def median3(src):
    src = c32(src)
    h, w = src.shape
    out = np.empty_like(src)
    lib().orc_median3_f(_ptr(src), w, h, _ptr(out))
    return out


def wls_solve(d, conf, guide, lam, sigma_c, max_iters, fp64=False, edge_mode=0):
    dt, s = (F64, "d") if fp64 else (F32, "f")
    d, conf, guide = (np.ascontiguousarray(x, dtype=dt) for x in (d, conf, guide))
    h, w = d.shape
    u = np.empty_like(d)
    rel = (C.c_double if fp64 else C.c_float)(0)
    it = C.c_size_t(0)
    getattr(lib(), f"orc_wls_solve_{s}")(_ptr(d), _ptr(conf), _ptr(guide), w, h, lam, sigma_c, max_iters, _ptr(u),
                                         C.byref(rel), C.byref(it), int(edge_mode))
    return u, rel.value, it.value


def wls_levels(guide):
    g = c32(guide)
    h, w = g.shape
    return lib().orc_wls_levels_f(_ptr(g), w, h)


def depth_from_slices(slices, fused, params: DepthParams | None = None, fp64=False):
    p = params or DepthParams()
    dt, s = (F64, "d") if fp64 else (F32, "f")
    sl = np.ascontiguousarray(slices, dtype=dt)
    fused = np.ascontiguousarray(fused, dtype=dt)
    _, h, w = fused.shape
    n = sl.shape[0]
    m = sl[0].size
    depth, conf = np.empty((h, w), dt), np.empty((h, w), dt)
    floor_cells = np.empty(m, dt)
    st = np.empty(7, F64)
    getattr(lib(), f"orc_depth_from_slices_{s}")(_ptr(sl), n, m, _ptr(fused), w, h, _ptr(_arr(p.arr())), _ptr(depth),
                                                 _ptr(conf), _ptr(floor_cells), _ptr(st))
    stats = dict(floor=st[0], p90=st[1], rel=st[2], iters=int(st[3]), iters_first=int(st[4]), dw=int(st[5]),
                 dh=int(st[6]))
    return depth, conf, floor_cells.reshape(int(st[6]), int(st[5])), stats


def weighted_average(frames, params: DepthParams | None = None, wav: "WavParams | None" = None, floor=None, guide=None):
    """wav.rs:92 `weighted_average` of (n, 3, h, w) f32 frames: floor on the depth grid (zeros: none),
    guide the fused (3, h, w) image or None (the box mean)."""
    p, wp = params or DepthParams(), wav or WavParams()
    fr = c32(frames)
    n, _, h, w = fr.shape
    k = 1 << p.scale
    fl = c32(floor if floor is not None else np.zeros((blocks(h, k), blocks(w, k)), F32))
    g = c32(guide) if guide is not None else None
    out = np.empty((3, h, w), F32)
    lib().orc_weighted_average_f(_ptr(fr), n, w, h, _ptr(_arr(p.arr())), _ptr(_arr([wp.power, wp.smooth, wp.gate, float(wp.edge)])),
                                 _ptr(fl), _ptr(g), _ptr(out))
    return out


# --------------------------------------------------------------------- stack
@dataclass
class StackResult:
    image: np.ndarray  # (3, h, w) float64 (exact copy of the f32 or f64 result)
    image_u16: np.ndarray  # (h, w, 3) uint16
    winner: np.ndarray  # (h, w) float32 (the fuse winner map, upsampled)
    depth: np.ndarray | None
    conf: np.ndarray | None
    floor_cells: np.ndarray | None
    sims: np.ndarray  # (n, 8)
    gains: np.ndarray  # (n, 3)
    shares: np.ndarray
    stats: dict
    wav: np.ndarray | None = None  # (3, h, w) float64, the weighted average when asked for
    # stack.rs:872 the slabs when asked for: (lo, hi) and each one's fused image (3, h, w) float64, uncut
    slab_ranges: list | None = None
    slabs: np.ndarray | None = None


def slab_ranges(count, size, overlap=0):
    """stack.rs:76 `slab_ranges`: inclusive (lo, hi) frame ranges."""
    k = lib().orc_slab_ranges(count, size, overlap, None, 0)
    buf = np.zeros(2 * max(k, 1), np.uint64)
    lib().orc_slab_ranges(count, size, overlap, _ptr(buf), k)
    return [(int(buf[2 * i]), int(buf[2 * i + 1])) for i in range(k)]


def resize(planes, w, h, interp=3):
    """prep.rs:46 `resize` / :63 `resize_plane` in f32: (p, ph, pw) or (ph, pw) planes to (..., h, w)."""
    a = c32(planes)
    one = a.ndim == 2
    if one:
        a = a[None]
    out = np.empty((a.shape[0], h, w), F32)
    lib().orc_resize_f(_ptr(a), a.shape[0], a.shape[2], a.shape[1], w, h, int(interp), _ptr(out))
    return out[0] if one else out


def run_stack(frames_u16, params: StackParams | None = None, fp64=False) -> StackResult:
    """stack.rs run_with over in-memory interleaved RGB u16 frames (n, h, w, 3)."""
    p = params or StackParams()
    fr = np.ascontiguousarray(frames_u16, dtype=np.uint16)
    n, h, w, _ = fr.shape
    return _result_of(lib().orc_run_stack(_ptr(fr), n, w, h, _ptr(p.arr()), int(fp64)), p, n, w, h)


class StackRun:
    """The same stack one frame at a time: push() registers, gains and folds a frame (the per-frame body
    of stack.rs:785-821), finish() the shares, the fused image, the depth pass and the crop
    (stack.rs:833, 1047-1060). n is the stack's frame count (registration is on only when n > 1)."""

    def __init__(self, n, w, h, params: StackParams | None = None, fp64=False):
        self.p, self.n, self.w, self.h, self.pushed = params or StackParams(), n, w, h, 0
        self._h = lib().orc_stack_begin(n, w, h, _ptr(self.p.arr()), int(fp64))

    def push(self, frame_u16, last=None):
        f = np.ascontiguousarray(frame_u16, dtype=np.uint16)
        assert f.shape == (self.h, self.w, 3)
        last = self.pushed + 1 == self.n if last is None else last
        lib().orc_stack_push(self._h, _ptr(f), int(last))
        self.pushed += 1

    def cycle_slices(self, n_total):
        """For timing only: repeat the pushed frames' focus slices in order up to n_total, so that the
        depth pass runs over a whole stack's worth of slices after a sample of its frames."""
        lib().orc_stack_cycle_slices(self._h, n_total)

    def finish(self) -> "StackResult":
        h, self._h = self._h, None
        return _result_of(lib().orc_stack_end(h), self.p, self.pushed, self.w, self.h)

    def __del__(self):
        try:
            if self._h:
                lib().orc_stack_abort(self._h)
        except Exception:
            pass


def set_threads(n=0):
    """OpenMP threads of every later oracle call (0: all the host's); returns the count now in use."""
    lib().orc_set_threads(int(n))
    return lib().orc_threads()


def synth_stack(w, h, n, seed=0x1A957ACC, mag_step=0.002, noise_std=0.003, blur_px=6.0, warp=False, warp_scale=0.004,
                warp_rot_deg=0.2, warp_shift=8.0, frames=None):
    """The seeded synthetic stack (n, h, w, 3) u16 and the applied transforms (n, 4), made on the host by
    the oracle's twin of the engine's generator (no CUDA library involved). frames=(k0, count): only
    those frames of the n-frame stack."""
    d = _arr([w, h, n, int(warp), seed & 0xFFFFFFFF, seed >> 32, mag_step, noise_std, blur_px, warp_scale, warp_rot_deg,
              warp_shift])
    k0, count = frames or (0, n)
    out = np.empty((count, h, w, 3), np.uint16)
    truth = np.empty((n, 4), F64)
    if lib().orc_synth_stack(_ptr(d), _ptr(out), _ptr(truth), k0, count) != 0:
        raise ValueError("synth_stack: bad description")
    return out, truth


def _result_of(r, p, n, w, h) -> "StackResult":
    L = lib()
    try:
        img = np.empty((3, h, w), F64)
        u16 = np.empty((h, w, 3), np.uint16)
        L.orc_stack_image(r, _ptr(img), _ptr(u16))
        win = np.empty((h, w), F32)
        L.orc_stack_winner(r, _ptr(win))
        st = np.empty(13, F64)
        L.orc_stack_stats(r, _ptr(st))
        stats = dict(levels=int(st[0]), dw=int(st[1]), dh=int(st[2]), floor=st[3], p90=st[4], rel=st[5],
                     iters=int(st[6]), iters_first=int(st[7]), align_evals=int(st[8]),
                     crop=(int(st[9]), int(st[10]), int(st[11]), int(st[12])))
        depth = conf = floor_cells = None
        if p.depth is not None:
            depth, conf = np.empty((h, w), F64), np.empty((h, w), F64)
            floor_cells = np.empty((stats["dh"], stats["dw"]), F64)
            L.orc_stack_depth(r, _ptr(depth), _ptr(conf), _ptr(floor_cells))
        sims, gains = np.empty((n, 8), F64), np.empty((n, 3), F32)
        shares = np.zeros(n, F32)
        L.orc_stack_sims(r, _ptr(sims), _ptr(gains), _ptr(shares))
        wav = np.empty((3, h, w), F64)
        if not L.orc_stack_wav(r, _ptr(wav)):
            wav = None
        ranges = slabs = None
        k = L.orc_stack_slabs(r, None, None)
        if k:
            lohi = np.zeros(2 * k, np.uint64)
            slabs = np.empty((k, 3, h, w), F64)
            L.orc_stack_slabs(r, _ptr(lohi), _ptr(slabs))
            ranges = [(int(lohi[2 * i]), int(lohi[2 * i + 1])) for i in range(k)]
        return StackResult(img, u16, win, depth, conf, floor_cells, sims, gains, shares, stats, wav, ranges, slabs)
    finally:
        L.orc_stack_free(r)


# --------------------------------------------------------------- frame prep
@dataclass
class DustSpot:  # dust.rs:85 Spot: its window at (x, y), mask (h, w) 1 = dust, gain (h, w) for flat mode
    x: int
    y: int
    mask: np.ndarray
    gain: np.ndarray | None = None


@dataclass
class DustMap:  # dust.rs:105 DustMap; mode dust.rs:42 "fill" (pull-push) or "flat"
    w: int
    h: int
    spots: list
    mode: str = "fill"


def _dust_arrays(m: DustMap):
    n = len(m.spots)
    rects = np.zeros((max(n, 1), 4), np.uint64)
    masks, gains = [], []
    for k, s in enumerate(m.spots):
        mk = np.ascontiguousarray(s.mask, dtype=np.uint8)
        rects[k] = (s.x, s.y, mk.shape[1], mk.shape[0])
        masks.append(mk.ravel())
        g = np.ones(mk.shape, F32) if s.gain is None else np.asarray(s.gain, F32)
        gains.append(np.ascontiguousarray(g).ravel())
    masks = np.concatenate(masks) if masks else np.zeros(1, np.uint8)
    gains = np.concatenate(gains) if gains else np.zeros(1, F32)
    return rects, n, masks, gains, {"fill": 0, "flat": 1}[m.mode]


def dust_apply_rgb16(m: DustMap, rgb):
    """dust.rs:487 `apply_rgb16` on a copy of an interleaved (h, w, 3) u16 frame."""
    out = np.array(rgb, dtype=np.uint16, copy=True, order="C")
    rects, n, masks, gains, mode = _dust_arrays(m)
    lib().orc_dust_apply_rgb16(_ptr(rects), n, _ptr(masks), _ptr(gains), m.w, m.h, mode, _ptr(out), out.shape[1], out.shape[0])
    return out


def dust_apply(m: DustMap, planes):
    """dust.rs:478 `apply` on a copy of (3, h, w) f32 planes."""
    out = np.array(planes, dtype=F32, copy=True, order="C")
    rects, n, masks, gains, mode = _dust_arrays(m)
    lib().orc_dust_apply_f(_ptr(rects), n, _ptr(masks), _ptr(gains), m.w, m.h, mode, _ptr(out), out.shape[2], out.shape[1])
    return out


def pull_push(v, wt):
    """dust.rs:591 `pull_push` of (h, w) f32 values with weights in [0, 1]."""
    v, wt = c32(v), c32(wt)
    out = np.empty_like(v)
    lib().orc_pull_push_f(_ptr(v), _ptr(wt), v.shape[1], v.shape[0], _ptr(out))
    return out


def rotate(planes, quarters, flip=False):
    """prep.rs:16 `rotate` of (3, h, w) f32 planes: quarter turns clockwise after an optional mirror."""
    a = c32(planes)
    h, w = a.shape[1:]
    out = np.empty((3, w, h) if quarters % 2 else (3, h, w), F32)
    lib().orc_rotate_f(_ptr(a), w, h, int(quarters), int(flip), _ptr(out))
    return out


def draft_reduce(planes, levels):
    """prep.rs:77 `reduce`: (3, h, w) f32 planes block-averaged by 2^levels."""
    a = c32(planes)
    h, w = a.shape[1:]
    k = 1 << levels
    out = np.empty((3, max(-(-h // k), 1), max(-(-w // k), 1)), F32)
    lib().orc_draft_reduce_f(_ptr(a), w, h, int(levels), _ptr(out))
    return out


def prep_rgb16(rgb, dust: DustMap | None = None, rotate=0, draft=0, size=None):
    """lapstack-web lib.rs:766-784 on an interleaved (h, w, 3) u16 frame: the dust map (frames of its size
    only), the quarter turns, the draft block mean (decode.rs:68, 92) and, with size = (w, h), the run's
    size (decode.rs:125 bilinear)."""
    f = np.ascontiguousarray(rgb, dtype=np.uint16)
    h, w = f.shape[:2]
    rects, n, masks, gains, mode = _dust_arrays(dust) if dust is not None else (np.zeros((1, 4), np.uint64), 0, np.zeros(1, np.uint8),
                                                                                  np.zeros(1, F32), 0)
    mw, mh = (dust.w, dust.h) if dust is not None else (0, 0)
    rw, rh = size if size is not None else (0, 0)
    dims = np.zeros(2, np.uint64)
    L = lib()
    L.orc_prep_rgb16(_ptr(rects), n, _ptr(masks), _ptr(gains), mw, mh, mode, int(rotate), int(draft), _ptr(f), w, h, rw, rh, None, _ptr(dims))
    out = np.empty((int(dims[1]), int(dims[0]), 3), np.uint16)
    L.orc_prep_rgb16(_ptr(rects), n, _ptr(masks), _ptr(gains), mw, mh, mode, int(rotate), int(draft), _ptr(f), w, h, rw, rh, _ptr(out),
                     _ptr(dims))
    return out
