"""ctypes binding of liblapstack_b200.so (include/lapstack_b200.h).

The engine is CUDA-only: loading fails loudly when the library is missing,
and every compute entry point returns the library's error string (raised as
LsbError) when no B200 is present. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_build", "liblapstack_b200.so")
ROOT = os.path.dirname(PKG)
HEADER = os.path.join(ROOT, "include", "lapstack_b200.h")

ABI_VERSION = 1


class LsbError(RuntimeError):
    pass


LOG_FN = C.CFUNCTYPE(None, C.c_char_p, C.c_void_p)


class Config(C.Structure):
    _fields_ = [("device", C.c_int32), ("storage", C.c_int32), ("grid_limit", C.c_int32), ("flags", C.c_int32),
                ("log", LOG_FN), ("user", C.c_void_p)]


class FuseParamsC(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("energy_radius", C.c_uint32), ("top_rule", C.c_uint32), ("top_radius", C.c_uint32),
                ("entropy_bins", C.c_uint32), ("use_chroma", C.c_uint32), ("depth_level", C.c_uint32), ("halo", C.c_float)]


class AlignParamsC(C.Structure):
    _fields_ = [("enabled", C.c_uint32), ("shift", C.c_uint32), ("scale", C.c_uint32), ("rotation", C.c_uint32),
                ("model", C.c_uint32), ("coarsen", C.c_uint32), ("interp", C.c_uint32), ("host_search", C.c_uint32)]


class DepthParamsC(C.Structure):
    _fields_ = [("enabled", C.c_uint32), ("scale", C.c_uint32), ("focus", C.c_uint32), ("r_in", C.c_uint32),
                ("r_out", C.c_uint32), ("sml_step", C.c_uint32), ("agg_radius", C.c_uint32), ("agg_eps", C.c_float),
                ("lam", C.c_float), ("sigma_c", C.c_float), ("cg_iters", C.c_uint32), ("median", C.c_uint32),
                ("upsample", C.c_uint32), ("up_radius", C.c_uint32), ("up_eps", C.c_float), ("gate", C.c_float),
                ("robust", C.c_float), ("edge_mode", C.c_uint32), ("vcycle_mode", C.c_uint32)]


class Result(C.Structure):
    _fields_ = [("w", C.c_uint32), ("h", C.c_uint32), ("n_frames", C.c_uint32), ("levels", C.c_uint32), ("dw", C.c_uint32),
                ("dh", C.c_uint32), ("image_u16", C.POINTER(C.c_uint16)), ("image_f32", C.POINTER(C.c_float)),
                ("winner", C.POINTER(C.c_float)), ("depth", C.POINTER(C.c_float)), ("conf", C.POINTER(C.c_float)),
                ("floor_cells", C.POINTER(C.c_float)), ("sims", C.POINTER(C.c_double)), ("gains", C.POINTER(C.c_float)),
                ("shares", C.POINTER(C.c_float)), ("crop", C.c_uint32 * 4), ("floor_value", C.c_float), ("p90", C.c_float),
                ("wls_rel", C.c_float), ("wls_iters", C.c_uint32), ("wls_iters_first", C.c_uint32),
                ("align_evals", C.c_uint32), ("wls_rel64", C.c_double), ("ms", C.c_double * 12)]


class Tuning(C.Structure):
    _fields_ = [("candidates", C.c_uint32 * 3), ("fold_ms", C.c_double * 3), ("aggregate_ms", C.c_double * 3),
                ("grid_select", C.c_uint32), ("grid_aggregate", C.c_uint32)]


class WavParamsC(C.Structure):
    _fields_ = [("power", C.c_float), ("smooth", C.c_uint32), ("gate", C.c_float), ("edge", C.c_uint32)]


class DustSpotC(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32), ("w", C.c_uint32), ("h", C.c_uint32), ("mask", C.c_void_p),
                ("gain", C.c_void_p)]


class DustMapC(C.Structure):
    _fields_ = [("w", C.c_uint32), ("h", C.c_uint32), ("mode", C.c_uint32), ("n_spots", C.c_uint32),
                ("spots", C.POINTER(DustSpotC))]


class FramePrepC(C.Structure):
    _fields_ = [("dust", C.POINTER(DustMapC)), ("rotate", C.c_uint32), ("draft", C.c_uint32)]


class SynthDesc(C.Structure):
    _fields_ = [("w", C.c_uint32), ("h", C.c_uint32), ("n", C.c_uint32), ("warp", C.c_uint32), ("seed", C.c_uint64),
                ("mag_step", C.c_float), ("noise_std", C.c_float), ("blur_px", C.c_float), ("warp_scale", C.c_float),
                ("warp_rot_deg", C.c_float), ("warp_shift", C.c_float)]


P = C.c_void_p
ERR = C.c_void_p  # char* owned by the library until lsb_free_str

# name -> (restype, argtypes): every entry point include/lapstack_b200.h declares
SIGNATURES = {
    "lsb_abi": (C.c_uint32, []),
    "lsb_free_str": (None, [P]),
    "lsb_launch_count": (C.c_uint64, []),
    "lsb_engine_create": (ERR, [C.POINTER(Config), C.POINTER(P)]),
    "lsb_engine_destroy": (None, [P]),
    "lsb_engine_stream": (P, [P]),
    "lsb_check_params": (ERR, [C.POINTER(FuseParamsC), C.POINTER(AlignParamsC), C.POINTER(DepthParamsC)]),
    "lsb_stack_begin": (ERR, [P, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(FuseParamsC), C.POINTER(AlignParamsC),
                              C.POINTER(DepthParamsC), C.c_int32, C.c_int32, C.POINTER(P)]),
    "lsb_stack_push_u16": (ERR, [P, P, C.c_size_t]),
    "lsb_stack_push_f32": (ERR, [P, C.POINTER(P)]),
    "lsb_stack_frames_device": (ERR, [P, C.POINTER(P)]),
    "lsb_stack_set_count": (ERR, [P, C.c_uint32]),
    "lsb_stack_shares": (ERR, [P, P]),
    "lsb_stack_finish": (ERR, [P, C.POINTER(Result)]),
    "lsb_stack_run": (ERR, [P, P]),
    "lsb_stack_destroy": (None, [P]),
    "lsb_result_free": (None, [C.POINTER(Result)]),
    "lsb_depth_from_slices": (ERR, [P, P, C.c_uint32, P, C.c_uint32, C.c_uint32, C.POINTER(DepthParamsC), C.POINTER(Result)]),
    "lsb_wls_solve": (ERR, [P, P, P, P, C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_uint32, C.c_uint32, C.c_uint32, P, P,
                            P, P]),
    "lsb_align_pair": (ERR, [P, P, P, C.c_uint32, C.c_uint32, P, P, C.c_uint32, P, P]),
    "lsb_warp_cost": (ERR, [P, P, C.c_uint32, C.c_uint32, P, C.c_uint32, C.c_uint32, P, P]),
    "lsb_warp_cost_noalloc": (C.c_char_p, [P, C.c_uint32, C.c_uint32, P, C.c_uint32, C.c_uint32, P, C.c_uint32, P, P]),
    "lsb_synth_stack_host": (C.c_char_p, [C.POINTER(SynthDesc), P, P]),
    "lsb_synth_stack_device": (C.c_char_p, [C.POINTER(SynthDesc), P, P, P]),
    "lsb_unet_create": (ERR, [C.c_int32, C.c_uint64, C.POINTER(P)]),
    "lsb_unet_destroy": (None, [P]),
    "lsb_unet_sizes": (None, [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "lsb_unet_get_params": (ERR, [P, P, P, P, P]),
    "lsb_unet_set_params": (ERR, [P, P, P]),
    "lsb_unet_set_conv": (ERR, [P, C.c_uint32]),
    "lsb_unet_grid": (None, [C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "lsb_unet_prepare": (ERR, [P, P, P, C.c_uint32, C.c_uint32, C.c_float, P, P, C.c_uint32, P]),
    "lsb_unet_forward": (ERR, [P, P, P, C.c_uint32, C.c_uint32, C.c_uint32, P]),
    "lsb_unet_forward_ms": (ERR, [P, P]),
    "lsb_unet_train_step": (ERR, [P, P, P, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.POINTER(C.c_double)]),
    "lsb_stack_set_warm_start": (ERR, [P, P]),
    "lsb_stack_weighted_average": (ERR, [P, C.POINTER(WavParamsC), P]),
    "lsb_stack_set_prep": (ERR, [P, C.POINTER(FramePrepC)]),
    "lsb_stack_push_u16_sized": (ERR, [P, P, C.c_uint32, C.c_uint32]),
    "lsb_prep_frame_u16": (ERR, [P, C.POINTER(FramePrepC), P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, P,
                                 C.POINTER(C.c_uint32)]),
    "lsb_slab_ranges": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_uint32, P, C.c_uint32]),
    "lsb_stack_fuse_range": (ERR, [P, C.c_uint32, C.c_uint32, P, C.c_uint32, C.c_uint32, C.c_uint32, P]),
    "lsb_resize": (ERR, [P, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, P]),
    "lsb_batch_run": (ERR, [C.POINTER(P), C.c_uint32, C.POINTER(Result)]),
    "lsb_stack_autotune": (ERR, [P, C.POINTER(Tuning)]),
    "lsb_stack_depth_planes": (ERR, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(C.c_uint32),
                                     C.POINTER(C.c_uint32)]),
}

_lib = None


def load():
    """Load the in-tree library (build it first with lapstack_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LsbError(f"{LIB_PATH} is missing: build the CUDA engine first (python -m lapstack_b200.build)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if lib.lsb_abi() != ABI_VERSION:
        raise LsbError(f"ABI {lib.lsb_abi()} != {ABI_VERSION}")
    _lib = lib
    return lib


def check(err):
    """Raise the library's error string (and free it)."""
    if err:
        msg = C.cast(err, C.c_char_p).value.decode(errors="replace")
        load().lsb_free_str(err)
        raise LsbError(msg)
