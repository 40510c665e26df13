"""lapstack-b200: the stacking-engine hot path of ragtux/LAPSTACK on B200.

The compute is hand-written CUDA for sm_100a in liblapstack_b200.so (C ABI in
include/lapstack_b200.h); this package is its host-side binding, mirroring
lapstack-core's interface (see engine.py).
"""
from ._lib import LIB_PATH, LsbError, load  # noqa: F401
from .engine import (AlignParams, DepthMap, DepthParams, DustMap, DustSpot, Engine, FramePrep, FuseParams, GpuFuser, Output, Stack, SynthSpec,  # noqa: F401
                     batch_run, check_params, default_engine, depth_from_slices, multiscale_align, synth_stack,
                     synth_stack_device, slab_ranges, warp_cost, wls_solve, WavParams)
from .unet import UNet  # noqa: F401,E402
