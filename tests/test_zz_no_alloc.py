"""lsb_warp_cost_noalloc: the registration cost for callers that cannot
allocate device memory (a host running its own Nelder-Mead search over level
planes it already keeps on the GPU, inside a pool or arena it sized up front,
where a cudaMalloc mid-search would synchronise the device or is not allowed
at all). It must give the same costs as lsb_warp_cost, which allocates, and
as the oracle's warp_cost (the CPU restatement of align.rs:581), and keep
doing so on a second call that reuses its fixed device scratch, also when
the reference plane is smaller than the target (the inverse mapping and the
edge clamps then differ from the same-size case).

Named to run last, so a run that stops at the first failure has run every
other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

import lapstack_b200 as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _planes(w, h, seed):
    rng = np.random.default_rng(seed)
    a = rng.random((h, w)).astype(np.float32)
    k = np.array([1, 4, 6, 4, 1], np.float32) / np.float32(16)
    for _ in range(2):  # a little smoothness so the costs vary with the transform
        a = np.apply_along_axis(lambda r: np.convolve(r, k, mode="same"), 1, a).astype(np.float32)
        a = np.apply_along_axis(lambda c: np.convolve(c, k, mode="same"), 0, a).astype(np.float32)
    return np.ascontiguousarray(a)  # row-major, as the device planes are read


def _noalloc(rf_dev, tg_dev, sims, stream):
    lib = L.load()
    s = np.ascontiguousarray(np.asarray(sims, np.float64).reshape(-1, 8))
    out = np.zeros(len(s), np.float64)
    err = lib.lsb_warp_cost_noalloc(C.c_void_p(rf_dev.data_ptr()), rf_dev.shape[1], rf_dev.shape[0], C.c_void_p(tg_dev.data_ptr()),
                                    tg_dev.shape[1], tg_dev.shape[0], C.c_void_p(s.ctypes.data), len(s),
                                    C.c_void_p(out.ctypes.data), C.c_void_p(stream))
    assert err is None, err.decode()
    return out


FIRST = [[0, 0, 1, 0, 1, 0, 0, 0], [0.01, -0.02, 1.01, 0.003, 1, 0, 0, 0], [0.3, 0, 1, 0, 1, 0, 0, 0]]
SECOND = [[-0.005, 0.004, 0.995, -0.002, 1, 0, 0, 0], [0, 0, 1, 0, 1, 0.01, 0.02, -0.01], [2.0, 0, 1, 0, 1, 0, 0, 0],
          [0.02, 0.01, 1.0, 0.0, 1, 0, 0, 0]]


@pytest.mark.parametrize("ref_size", [(200, 150), (120, 90)])
def test_noalloc_cost_matches_the_allocating_entry_point_and_the_oracle_twice(ref_size):
    import torch
    aw, ah = ref_size
    rf, tg = _planes(aw, ah, 1), _planes(200, 150, 2)
    rf_dev, tg_dev = torch.from_numpy(rf).cuda(), torch.from_numpy(tg).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for sims in (FIRST, SECOND):
        got = _noalloc(rf_dev, tg_dev, sims, stream)
        want = np.array([L.warp_cost(rf, tg, s) for s in sims])
        oracle = np.array([O.warp_cost(rf, tg, s) for s in sims])
        assert np.all(np.abs(got - want) <= 1e-12 * np.maximum(want, 1.0)), (got, want)
        assert np.all(np.abs(got - oracle) <= 1e-12 * np.maximum(oracle, 1.0)), (got, oracle)
    assert _noalloc(rf_dev, tg_dev, [[2.0, 0, 1, 0, 1, 0, 0, 0]], stream)[0] == 1e9  # no overlap: the sentinel


def test_noalloc_rejects_too_many_transforms():
    import torch
    lib = L.load()
    a = torch.zeros((16, 16), device="cuda")
    sims = np.tile(np.array([0, 0, 1, 0, 1, 0, 0, 0], np.float64), 10)
    out = np.zeros(10, np.float64)
    err = lib.lsb_warp_cost_noalloc(C.c_void_p(a.data_ptr()), 16, 16, C.c_void_p(a.data_ptr()), 16, 16,
                                    C.c_void_p(sims.ctypes.data), 10, C.c_void_p(out.ctypes.data), None)
    assert err is not None and b"1 to 9" in err
    # sides beyond the other entry points' limits are refused before any launch
    err = lib.lsb_warp_cost_noalloc(C.c_void_p(a.data_ptr()), 70000, 16, C.c_void_p(a.data_ptr()), 16, 16,
                                    C.c_void_p(sims.ctypes.data), 1, C.c_void_p(out.ctypes.data), None)
    assert err is not None and b"65535" in err
