"""Settings and sizes the engine refuses through its real entry points, on a
device: each refusal comes back as an error before any device work, and the
engine stays usable for the next stack."""
import ctypes as C

import numpy as np
import pytest

import lapstack_b200 as L

pytestmark = pytest.mark.gpu


def _msg(lib, err):
    text = C.cast(err, C.c_char_p).value.decode()
    lib.lsb_free_str(err)
    return text


def test_refused_settings_and_sizes_leave_the_engine_usable():
    eng = L.default_engine()
    lib = L.load()
    fp, dp = L.FuseParams().c(), L.DepthParams().c(enabled=False)
    for field, value, text in [("model", 3, "model"), ("interp", 6, "interp")]:
        ap = L.AlignParams().c()
        setattr(ap, field, value)
        hnd = C.c_void_p()
        err = lib.lsb_stack_begin(eng._h, 64, 48, 2, C.byref(fp), C.byref(ap), C.byref(dp), 1, 1, C.byref(hnd))
        assert err and text in _msg(lib, err)
        assert not hnd.value
    with pytest.raises(L.LsbError, match="65535"):
        eng.stack(70000, 2, 2)
    with pytest.raises(L.LsbError, match="agg_radius"):
        eng.stack(64, 48, 2, depth=L.DepthParams(agg_radius=20))
    plane = np.zeros((1, 70000), np.float32)
    with pytest.raises(L.LsbError, match="65535"):
        L.wls_solve(plane, plane, plane, 3.0, 0.04, engine=eng)
    small = np.zeros((8, 8), np.float32)
    with pytest.raises(L.LsbError, match="edge_mode"):
        L.wls_solve(small, small, small, 3.0, 0.04, edge_mode=2, engine=eng)
    # the engine still runs a stack
    frames, _ = L.synth_stack(L.SynthSpec(96, 64, 3, seed=11))
    st = eng.stack(96, 64, 3, L.FuseParams(), None, None)
    for f in frames:
        st.push_u16(f)
    out = st.finish()
    assert out.image_u16.shape == (64, 96, 3)
