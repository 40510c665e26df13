"""The committed golden fixtures (tests/golden/make_golden.py): the oracle's
results on small seeded stacks. CPU: the generator and the oracle still
reproduce them exactly. GPU: the CUDA path through the C ABI against them --
fused u16 image, winner map, gains and shares bit-exact, transforms to 1e-9,
the depth map within 1e-3 of the frame range on all but 0.1 % of pixels."""
import hashlib

import numpy as np
import pytest

from tests.golden import make_golden as G

CASES = sorted(G.CASES)


def load(case):
    return np.load(G.os.path.join(G.HERE, f"{case}.npz"))


@pytest.mark.parametrize("case", CASES)
def test_oracle_reproduces_golden(case):
    from oracle import oracle as O
    g = load(case)
    fr = G.inputs(case)
    assert hashlib.sha256(np.ascontiguousarray(fr).tobytes()).hexdigest() == str(g["input_sha256"])
    fp, ap, dp = G.params(case, O)
    r = O.run_stack(fr, O.StackParams(fuse=fp, align=ap, depth=dp))
    assert np.array_equal(r.image_u16, g["image_u16"])
    assert np.array_equal(r.winner, g["winner"])
    assert np.array_equal(r.sims, g["sims"]) and np.array_equal(r.gains, g["gains"])
    if "depth" in g:
        assert np.array_equal(r.depth.astype(np.float32), g["depth"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_cuda_path_matches_golden(case):
    import lapstack_b200 as L
    g = load(case)
    fr = G.inputs(case)
    fp, ap, dp = G.params(case, L)
    n, h, w, _ = fr.shape
    st = L.default_engine().stack(w, h, n, fp, ap, dp)
    for f in fr:
        st.push_u16(f)
    out = st.finish()
    assert np.array_equal(out.image_u16, g["image_u16"])
    assert np.array_equal(out.winner, g["winner"])
    assert np.array_equal(out.gains, g["gains"]) and np.array_equal(out.shares, g["shares"])
    assert np.max(np.abs(out.align - g["sims"])) < 1e-9
    assert tuple(out.crop) == tuple(g["crop"])
    if "depth" in g:
        d = np.abs(out.depth.depth.astype(np.float64) - g["depth"].astype(np.float64))
        assert np.mean(d > 1e-3 * (n - 1)) <= 1e-3, d.max()
