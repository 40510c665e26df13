"""The learned warm start: the U-Net is trained on solver pairs the plain
method makes, then the WLS solves of unseen stacks start from its
prediction. Both starts must reach the solver's relative residual and the
same depth, in about as many iterations, and the learned start must not cost
solve time. The network replaces the FGS sweeps of each solve; since those
run by the partition method they are cheap, and what the learned start gains
at the benchmark's size is reported by bench.py (wls.learned_vs_plain)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_learned_warm_start_reaches_the_same_solution():
    import lapstack_b200 as L
    from lapstack_b200 import unet as U
    eng = L.default_engine()
    inp, d_in, tgt, _ = U.solver_pairs(8, 2048, 1536, frames=(8, 12), engine=eng)
    net = U.UNet(seed=0)
    losses = U.train(net, inp, d_in, tgt, steps=200, batch=8, crop=128, lr=1e-3)
    identity = float(((d_in - tgt) ** 2).mean())
    assert np.mean(losses[-20:]) < identity  # better than taking the raw depth as the solution
    rows = U.compare_warm_start(net, 2048, 1536, 10, seeds=(7001, 7002, 7003), engine=eng)
    ratios = []
    for r in rows:
        p, l = r["plain"], r["learned"]
        assert p["rel"] < 1e-5 and l["rel"] < 1e-5
        assert np.abs(p["depth"] - l["depth"]).max() <= 1e-3 * 9 * 3  # both solve the same system to 1e-5
        assert l["iters"] <= p["iters"] + 2
        ratios.append(p["ms"] / l["ms"])
    print("plain / learned WLS time:", [round(x, 2) for x in ratios])
    assert np.median(ratios) > 0.9
