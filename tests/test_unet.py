"""The learned warm start's network: the numpy oracle's backward pass against
finite differences, its layer table and grid rule (CPU), and the library's forward, backward and training
kernels against the oracle on the same parameters and inputs (GPU)."""
import numpy as np
import pytest

from oracle import unet_ref as U


def _case(seed, B=1, H=8, W=8):
    rng = np.random.default_rng(seed)
    inp = np.zeros((B, H, W, 32), np.float32)
    inp[..., :3] = rng.random((B, H, W, 3), dtype=np.float32)
    d_in = rng.random((B, H, W), dtype=np.float32)
    tgt = np.clip(d_in + 0.1 * rng.standard_normal((B, H, W)).astype(np.float32), 0, 1).astype(np.float32)
    return U.bf16(inp), d_in, tgt


def test_oracle_backward_matches_finite_differences():
    w, b = U.init_params(1)
    w, b = w.astype(np.float64), b.astype(np.float64)
    inp, d_in, tgt = _case(0)
    inp, d_in, tgt = inp.astype(np.float64), d_in.astype(np.float64), tgt.astype(np.float64)
    act, out0 = U.forward(inp, w, b, bf16_round=False)
    _, gw, gb = U.backward(act, out0, d_in, tgt, w, bf16_round=False)

    def loss(wv, bv):
        _, o = U.forward(inp, wv, bv, bf16_round=False)
        e = d_in + o - tgt
        return float(np.mean(e * e))

    rng = np.random.default_rng(2)
    offs, _, _ = U.offsets()
    checked = 0
    for i, (wo, bo) in enumerate(offs):
        c1, c2, co = U.LAYERS[i][2], U.LAYERS[i][5], U.LAYERS[i][6]
        n = 9 * co * (c1 + c2)
        live = np.flatnonzero(np.abs(gw[wo:wo + n]) > 0)
        for k in rng.choice(live, size=min(3, live.size), replace=False):
            eps = 1e-6
            wp, wm = w.copy(), w.copy()
            wp[wo + k] += eps
            wm[wo + k] -= eps
            fd = (loss(wp, b) - loss(wm, b)) / (2 * eps)
            assert abs(fd - gw[wo + k]) <= 1e-4 * abs(fd) + 1e-9, (i, k, fd, gw[wo + k])
            checked += 1
        j = bo + int(rng.integers(0, 1 if i == len(offs) - 1 else co))
        bp, bm = b.copy(), b.copy()
        bp[j] += 1e-6
        bm[j] -= 1e-6
        fd = (loss(w, bp) - loss(w, bm)) / 2e-6
        assert abs(fd - gb[j]) <= 1e-4 * abs(fd) + 1e-9, (i, j, fd, gb[j])
    assert checked >= 40


def _to_gpu(inp, d_in, tgt):
    import torch
    t_in = torch.from_numpy(inp).to(torch.bfloat16).cuda()  # exact: inp is bf16-representable
    return t_in, torch.from_numpy(d_in).cuda(), torch.from_numpy(tgt).cuda()


def test_flops_table_is_the_oracle_architecture():
    """The convolution table behind the bench's U-Net FLOP count describes the oracle's network."""
    from lapstack_b200 import unet as N
    assert N.CONVS == [(c1 + c2, co, lv) for (_, _, c1, _, _, c2, co, lv, _) in U.LAYERS]
    _, nw, _ = U.offsets()
    assert nw == 9 * sum(ci * co for ci, co, _ in N.CONVS)
    H, W = 64, 96
    assert N.forward_flops(H, W, B=2) == 2 * 9 * sum(ci * co * 2 * (H >> lv) * (W >> lv) for ci, co, lv in N.CONVS)


def test_network_grid_is_half_the_depth_grid_in_multiples_of_8():
    from lapstack_b200 import unet as N
    for dw, dh in [(1, 1), (15, 9), (16, 16), (17, 33), (4128, 2752), (4127, 2751)]:
        H, W = N.grid_of(dw, dh)
        hw, hh = (dw + 1) // 2, (dh + 1) // 2
        assert W % 8 == 0 and H % 8 == 0  # three 2x2 poolings
        assert hw <= W < hw + 8 and hh <= H < hh + 8


@pytest.mark.gpu
def test_network_size_matches_oracle():
    import lapstack_b200 as L
    net = L.UNet(seed=3)
    _, nw, nb = U.offsets()
    assert (net.n_weights, net.n_biases) == (nw, nb)
    w, b = net.params()
    _, _, _ = w, b, net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(1, 8, 8), (2, 16, 24)])
def test_forward_matches_oracle(shape):
    import lapstack_b200 as L
    B, H, W = shape
    w, b = U.init_params(5)
    inp, d_in, tgt = _case(7, B, H, W)
    net = L.UNet(seed=0)
    net.set_params(w, b)
    out = net.forward(*_to_gpu(inp, d_in, tgt)[:2]).cpu().numpy()
    _, ref = U.forward(inp, w, b)
    scale = max(float(np.abs(ref).max()), 1e-3)
    assert np.abs(out - ref).max() <= 2e-2 * scale, (np.abs(out - ref).max(), scale)
    assert np.corrcoef(out.ravel(), ref.ravel())[0, 1] > 0.999


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(1, 8, 8), (2, 16, 16)])
def test_gradients_match_oracle(shape):
    import lapstack_b200 as L
    B, H, W = shape
    w, b = U.init_params(11)
    inp, d_in, tgt = _case(13, B, H, W)
    net = L.UNet(seed=0)
    net.set_params(w, b)
    loss = net.train_step(*_to_gpu(inp, d_in, tgt), lr=0.0)
    gw, gb = net.grads()
    act, out0 = U.forward(inp, w, b)
    rloss, rgw, rgb = U.backward(act, out0, d_in, tgt, w)
    assert abs(loss - rloss) <= 1e-3 * rloss
    offs, _, _ = U.offsets()
    for i, (wo, bo) in enumerate(offs):
        c1, c2, co = U.LAYERS[i][2], U.LAYERS[i][5], U.LAYERS[i][6]
        n = 9 * co * (c1 + c2)
        g, r = gw[wo:wo + n], rgw[wo:wo + n]
        scale = max(float(np.abs(r).max()), 1e-12)
        rel = float(np.linalg.norm(g - r) / max(np.linalg.norm(r), 1e-30))
        assert np.abs(g - r).max() <= 3e-2 * scale and rel <= 2e-2, (i, np.abs(g - r).max(), scale, rel)
        gbb, rbb = gb[bo:bo + co], rgb[bo:bo + co]
        assert np.abs(gbb - rbb).max() <= 3e-2 * max(float(np.abs(rbb).max()), 1e-12), (i, gbb[:4], rbb[:4])


@pytest.mark.gpu
def test_training_fits_a_fixed_batch():
    """Adam on the library's gradients learns a correction that depends on the guide channel."""
    import lapstack_b200 as L
    inp, d_in, _ = _case(21, 4, 32, 32)
    tgt = (d_in + 0.2 * (inp[..., 0] - 0.5)).astype(np.float32)
    net = L.UNet(seed=4)
    t = _to_gpu(inp, d_in, tgt)
    first = net.train_step(*t, lr=0.0)
    for _ in range(150):
        last = net.train_step(*t, lr=2e-3)
    assert last < 0.2 * first, (first, last)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(1, 8, 8), (2, 40, 56), (1, 64, 128)])
def test_tcgen05_convolutions_match_the_mma_sync_path(shape):
    """The 3x3 convolutions on tcgen05 (TMEM accumulators, the default) against the mma.sync path on the
    same parameters and inputs: the same bf16 products summed in another order, so the forward output
    agrees to bf16 rounding (partial 16 x 8 tiles at every level of the shapes here) and the gradients
    of one step too; both are held to the oracle as above."""
    import lapstack_b200 as L
    B, H, W = shape
    w, b = U.init_params(17)
    inp, d_in, tgt = _case(19, B, H, W)
    outs, grads = {}, {}
    for path in ("tcgen05", "mma.sync"):
        net = L.UNet(seed=0)
        net.set_conv(path)
        net.set_params(w, b)
        t = _to_gpu(inp, d_in, tgt)
        outs[path] = net.forward(*t[:2]).cpu().numpy()
        net.train_step(*t, lr=0.0)
        grads[path] = net.grads()[0]
        net.close()
    a, m = outs["tcgen05"], outs["mma.sync"]
    scale = max(float(np.abs(m).max()), 1e-3)
    assert np.abs(a - m).max() <= 1e-2 * scale, (np.abs(a - m).max(), scale)
    assert np.corrcoef(a.ravel(), m.ravel())[0, 1] > 0.9999
    ga, gm = grads["tcgen05"], grads["mma.sync"]
    assert np.linalg.norm(ga - gm) <= 2e-2 * np.linalg.norm(gm)
    _, ref = U.forward(inp, w, b)
    assert np.abs(a - ref).max() <= 2e-2 * max(float(np.abs(ref).max()), 1e-3)
