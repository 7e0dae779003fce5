"""The learned preconditioner's network on the device against the numpy
oracle (oracle/unet.py), which stores the same values in bf16 and computes
the rest in FP64.  The device accumulates in f32, so a stored bf16 value can
round the other way now and then; comparisons are therefore relative in
norm: forward output within 1e-2, loss within 1e-2, and every layer's weight
and bias gradient within 5e-2 of the oracle's (relative L2)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))


def setup(msbg, ctx, seed=0, n_axis=3, n_active=9):
    import unet

    rng = np.random.default_rng(seed)
    act = np.sort(rng.choice(n_axis ** 3, n_active, replace=False)).astype(np.uint64)
    size = 16 * n_axis
    net = msbg.UNet(ctx, size, size, size, act, seed=seed + 1)
    nbr = unet.nbr27(act.astype(np.int64), n_axis)
    return unet, net, act, nbr, rng


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


def test_layer_table_matches_oracle(msbg, ctx):
    unet, net, act, nbr, rng = setup(msbg, ctx)
    offs, n = unet.param_offsets()
    assert net.n_params == n
    t = net.layers()
    for i, (lv, ci, co, cir, cor, relu) in enumerate(unet.LAYERS):
        assert tuple(t[i][:6]) == (lv, ci, co, cir, cor, int(relu))
        assert tuple(t[i][6:]) == offs[i]


def test_forward_matches_oracle(msbg, ctx):
    import torch
    unet, net, act, nbr, rng = setup(msbg, ctx, seed=3)
    r = rng.standard_normal(net.n).astype(np.float32)
    d_r = torch.from_numpy(r).cuda()
    y = torch.empty(net.n, device="cuda")
    net.forward_raw(d_r, y)
    ref = unet.UNet(nbr, net.params()).forward(r)
    assert rel(y.cpu().numpy(), ref) < 1e-2


def test_gradients_match_oracle(msbg, ctx):
    import torch
    unet, net, act, nbr, rng = setup(msbg, ctx, seed=5)
    net.set_output_scale(2.0)
    r = rng.standard_normal(net.n).astype(np.float32)
    e = rng.standard_normal(net.n).astype(np.float32)
    d_r, d_e = torch.from_numpy(r).cuda(), torch.from_numpy(e).cuda()
    loss = net.train_step(d_r, d_e, lr=0.0, update=False)
    g = net.grads()
    lo, go = unet.UNet(nbr, net.params(), out_scale=2.0).grads(r, e)
    assert abs(loss - lo) <= 1e-2 * lo
    offs, _ = unet.param_offsets()
    for i, (lv, ci, co, cir, cor, _) in enumerate(unet.LAYERS):
        o, ob = offs[i]
        assert rel(g[o:ob], go[o:ob]) < 5e-2, (i, rel(g[o:ob], go[o:ob]))
        assert rel(g[ob:ob + co], go[ob:ob + co]) < 5e-2, (i, "bias")
        # padded channels carry no gradient
        gw = g[o:ob].reshape(27, co, ci)
        assert not np.any(gw[:, cor:, :]) and not np.any(gw[:, :, cir:])


def test_training_reduces_loss_and_keeps_padding(msbg, ctx):
    import torch
    unet, net, act, nbr, rng = setup(msbg, ctx, seed=7)
    r = rng.standard_normal(net.n).astype(np.float32)
    e = (0.5 * r + 0.1 * rng.standard_normal(net.n)).astype(np.float32)
    d_r, d_e = torch.from_numpy(r).cuda(), torch.from_numpy(e).cuda()
    first = net.train_step(d_r, d_e, lr=1e-3)
    for _ in range(60):
        last = net.train_step(d_r, d_e, lr=1e-3)
    assert last < 0.5 * first, (first, last)
    p = net.params()
    offs, _ = unet.param_offsets()
    for i, (lv, ci, co, cir, cor, _) in enumerate(unet.LAYERS):
        o, ob = offs[i]
        w = p[o:ob].reshape(27, co, ci)
        assert not np.any(w[:, cor:, :]) and not np.any(w[:, :, cir:])
        assert not np.any(p[ob + cor:ob + co])


@pytest.mark.parametrize("n_axis,n_active", [(1, 1), (2, 3)])
def test_tiny_networks_match_oracle(msbg, ctx, n_axis, n_active):
    """One and three blocks: every level's last tensor-core tile is partial
    (a single 16^3 block has 64 level-2 cells, half a 128-cell tile)."""
    import torch
    unet, net, act, nbr, rng = setup(msbg, ctx, seed=11 + n_active, n_axis=n_axis, n_active=n_active)
    net.set_output_scale(0.5)
    r = rng.standard_normal(net.n).astype(np.float32)
    e = rng.standard_normal(net.n).astype(np.float32)
    d_r, d_e = torch.from_numpy(r).cuda(), torch.from_numpy(e).cuda()
    y = torch.empty(net.n, device="cuda")
    net.forward_raw(d_r, y)
    o = unet.UNet(nbr, net.params(), out_scale=0.5)
    assert rel(y.cpu().numpy(), o.forward(r)) < 1e-2
    net.train_step(d_r, d_e, lr=0.0, update=False)
    g = net.grads()
    _, go = o.grads(r, e)
    assert rel(g, go) < 5e-2
