"""Block-sparse 3x3x3 convolution on the tensor cores against the FP64 oracle
(oracle/unet.py).  Inputs and weights are bf16 values; the kernels multiply
them exactly and accumulate in FP32, so the forward result and the weight
gradient must agree with the FP64 sums within FP32 accumulation error:
|gpu - ref| <= 1e-5 * sum|terms| + 1e-30 elementwise."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    # (domain blocks per axis, lg, active fraction, cin, cout)
    (6, 3, 0.6, 16, 32),
    (6, 3, 0.6, 32, 16),
    (5, 3, 0.5, 32, 32),
    (8, 2, 0.55, 32, 64),
    (8, 2, 0.55, 64, 64),
    (7, 2, 0.5, 64, 32),
    (4, 4, 0.7, 16, 16),
    (4, 3, 0.6, 32, 64),
    (4, 3, 0.6, 64, 16),
    (4, 3, 0.7, 16, 64),
    (4, 3, 0.6, 64, 32),
]


def level(nb, lg, frac, seed):
    import sys
    import os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    import unet

    rng = np.random.default_rng(seed)
    n_all = nb ** 3
    act = np.sort(rng.choice(n_all, max(1, int(frac * n_all)), replace=False)).astype(np.int64)
    nbr = unet.nbr27(act, nb)
    taps = unet.tap_index(nbr, lg)
    return unet, act, nbr, taps


def dev_bits(bits):
    import torch
    return torch.from_numpy(np.ascontiguousarray(bits).view(np.int16)).cuda()


@pytest.mark.parametrize("nb,lg,frac,cin,cout", CASES)
def test_conv3_forward_matches_oracle(msbg, ctx, nb, lg, frac, cin, cout):
    import torch
    unet, act, nbr, taps = level(nb, lg, frac, seed=cin * 7 + cout)
    cells = len(act) << (3 * lg)
    rng = np.random.default_rng(1)
    xb = unet.bf16_bits(rng.standard_normal((cells, cin)).astype(np.float32))
    wb = unet.bf16_bits((rng.standard_normal((27, cout, cin)) / np.sqrt(27 * cin)).astype(np.float32))
    bias = rng.standard_normal(cout).astype(np.float32)
    x, w = unet.bf16_value(xb), unet.bf16_value(wb)
    ref = unet.conv3(x, w, bias, taps)
    absum = unet.conv3(np.abs(x), np.abs(w), np.abs(bias), taps)
    d_nbr = torch.from_numpy(nbr).cuda()
    d_x, d_w = dev_bits(xb), dev_bits(wb)
    d_b = torch.from_numpy(bias).cuda()
    y = torch.empty((cells, cout), dtype=torch.float32, device="cuda")
    ptr = msbg._lib.ptr
    msbg._lib.call("msbg_conv3_forward_device", ctx.handle, ptr(d_nbr), len(act), lg, cin, cout, ptr(d_x), ptr(d_w),
                   ptr(d_b), 0, 1, ptr(y))
    got = y.cpu().numpy().astype(np.float64)
    err = np.abs(got - ref)
    assert np.all(err <= 1e-5 * absum + 1e-30), (err.max(), np.argmax(err / (absum + 1e-30)))
    # ReLU + bf16 output: equal to the rounded f32 result
    yb = torch.empty((cells, cout), dtype=torch.int16, device="cuda")
    msbg._lib.call("msbg_conv3_forward_device", ctx.handle, ptr(d_nbr), len(act), lg, cin, cout, ptr(d_x), ptr(d_w),
                   ptr(d_b), 1, 0, ptr(yb))
    want = unet.bf16_bits(np.maximum(got, 0).astype(np.float32))
    assert np.array_equal(yb.cpu().numpy().view(np.uint16), want)


@pytest.mark.parametrize("nb,lg,frac,cin,cout", CASES)
def test_conv3_wgrad_matches_oracle(msbg, ctx, nb, lg, frac, cin, cout):
    import torch
    unet, act, nbr, taps = level(nb, lg, frac, seed=cin * 5 + cout)
    cells = len(act) << (3 * lg)
    rng = np.random.default_rng(2)
    xb = unet.bf16_bits(rng.standard_normal((cells, cin)).astype(np.float32))
    gb = unet.bf16_bits(rng.standard_normal((cells, cout)).astype(np.float32))
    x, g = unet.bf16_value(xb), unet.bf16_value(gb)
    ref = unet.conv3_wgrad(x, g, taps)
    absum = unet.conv3_wgrad(np.abs(x), np.abs(g), taps)
    d_nbr = torch.from_numpy(nbr).cuda()
    d_x, d_g = dev_bits(xb), dev_bits(gb)  # kept alive across the call
    dw = torch.empty((27, cout, cin), dtype=torch.float32, device="cuda")
    ptr = msbg._lib.ptr
    msbg._lib.call("msbg_conv3_wgrad_device", ctx.handle, ptr(d_nbr), len(act), lg, cin, cout, ptr(d_x), ptr(d_g),
                   ptr(dw))
    got = dw.cpu().numpy().astype(np.float64)
    err = np.abs(got - ref)
    assert np.all(err <= 1e-5 * absum + 1e-30), err.max()


def test_conv3_data_gradient_is_mirrored_forward(msbg, ctx):
    """The data gradient runs as the forward kernel with mirrored, transposed
    weights; check that identity against the oracle's adjoint."""
    import torch
    unet, act, nbr, taps = level(6, 3, 0.6, seed=11)
    cells = len(act) << 9
    rng = np.random.default_rng(3)
    gb = unet.bf16_bits(rng.standard_normal((cells, 32)).astype(np.float32))
    wb = unet.bf16_bits((rng.standard_normal((27, 32, 16)) / 20).astype(np.float32))
    g, w = unet.bf16_value(gb), unet.bf16_value(wb)
    ref = unet.conv3_dgrad(g, w, taps)
    wt = np.ascontiguousarray(np.transpose(wb[::-1], (0, 2, 1)))  # [27][16][32]
    dx = torch.empty((cells, 16), dtype=torch.float32, device="cuda")
    d_nbr, d_g, d_wt = torch.from_numpy(nbr).cuda(), dev_bits(gb), dev_bits(wt)  # kept alive across the call
    ptr = msbg._lib.ptr
    msbg._lib.call("msbg_conv3_forward_device", ctx.handle, ptr(d_nbr), len(act), 3, 32, 16, ptr(d_g), ptr(d_wt), None,
                   0, 1, ptr(dx))
    absum = unet.conv3_dgrad(np.abs(g), np.abs(w), taps)
    assert np.all(np.abs(dx.cpu().numpy() - ref) <= 1e-5 * absum + 1e-30)
