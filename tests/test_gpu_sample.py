"""Sampler beyond the trilinear value (math/sample.rs:493-649): cubic B-spline
value, gradient and Hessian (math/bspline.rs:4-32) and the trilinear gradient
on the device, bit-exact against the oracle's restatement of the same f32
operation order, and the difftest_interp goldens of every column within the
reference's tolerance (1e-4)."""
import numpy as np
import pytest

from test_gpu_grid import random_sparse

pytestmark = pytest.mark.gpu


def interp_grid(msbg):
    from fields import interp_field
    g = msbg.HostGrid("interp", 48, 48, 48, 0.0, 1.0, 16)
    zz, yy, xx = np.meshgrid(np.arange(48), np.arange(48), np.arange(48), indexing="ij")
    dense = interp_field(xx, yy, zz)
    for bid in range(g.n_blocks):
        bx, by, bz = g.get_block_coords_by_id(bid)
        g.ensure_block(bid)
        g.blocks[bid][:] = dense[bz * 16:(bz + 1) * 16, by * 16:(by + 1) * 16, bx * 16:(bx + 1) * 16].reshape(-1)
    return g


def test_interp_goldens_all_columns(msbg, ctx, oracle, goldens):
    """tests/difftest_interp.rs:65-91 (Corner, Clamp): the 14 columns."""
    G = goldens["interp"]
    host = interp_grid(msbg)
    dev = msbg.SparseGrid.from_host(ctx, host)
    smp = msbg.Sampler(dev, msbg.CORNER, msbg.CLAMP)
    p = np.array(G["positions"], np.float32)
    got = np.concatenate([smp.sample(p)[:, None], smp.gradient(p), smp.sample(p, msbg.CUBIC_BSPLINE)[:, None],
                          smp.gradient(p, msbg.CUBIC_BSPLINE), smp.hessian(p)], axis=1)
    np.testing.assert_allclose(got, np.array(G["golden"], np.float32), atol=G["tol"], rtol=0)
    for mode in range(4):
        assert np.array_equal(dev.sample_ext(p, mode, 0, msbg.CLAMP), oracle.sample_ext(host, p, mode, msbg.CLAMP, 0))


@pytest.mark.parametrize("bsx", [16, 8])
@pytest.mark.parametrize("bc", [0, 1, 2])
def test_sample_ext_bit_exact(msbg, ctx, oracle, bsx, bc):
    """Sparse grid with absent blocks (empty value), full dummies and partial
    trailing blocks; positions inside, on block seams, on cell centres and
    outside the domain."""
    host = random_sparse(msbg, 40, 36, 44, bsx, 0.6, seed=bsx + bc)
    dev = msbg.SparseGrid.from_host(ctx, host)
    r = np.random.default_rng(50 + bc)
    p = np.concatenate([r.uniform(-3, 47, (4000, 3)),
                        r.integers(0, 44, (300, 3)) + 0.5,
                        r.integers(0, 44, (300, 3)).astype(np.float64)]).astype(np.float32)
    for mode in range(4):
        for align in ((0, 1) if mode == 3 else (0,)):
            got = dev.sample_ext(p, mode, align, bc)
            want = oracle.sample_ext(host, p, mode, bc, align)
            assert np.array_equal(got, want), (mode, align)


@pytest.mark.parametrize("dtype", ["u16", "bf16", "u8", "f16"])
def test_sampler_reads_every_storage_type(msbg, ctx, oracle, dtype):
    """Sampler over quantised storage: every sample is read through Dequant
    (math/sample.rs:45-70; Density8 linearly), so the device equals the oracle
    on the dequantised f32 grid."""
    from test_gpu_grid import dequantized
    host = random_sparse(msbg, 40, 36, 44, 8, 0.6, seed=9, dtype=dtype)
    dev = msbg.SparseGrid.from_host(ctx, host)
    fhost = dequantized(host)
    r = np.random.default_rng(4)
    p = np.concatenate([r.uniform(-3, 47, (3000, 3)), r.integers(0, 44, (200, 3)) + 0.5]).astype(np.float32)
    for mode in range(4):
        assert np.array_equal(dev.sample_ext(p, mode, 0, msbg.NEUMANN), oracle.sample_ext(fhost, p, mode, msbg.NEUMANN, 0))
    smp = msbg.Sampler(dev, msbg.CELL_CENTERED, msbg.CLAMP)
    fdev = msbg.SparseGrid.from_host(ctx, fhost)
    assert np.array_equal(smp.sample(p), msbg.Sampler(fdev, msbg.CELL_CENTERED, msbg.CLAMP).sample(p))
