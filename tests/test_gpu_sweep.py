"""The fused halo + stencil 8-colour sweep on the GPU against the reference's
golden vectors and, bit for bit, against the CPU oracle (solver.rs:141-267,
laplacian.rs, meancurv.rs, bilaplacian.rs).  Equality is exact: the kernel
reproduces the reference's f32 operation order (no contraction, fmaf at the
mul_add sites, IEEE sqrt and division)."""
import numpy as np
import pytest

from fields import dense_grid, smoother_field, stencil_field
from test_gpu_grid import dequantized, random_sparse

pytestmark = pytest.mark.gpu


def run_device(msbg, ctx, host, active, stencil, dt, iters, clamp):
    dev = msbg.SparseGrid.from_host(ctx, host)
    msbg.Sweeper(dev).sweep(active, stencil, msbg.PdeParams(dt, iters, clamp))
    ctx.synchronize()
    return dev


def assert_same_blocks(dev, host, ids):
    got = dev.read_blocks(ids)
    for k, b in enumerate(ids):
        want = host.block_array(int(b))
        if not np.array_equal(got[k], want):
            bad = np.nonzero(got[k] != want)[0]
            raise AssertionError(f"block {b}: {len(bad)} voxels differ, first {bad[:5]}: "
                                 f"{got[k][bad[:5]]} vs {want[bad[:5]]}")


def test_stencil_goldens_on_gpu(msbg, ctx, oracle, goldens):
    """tests/difftest_stencil.rs: one application on block 21 == a one-block sweep."""
    G = goldens["stencil"]
    for st, name in enumerate(["laplacian", "mean_curvature", "bilaplacian"]):
        host = dense_grid(msbg.HostGrid, 64, stencil_field)
        dev = run_device(msbg, ctx, host, [21], st, G["dt"], 1, False)
        got = dev.read_blocks([21])[0]
        np.testing.assert_allclose(got[G["sample_idx"]], G["golden"][name], atol=G["tol"], rtol=0, err_msg=name)
        oracle.sweep(host, [21], st, G["dt"], 1, False)
        assert_same_blocks(dev, host, [21])


def test_smoother_goldens_on_gpu(msbg, ctx, oracle, goldens):
    """tests/difftest_smoother.rs: 4 full sweeps of a 64^3 field."""
    G = goldens["smoother"]
    for st, name in [(0, "laplacian"), (1, "mean_curvature")]:
        host = dense_grid(msbg.HostGrid, 64, smoother_field)
        dev = run_device(msbg, ctx, host, np.arange(64), st, G["dt"], G["iterations"], False)
        flat = dev.read_blocks(np.arange(64)).reshape(-1)
        np.testing.assert_allclose(flat[G["sample_idx"]], G["golden"][name], atol=G["tol"][name], rtol=0)
        oracle.sweep(host, np.arange(64), st, G["dt"], G["iterations"], False)
        assert_same_blocks(dev, host, np.arange(64))


SWEEP_CASES = [
    # sx, sy, sz, bsx, frac, iterations
    (64, 64, 64, 16, 0.55, 3),
    (40, 33, 17, 8, 0.7, 2),
    (24, 24, 24, 4, 0.6, 2),
]


def test_sweep_laplacian_large_active_set(msbg, ctx, oracle):
    """The 7-tap stencil on more than 16,384 active blocks runs a kernel per
    colour phase (smaller sets run every phase in one launch): bit-exact
    against the oracle, on a domain whose last block layer is partial."""
    host = random_sparse(msbg, 260, 256, 256, 8, 0.55, 31, empty=0.1, full=0.9)
    active = sorted(host.blocks)
    assert len(active) > 16384
    dev = run_device(msbg, ctx, host, active, 0, 0.05, 2, False)
    oracle.sweep(host, active, 0, 0.05, 2, False)
    ids = np.array(active)[np.random.default_rng(2).choice(len(active), 2000, replace=False)]
    assert_same_blocks(dev, host, np.sort(ids))


@pytest.mark.parametrize("case", SWEEP_CASES)
@pytest.mark.parametrize("stencil", [0, 1, 2])
@pytest.mark.parametrize("clamp", [False, True])
def test_sweep_matches_oracle_f32(msbg, ctx, oracle, case, stencil, clamp):
    sx, sy, sz, bsx, frac, iters = case
    host = random_sparse(msbg, sx, sy, sz, bsx, frac, 5 + stencil, empty=0.1, full=0.9)
    r = np.random.default_rng(9)
    # value blocks, full dummies and absent blocks, each listed once
    extra = [int(b) for b in r.integers(0, host.n_blocks, 6) if int(b) not in host.blocks]
    active = sorted(set(list(host.blocks) + list(host.full) + extra))
    active = [int(b) for b in r.permutation(active)]
    dt = 0.05 if stencil != 2 else 0.01
    dev = run_device(msbg, ctx, host, active, stencil, dt, iters, clamp)
    oracle.sweep(host, active, stencil, dt, iters, clamp)
    assert_same_blocks(dev, host, np.arange(host.n_blocks))


@pytest.mark.parametrize("dtype", ["u16", "bf16", "f16"])
@pytest.mark.parametrize("stencil", [0, 1, 2])
def test_sweep_matches_oracle_quantized(msbg, ctx, oracle, dtype, stencil):
    """Density (u16, round half away), bf16 and binary16 storage: dequantise
    on gather, quantise on store (stencil.rs:142-192)."""
    host = random_sparse(msbg, 48, 48, 48, 16, 0.6, 21, empty=0.1, full=0.9, dtype=dtype)
    if dtype == "u16":
        for b in host.blocks:
            host.blocks[b][:] = np.random.default_rng(b).integers(0, 65536, host.N)
    active = list(host.blocks)
    dev = run_device(msbg, ctx, host, active, stencil, 0.05, 2, True)
    oracle.sweep(host, active, stencil, 0.05, 2, True)
    assert_same_blocks(dev, host, np.arange(host.n_blocks))


DENSITY8_CASES = [
    # sx, bsx, frac, lanes, stencil, clamp
    (48, 16, 0.6, 16, 0, True),
    (48, 16, 0.6, 8, 1, True),
    (48, 16, 0.6, 16, 2, True),
    (48, 16, 0.6, 16, 0, False),  # out-of-range results take the wrapping u8 cast
    (40, 8, 0.7, 8, 1, True),
    (20, 4, 0.7, 4, 2, True),
]


@pytest.mark.parametrize("case", DENSITY8_CASES)
def test_sweep_density8_stochastic(msbg, ctx, oracle, case):
    """Density8 storage: linear read, sqrt-compressed stochastic store
    (stencil.rs:103-132, 176-192), bit for bit against the oracle's serial
    one-thread generator stream, including a second call that continues the
    stream."""
    sx, bsx, frac, lanes, stencil, clamp = case
    host = random_sparse(msbg, sx, sx, sx, bsx, frac, 5 + bsx, empty=0.1, full=0.9, dtype="u8")
    active = list(host.blocks)
    dev = msbg.SparseGrid.from_host(ctx, host)
    sw = msbg.Sweeper(dev, seed=0x2468ACE1, lanes=lanes)
    sw.sweep(active, stencil, msbg.PdeParams(0.05, 2, clamp))
    pos = oracle.sweep_stochastic(host, active, stencil, 0.05, 2, clamp, 0x2468ACE1, lanes, 0)
    assert sw.stream_pos == pos == 2 * len(active) * host.N // lanes
    assert_same_blocks(dev, host, np.arange(host.n_blocks))
    sw.sweep(active, stencil, msbg.PdeParams(0.05, 1, clamp))
    pos = oracle.sweep_stochastic(host, active, stencil, 0.05, 1, clamp, 0x2468ACE1, lanes, pos)
    assert sw.stream_pos == pos
    assert_same_blocks(dev, host, np.arange(host.n_blocks))


def test_sweep_density8_plain_entry_is_a_fresh_sweeper(msbg, ctx, oracle):
    """msbg_sweep on Density8 storage: apply_pde's fresh sweeper, the first
    rayon slot's generator (seed 0xdeadbeef, 16 lanes, solver.rs:109-119)."""
    from msbg_rs_b200._lib import call, ptr
    host = random_sparse(msbg, 48, 48, 48, 16, 0.5, 77, empty=0.0, full=1.0, dtype="u8")
    active = np.array(sorted(host.blocks), np.uint64)
    dev = msbg.SparseGrid.from_host(ctx, host)
    for _ in range(2):  # each call starts the stream again
        call("msbg_sweep", dev.handle, ptr(active), len(active), 1, 0.05, 1, 1)
        oracle.sweep_stochastic(host, active.astype(np.int64), 1, 0.05, 1, True, 0xDEADBEEF, 16, 0)
    assert_same_blocks(dev, host, np.arange(host.n_blocks))


def shell_blocks(n_per_axis, bsx, radius, thickness):
    """Blocks whose AABB meets the shell | |x - c| - r | <= t / 2."""
    c = n_per_axis * bsx / 2.0
    b = np.arange(n_per_axis)
    bz, by, bx = np.meshgrid(b, b, b, indexing="ij")
    lo = np.stack([bx, by, bz], -1) * bsx
    hi = lo + bsx
    near = np.clip(c, lo, hi)
    dmin = np.linalg.norm(near - c, axis=-1)
    far = np.maximum(np.abs(lo - c), np.abs(hi - c))
    dmax = np.linalg.norm(far, axis=-1)
    hit = (dmin <= radius + thickness / 2) & (dmax >= radius - thickness / 2)
    return np.nonzero(hit.reshape(-1))[0]


def test_config1_shell_laplacian_bit_exact(msbg, ctx, oracle):
    """128^3, 16^3 blocks, shell r = 44.8, t = 12 (272 blocks), U[-1,1], 10 sweeps."""
    active = shell_blocks(8, 16, 44.8, 12.0)
    assert len(active) == 272
    host = msbg.HostGrid("shell", 128, 128, 128, 0.0, 1.0, 16)
    r = np.random.default_rng(1)
    for b in active:
        host.ensure_block(int(b))
        host.blocks[int(b)][:] = r.uniform(-1, 1, 4096).astype(np.float32)
    dev = run_device(msbg, ctx, host, active, 0, 0.025, 10, False)
    oracle.sweep(host, active, 0, 0.025, 10, False, threads=oracle.num_threads())
    assert_same_blocks(dev, host, active)


def test_sweep_duplicate_ids_swept_once(msbg, ctx, oracle):
    """A block listed twice is swept once per colour phase (in the reference
    two threads would update it concurrently)."""
    host = random_sparse(msbg, 64, 64, 64, 16, 0.5, 8)
    ids = list(host.blocks)
    dev = run_device(msbg, ctx, host, ids + ids[:5], 0, 0.05, 2, False)
    oracle.sweep(host, ids, 0, 0.05, 2, False)
    assert_same_blocks(dev, host, np.arange(64))


def test_sweep_deterministic_and_empty(msbg, ctx):
    host = random_sparse(msbg, 64, 64, 64, 16, 0.5, 3)
    a = run_device(msbg, ctx, host, list(host.blocks), 1, 0.05, 3, False).read_blocks(np.arange(64))
    b = run_device(msbg, ctx, host, list(host.blocks), 1, 0.05, 3, False).read_blocks(np.arange(64))
    assert np.array_equal(a, b)
    dev = msbg.SparseGrid.from_host(ctx, host)
    before = dev.read_blocks(np.arange(64))
    msbg.Sweeper(dev).sweep([], 0, msbg.PdeParams(0.05, 2, True))  # solver.rs:434-440
    ctx.synchronize()
    assert np.array_equal(dev.read_blocks(np.arange(64)), before)


def test_multires_sweep_matches_oracle(msbg, ctx, oracle):
    """fill_multires halos (multires/halo.rs:187-358): coarser neighbours are
    sampled from the coarse level at >> 1."""
    n = 4
    fine = msbg.HostGrid("fine", 64, 64, 64, 0.0, 0.0, 16)
    coarse = msbg.HostGrid("coarse", 32, 32, 32, 0.0, 0.0, 8)
    r = np.random.default_rng(4)
    levels = (r.random(n ** 3) < 0.4).astype(np.uint8)
    for b in range(n ** 3):
        if levels[b] == 0:
            fine.ensure_block(b)
            fine.blocks[b][:] = r.uniform(0, 1, 4096)
        else:
            coarse.ensure_block(b)
            coarse.blocks[b][:] = r.uniform(0, 1, 512)
    active = [b for b in range(n ** 3) if levels[b] == 0]
    dfine = msbg.SparseGrid.from_host(ctx, fine)
    dcoarse = msbg.SparseGrid.from_host(ctx, coarse)
    msbg.Sweeper(dfine).sweep_multires(dcoarse, levels, active, 1, msbg.PdeParams(0.05, 2, False))
    ctx.synchronize()
    oracle.sweep_multires(fine, coarse, levels, active, 1, 0.05, 2, False)
    assert_same_blocks(dfine, fine, active)
