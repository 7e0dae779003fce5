"""Device sparse grid: block transfer, dummies and the halo gather, bit-exact
against the CPU oracle (multires/halo.rs:31-170, sparse_grid.rs)."""
import itertools

import numpy as np
import pytest

from test_oracle_golden import fnv1a, sparse_grid_script

pytestmark = pytest.mark.gpu


def random_sparse(msbg, sx, sy, sz, bsx, frac, seed, n_full=3, empty=0.25, full=0.75, dtype="f32"):
    r = np.random.default_rng(seed)
    g = msbg.HostGrid("r", sx, sy, sz, empty, full, bsx, dtype)
    bids = np.nonzero(r.random(g.n_blocks) < frac)[0]
    for b in bids:
        g.ensure_block(int(b))
        v = r.uniform(-1, 1, g.N).astype(np.float32)
        if dtype == "f32":
            g.blocks[int(b)][:] = v
        elif dtype == "u16":
            g.blocks[int(b)][:] = r.integers(0, 65536, g.N)
        elif dtype == "u8":
            g.blocks[int(b)][:] = r.integers(0, 256, g.N)
        elif dtype == "f16":
            g.blocks[int(b)][:] = v.astype(np.float16).view(np.uint16)
        else:
            g.blocks[int(b)][:] = (v.view(np.uint32) >> 16).astype(np.uint16)
    rest = [b for b in range(g.n_blocks) if b not in g.blocks]
    for b in r.permutation(rest)[:n_full]:
        g.set_full_block(int(b))
    return g


def quantized_value(dtype, v):
    """The float a dummy of value v reads after storage in `dtype`."""
    f = np.float32
    if dtype == "u16":
        q = np.floor(f(v) * f(65535.0) + f(0.5))
        return float(f(min(max(q, 0.0), 65535.0)) * (f(1.0) / f(65535.0)))
    if dtype == "u8":
        q = np.floor(f(v) * f(255.0) + f(0.5))
        return float(f(min(max(q, 0.0), 255.0)) * (f(1.0) / f(255.0)))
    if dtype == "f16":
        return float(np.array([v], f).astype(np.float16).astype(f)[0])
    if dtype == "bf16":
        b = int(np.array([v], f).view(np.uint32)[0])
        b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
        return float(np.array([b], np.uint32).view(f)[0])
    return float(f(v))


def dequantized(host):
    """f32 copy of a u16/bf16 HostGrid as the reference's Dequant sees it."""
    if host.dtype == "f32":
        return host
    g = host.copy()
    g.dtype, g.np_dtype = "f32", np.float32
    for b, v in host.blocks.items():
        if host.dtype == "u16":
            g.blocks[b] = (v.astype(np.float32) * (np.float32(1.0) / np.float32(65535.0))).astype(np.float32)
        elif host.dtype == "u8":
            g.blocks[b] = (v.astype(np.float32) * (np.float32(1.0) / np.float32(255.0))).astype(np.float32)
        elif host.dtype == "f16":
            g.blocks[b] = v.view(np.float16).astype(np.float32)
        else:
            g.blocks[b] = (v.astype(np.uint32) << 16).view(np.float32)
    g.empty_value = quantized_value(host.dtype, host.empty_value)
    g.full_value = quantized_value(host.dtype, host.full_value)
    return g


def test_sparse_grid_hash_through_device(msbg, ctx, goldens):
    """The FNV difftest (tests/difftest_cpp.rs) read back from HBM."""
    host = sparse_grid_script(msbg.HostGrid)
    dev = msbg.SparseGrid.from_host(ctx, host)
    blocks = dev.read_blocks(np.arange(dev.n_blocks))
    h = 0xCBF29CE484222325
    for z in range(5):
        for y in range(33):
            for x in range(17):
                v = blocks[host.get_block_id(x, y, z)][host.get_voxel_id(x, y, z)]
                h = fnv1a(h, np.float32(v).tobytes())
    assert h == int(goldens["sparse_grid_hash"]["hash"], 16)


@pytest.mark.parametrize("dtype", ["f32", "u16", "bf16", "u8", "f16"])
def test_write_read_roundtrip(msbg, ctx, dtype):
    host = random_sparse(msbg, 40, 33, 17, 8, 0.5, 1, dtype=dtype)
    dev = msbg.SparseGrid.from_host(ctx, host)
    ids = np.arange(host.n_blocks)
    got = dev.read_blocks(ids)
    for b in ids:
        assert np.array_equal(got[b], host.block_array(int(b))), b
    assert list(dev.value_block_ids()) == host.value_block_ids()


def test_ensure_fill_and_errors(msbg, ctx):
    dev = msbg.SparseGrid(ctx, 32, 32, 32, 0.5, 1.0, 16)
    dev.ensure_blocks([3, 1, 3])
    assert list(dev.value_block_ids()) == [1, 3]
    assert np.all(dev.read_blocks([1])[0] == 0.5)
    dev.fill_blocks([1, 5], 2.0)
    assert np.all(dev.read_blocks([1])[0] == 2.0) and np.all(dev.read_blocks([5])[0] == 0.5)
    with pytest.raises(msbg.MsbgError):
        dev.ensure_blocks([8])
    with pytest.raises(msbg.MsbgError):
        dev.set_full_blocks([1])


CASES = [
    # sx, sy, sz, bsx, frac
    (64, 64, 64, 16, 0.6),
    (40, 33, 17, 8, 0.7),
    (48, 16, 32, 16, 0.5),
    (20, 20, 20, 4, 0.6),
]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("dtype", ["f32", "u16", "bf16", "u8", "f16"])
def test_halo_gather_matches_oracle(msbg, ctx, oracle, case, dtype):
    sx, sy, sz, bsx, frac = case
    host = random_sparse(msbg, sx, sy, sz, bsx, frac, 11 + bsx, dtype=dtype)
    dev = msbg.SparseGrid.from_host(ctx, host)
    fhost = dequantized(host)
    bids = np.arange(host.n_blocks)
    for halo, full, bc in itertools.product([1, 2], [0, 1], [0, 1, 2]):
        if halo > bsx:
            continue
        got = dev.halo_gather(bids, halo, full, bc)
        for b in bids:
            want = oracle.halo_fill(fhost, int(b), halo, full, bc)
            assert np.array_equal(got[b], want), (halo, full, bc, b)
