"""Pins the CPU oracle to the reference: its golden vectors (C++ MSBG outputs
hard-coded in the crate's difftests) and the unit-test known answers.  No GPU."""
import numpy as np
import pytest

from fields import dense_grid, interp_field, smoother_field, stencil_field

NEUMANN, CLAMP, DIRICHLET = 1, 0, 2


def test_stencil_goldens(msbg, oracle, goldens):
    """tests/difftest_stencil.rs:57-138: one kernel application on block 21."""
    G = goldens["stencil"]
    g = dense_grid(msbg.HostGrid, 64, stencil_field)
    for st, (name, halo, full) in enumerate([("laplacian", 1, False), ("mean_curvature", 1, True), ("bilaplacian", 2, True)]):
        h = oracle.halo_fill(g, G["block_id"], halo, full, NEUMANN)
        out = oracle.kernel(st, h, 16, G["dt"], False)
        got = out[G["sample_idx"]]
        np.testing.assert_allclose(got, G["golden"][name], atol=G["tol"], rtol=0, err_msg=name)


def test_smoother_goldens(msbg, oracle, goldens):
    """tests/difftest_smoother.rs:73-100: 4 full 8-colour sweeps."""
    G = goldens["smoother"]
    for st, name in [(0, "laplacian"), (1, "mean_curvature")]:
        g = dense_grid(msbg.HostGrid, 64, smoother_field)
        oracle.sweep(g, np.arange(64), st, G["dt"], G["iterations"], False)
        flat = np.concatenate([g.blocks[b] for b in range(64)])
        np.testing.assert_allclose(flat[G["sample_idx"]], G["golden"][name], atol=G["tol"][name], rtol=0, err_msg=name)


def test_interp_goldens(msbg, oracle, goldens):
    """tests/difftest_interp.rs:84-91: all 14 columns (Corner, Clamp)."""
    G = goldens["interp"]
    g = msbg.HostGrid("interp", 48, 48, 48, 0.0, 1.0, 16)
    zz, yy, xx = np.meshgrid(np.arange(48), np.arange(48), np.arange(48), indexing="ij")
    dense = interp_field(xx, yy, zz)
    for bid in range(g.n_blocks):
        bx, by, bz = g.get_block_coords_by_id(bid)
        g.ensure_block(bid)
        g.blocks[bid][:] = dense[bz * 16:(bz + 1) * 16, by * 16:(by + 1) * 16, bx * 16:(bx + 1) * 16].reshape(-1)
    pos = np.array(G["positions"], np.float32)
    gold = np.array(G["golden"], np.float32)
    np.testing.assert_allclose(oracle.sample_linear(g, pos, 0, CLAMP), gold[:, 0], atol=G["tol"], rtol=0)
    # columns 1-13: trilinear gradient, cubic B-spline value, gradient and
    # Hessian (sample_all, difftest_interp.rs:65-73)
    np.testing.assert_allclose(oracle.sample_ext(g, pos, 3, CLAMP, align=0), gold[:, 1:4], atol=G["tol"], rtol=0)
    np.testing.assert_allclose(oracle.sample_ext(g, pos, 0, CLAMP), gold[:, 4], atol=G["tol"], rtol=0)
    np.testing.assert_allclose(oracle.sample_ext(g, pos, 1, CLAMP), gold[:, 5:8], atol=G["tol"], rtol=0)
    np.testing.assert_allclose(oracle.sample_ext(g, pos, 2, CLAMP), gold[:, 8:14], atol=G["tol"], rtol=0)


def fnv1a(h, data: bytes):
    for b in data:
        h ^= b
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def sparse_grid_script(HostGrid):
    """tests/difftest_cpp.rs:22-43 write/read script."""
    g = HostGrid("diff", 17, 33, 5, 0.0, 1.0, 16)
    g.set_voxel(0, 0, 0, 42.0)
    g.set_voxel(16, 0, 0, 7.0)
    g.set_voxel(0, 32, 0, 3.0)
    g.set_voxel(16, 32, 4, 99.0)
    g.set_voxel(5, 5, 2, 123.5)
    g.set_voxel(3, 3, 3, 0.25)
    g.set_full_block(g.get_block_id(16, 16, 0))
    g.set_empty_block(g.get_block_id(0, 16, 0))
    return g


def test_sparse_grid_hash(msbg, goldens):
    """SparseGrid semantics pinned by the FNV-1a hash of the C++ difftest."""
    g = sparse_grid_script(msbg.HostGrid)
    h = 0xCBF29CE484222325
    for z in range(5):
        for y in range(33):
            for x in range(17):
                h = fnv1a(h, np.float32(g.get_voxel(x, y, z)).tobytes())
    assert h == int(goldens["sparse_grid_hash"]["hash"], 16)


def test_morton_known_answers(msbg, oracle, goldens):
    for x, y, z, v in goldens["morton3"]["cases"]:
        assert oracle.morton3(x, y, z) == v
        assert msbg.morton3_host(x, y, z) == v
    for x, y, z in [(0, 0, 2047), (2047, 0, 0), (1024, 1024, 1024), (2047, 2047, 2047)]:
        c = oracle.morton3(x, y, z)
        assert 0 < c < (1 << 63)
        assert c == msbg.morton3_host(x, y, z)


def test_sort_block_list_morton_coarse_first(oracle):
    """multires/sort.rs:103-123: a coarse block precedes its fine children."""
    levels = np.zeros(64, np.uint8)
    levels[21] = 1
    blocks = [21] + [bx + by * 4 + bz * 16 for bz in range(2, 4) for by in range(2, 4) for bx in range(2, 4)]
    out = oracle.sort_block_list_morton(blocks[::-1], 4, 4, levels, 2)
    assert out[0] == 21


def test_halo_known_answers(msbg, oracle):
    """multires/halo.rs:432-560 (center copy, 26 neighbours, BCs, partial block)."""
    H = msbg.HostGrid
    g = H("h", 16, 16, 16, 0.0, 1.0)
    for z in range(16):
        for y in range(16):
            for x in range(16):
                g.set_voxel(x, y, z, float(x + y * 16 + z * 256))
    h = oracle.halo_fill(g, 0, 1, True, NEUMANN).reshape(18, 18, 18)
    assert np.array_equal(h[1:17, 1:17, 1:17].reshape(-1), np.arange(4096, dtype=np.float32))

    g = H("h", 48, 48, 48, 0.0, 1.0)
    for bid in range(g.n_blocks):
        g.ensure_block(bid)
        g.blocks[bid][:] = bid
    h = oracle.halo_fill(g, 13, 1, True, NEUMANN).reshape(18, 18, 18)  # [z][y][x]
    at = lambda x, y, z: h[z, y, x]
    assert at(1, 1, 1) == 13 and at(0, 1, 1) == 12 and at(17, 1, 1) == 14
    assert at(1, 0, 1) == 10 and at(1, 17, 1) == 16 and at(1, 1, 0) == 4 and at(1, 1, 17) == 22
    assert at(0, 0, 0) == 0 and at(17, 17, 17) == 26 and at(0, 0, 1) == 9 and at(0, 17, 17) == 24

    g = H("h", 16, 16, 16, 0.0, 1.0)
    g.set_voxel(0, 0, 0, 42.0)
    g.set_empty_value(7.0)
    h = oracle.halo_fill(g, 0, 1, True, DIRICHLET).reshape(18, 18, 18)
    assert np.all(h[1:17, 1:17, 0] == 7.0)

    g = H("h", 16, 16, 16, 0.0, 1.0)
    for z in range(16):
        for y in range(16):
            for x in range(16):
                g.set_voxel(x, y, z, float(x))
    h = oracle.halo_fill(g, 0, 1, True, NEUMANN).reshape(18, 18, 18)
    assert h[1, 1, 0] == 0.0 and h[1, 1, 17] == 15.0

    g = H("h", 48, 48, 48, 0.0, 1.0)
    g.set_voxel(0, 0, 0, 5.0)
    g.set_empty_value(2.0)
    h = oracle.halo_fill(g, 0, 1, True, DIRICHLET).reshape(18, 18, 18)
    assert h[1, 1, 1] == 5.0 and h[1, 1, 0] == 2.0 and h[1, 0, 1] == 2.0 and h[0, 1, 1] == 2.0
    assert h[1, 1, 17] == 2.0 and h[0, 0, 0] == 2.0

    g = H("h", 17, 16, 16, 0.0, 1.0)
    for z in range(16):
        for y in range(16):
            for x in range(17):
                g.set_voxel(x, y, z, float(x))
    h = oracle.halo_fill(g, g.get_block_id(16, 0, 0), 1, True, NEUMANN).reshape(18, 18, 18)
    assert h[1, 1, 1] == 16.0 and h[1, 1, 2] == 16.0 and h[1, 1, 3] == 15.0


def test_meancurv_sphere_curvature(oracle):
    """meancurv.rs:195-206: curvature of |x - c| at r = 3 is 2/r."""
    hsx = 18
    z, y, x = np.meshgrid(np.arange(hsx), np.arange(hsx), np.arange(hsx), indexing="ij")
    halo = np.sqrt(((x - 1 - 8.0) ** 2 + (y - 1 - 8.0) ** 2 + (z - 1 - 8.0) ** 2)).astype(np.float32).reshape(-1)
    # D = clamp(dt * H) with dt = 1e-3 keeps the update linear in H.
    out = oracle.kernel(1, halo, 16, 1e-3, False)
    i_out = 11 + 8 * 16 + 8 * 256
    h_est = (out[i_out] - halo.reshape(hsx, hsx, hsx)[9, 9, 12]) / 1e-3
    assert abs(h_est - 2.0 / 3.0) < 2e-2


def test_sweep_affine_fixed_point(msbg, oracle):
    """solver.rs:334-361: an affine field is a fixed point of the Laplacian sweep."""
    g = msbg.HostGrid("s", 32, 32, 32, 0.0, 1.0)
    for z in range(32):
        for y in range(32):
            for x in range(32):
                g.set_voxel(x, y, z, 2.0 * x + 3.0 * y - z)
    oracle.sweep(g, np.arange(8), 0, 0.05, 1, False)
    d = g.dense()
    zz, yy, xx = np.meshgrid(np.arange(32), np.arange(32), np.arange(32), indexing="ij")
    want = (2.0 * xx + 3.0 * yy - zz).astype(np.float32)
    assert np.max(np.abs(d[1:31, 1:31, 1:31] - want[1:31, 1:31, 1:31])) < 1e-4


def test_sweep_clamp_and_skips(msbg, oracle):
    """solver.rs:397-431: dummies and unallocated blocks are skipped, clamp01 holds."""
    g = msbg.HostGrid("s", 32, 32, 32, 0.0, 1.0)
    g.set_voxel(0, 0, 0, 0.5)
    g.set_voxel(16, 16, 16, 0.7)
    g.set_full_block(g.get_block_id(0, 16, 0))
    oracle.sweep(g, [0, 7, g.get_block_id(0, 16, 0), 5], 0, 0.05, 1, True)
    assert 0.0 <= g.get_voxel(0, 0, 0) <= 1.0
    g = msbg.HostGrid("s", 16, 16, 16, 0.0, 1.0)
    for z in range(16):
        for y in range(16):
            for x in range(16):
                g.set_voxel(x, y, z, 100.0 + x)
    oracle.sweep(g, [0], 1, 1000.0, 1, True)
    assert np.all((g.blocks[0] >= 0) & (g.blocks[0] <= 1))


def test_bucket_known_answers(oracle):
    """particles/sort.rs:384-418."""
    pb, st, perm = oracle.bucket_indices([1, 0, 1, 0])
    assert list(pb) == [0, 1] and list(st) == [0, 2, 4] and list(perm) == [1, 3, 0, 2]
    pb, st, perm = oracle.bucket_indices([3])
    assert list(pb) == [3] and list(st) == [0, 1]
    pb, st, perm = oracle.bucket_indices([0, 0, 0])
    assert list(pb) == [0] and list(st) == [0, 3]
    pb, st, perm = oracle.bucket_indices([])
    assert len(pb) == 0 and list(st) == [0]
    big = [2**32 - 1, 0, 2**32, 0x1_0000_0001, 2**32 - 1]
    pb, st, perm = oracle.bucket_indices(big)
    assert list(pb) == sorted(set(big))
    i = list(pb).index(2**32 - 1)
    assert st[i + 1] - st[i] == 2


def test_bucket_equals_dense_counting_sort(oracle):
    """particles/sort.rs:420-453: random inputs vs the dense stable counting sort."""
    state = 0x9E3779B9
    for n, nb in [(0, 1), (1, 1), (1000, 64), (10000, 1024)]:
        bids = []
        for _ in range(n):
            state = (state * 1664525 + 1013904223) & 0xFFFFFFFF
            bids.append((state >> 8) % nb)
        pb, st, perm = oracle.bucket_indices(bids)
        counts = np.bincount(np.array(bids, np.int64), minlength=nb) if n else np.zeros(nb, np.int64)
        occupied = np.nonzero(counts)[0]
        assert list(pb) == list(occupied)
        assert list(st) == list(np.concatenate([[0], np.cumsum(counts[occupied])]))
        if n:
            assert list(perm) == list(np.argsort(np.array(bids), kind="stable"))


def _mac_hosts(msbg, s, active, chans):
    grids = []
    for c in range(6):
        g = msbg.HostGrid(f"c{c}", s, s, s, 0.0, 0.0)
        for k, bid in enumerate(active):
            g.ensure_block(int(bid))
            g.blocks[int(bid)][:] = chans[c][k]
        grids.append(g)
    return grids  # mass x,y,z then velocity x,y,z


def test_p2g_known_answers(msbg, oracle):
    """fluid/p2g.rs:538-619: rigid translation, radius cull, zero-mass guard."""
    s = 32
    u = np.array([1.5, -2.0, 0.5], np.float32)
    pos = np.array([[8, 8, 8], [12, 9, 7], [9, 14, 10]], np.float32)
    act, ch = oracle.p2g(pos, np.tile(u, (3, 1)), np.ones(3, np.float32), s, s, s, 16, 2.0)
    grids = _mac_hosts(msbg, s, act, ch)
    got = oracle.mac_sample(grids[3], grids[4], grids[5], pos, CLAMP)
    np.testing.assert_allclose(got, np.tile(u, (3, 1)), atol=1e-4)
    act, ch = oracle.p2g(np.array([[8, 8, 8]], np.float32), np.array([[1, 0, 0]], np.float32), np.ones(1, np.float32), s, s, s, 16, 2.0)
    grids = _mac_hosts(msbg, s, act, ch)
    assert grids[0].get_voxel(10, 8, 8) == 0.0 and grids[0].get_voxel(7, 8, 8) > 0.0
    assert grids[3].get_voxel(20, 20, 20) == 0.0 and np.isfinite(grids[3].get_voxel(7, 8, 8))


def test_p2g_staged_matches_naive(msbg, oracle):
    """fluid/p2g.rs:443-536: staged splat == exact Eq. 6 within 1e-4."""
    r = np.random.default_rng(7)
    for pos in (np.array([[8, 8, 8]], np.float32), np.array([[15.9, 8, 8]], np.float32),
                np.array([[0.1, 0.1, 0.1]], np.float32), r.uniform(0, 32, (200, 3)).astype(np.float32)):
        vel = r.normal(size=pos.shape).astype(np.float32)
        m = np.ones(len(pos), np.float32)
        act, staged = oracle.p2g(pos, vel, m, 32, 32, 32, 16, 2.0, normalize=False)
        exact, _ = oracle.p2g_f64(pos, vel, m, 32, 32, 32, 16, 2.0, act)
        np.testing.assert_allclose(staged, exact, atol=1e-4)


def test_downsample_known_answers(oracle):
    """multires/downsample.rs:96-209."""
    f = np.full((8, 4096), 0.5, np.float32)
    assert np.all(np.abs(oracle.downsample_avg(f, 16) - 0.5) < 1e-6)
    x = np.tile(np.arange(16, dtype=np.float32), 256).reshape(1, 4096)
    c = oracle.downsample_avg(x, 16).reshape(8, 8, 8)
    assert np.allclose(c[0, 0, :], 2 * np.arange(8) + 0.5)


def test_divergence_known_answer(msbg, oracle):
    """fluid/mac.rs:191-244: u=i+1, v=j+1, w=k+1 has divergence 3."""
    s = 32
    grids = []
    for a in range(3):
        g = msbg.HostGrid(f"u{a}", s, s, s, 0.0, 0.0)
        for z in range(s):
            for y in range(s):
                for x in range(s):
                    g.set_voxel(x, y, z, float((x, y, z)[a] + 1))
        grids.append(g)
    d = oracle.divergence(grids[0], grids[1], grids[2], np.arange(8))
    assert np.all(d == 3.0)


def test_g2p_face_center_exact(msbg, oracle):
    """fluid/g2p.rs:93-121."""
    s = 32
    grids = []
    for a in range(3):
        g = msbg.HostGrid(f"u{a}", s, s, s, 0.0, 0.0)
        for z in range(s):
            for y in range(s):
                for x in range(s):
                    g.set_voxel(x, y, z, float((x, y, z)[a] + 1))
        grids.append(g)
    got = oracle.mac_sample(grids[0], grids[1], grids[2], np.array([[5.0, 8.5, 8.5]], np.float32), CLAMP)
    assert list(got[0]) == [5.0, 8.5, 8.5]


def test_g2p_blend_endpoints(oracle):
    """fluid/g2p.rs:76-90."""
    uo, u, ut = (np.array([v], np.float32) for v in ([1, 2, 3], [4, 5, 6], [4.5, 4.5, 4.5]))
    assert np.array_equal(oracle.g2p_blend(uo, u, ut, 0.0), u)
    assert np.array_equal(oracle.g2p_blend(uo, u, ut, 1.0), uo + (u - ut))


def test_poisson_oracle_converges(oracle):
    """FP64 Poisson oracle (no reference counterpart; parity unpinned): plain MG
    and MG-PCG both reach 1e-8 on a shell problem; matvec of the solution
    reproduces b."""
    nx = 4
    active = np.array([b for b in range(nx ** 3) if (b % nx + (b // nx) % nx + b // nx ** 2) % 3 != 1], np.int64)
    r = np.random.default_rng(3)
    b = r.uniform(-1, 1, len(active) * 512)
    for mode in (0, 1):
        x, hist = oracle.poisson_solve(active, nx, nx, nx, 8, b, mode=mode, tol=1e-8, max_iter=100)
        assert hist[-1] <= 1e-8, (mode, hist)
        ax = oracle.poisson_matvec(active, nx, nx, nx, 8, x)
        assert np.linalg.norm(ax - b) <= 1e-7 * np.linalg.norm(b)
    # hierarchy: 8^3 blocks halve to 4, 2, then the block grid halves
    cells = oracle.poisson_levels(active, nx, nx, nx, 8)
    assert list(cells[:3]) == [len(active) * 512, len(active) * 64, len(active) * 8]
    assert cells[-1] <= 1024


# ---- surface reconstruction (particles/splat.rs, finalize.rs) --------------
R_PARTICLE, NB_DIST = 2.0, 2.0  # SurfaceConfig of the crate's splat tests


def _splat_voxels(oracle, pts, s=32, bsx=16):
    pts = np.array(pts, np.float32)
    act = oracle.surface_active(pts, s, s, s, bsx, R_PARTICLE + NB_DIST)
    vals = oracle.density_splat(pts, s, s, s, bsx, R_PARTICLE, NB_DIST, True, act)
    nb = s // bsx

    def get(x, y, z):
        b = (x // bsx) + (y // bsx) * nb + (z // bsx) * nb * nb
        k = np.searchsorted(act, b)
        if k >= len(act) or act[k] != b:
            return 0  # absent block: the grid's empty Density(0)
        return int(vals[k][(x % bsx) + (y % bsx) * bsx + (z % bsx) * bsx * bsx])
    return act, get


def test_density_splat_known_answers(oracle):
    """particles/splat.rs:371-459 (splat_01, 02, 04, 05, 06)."""
    _, get = _splat_voxels(oracle, [[8.0, 8.0, 8.0]])
    assert get(8, 8, 8) == 3072  # distSq 0.75
    assert get(5, 8, 8) == round((6.75 / 16.0) * 65535.0)
    assert get(1, 8, 8) == 65535
    assert get(4, 8, 8) == int(np.floor(np.float32(12.75 / 16.0) * np.float32(65535.0) + np.float32(0.5)))
    assert get(0, 8, 8) == 65535
    act, get = _splat_voxels(oracle, [[15.5, 8.0, 8.0]])
    assert 1 in act
    assert get(16, 8, 8) == round((1.5 / 16.0) * 65535.0)
    _, get = _splat_voxels(oracle, [[0.1, 0.1, 0.1]])
    assert get(0, 0, 0) != 65535
    _, get = _splat_voxels(oracle, [[16.0, 16.0, 16.0]])
    assert get(21, 16, 16) == 65535 and get(20, 16, 16) == 65535


def test_density_splat_min_order_independent(oracle):
    """particles/splat.rs:411-431 (splat_03): min is order-independent."""
    a = [[10.0, 8.0, 8.0], [12.0, 8.0, 8.0]]
    act1, _ = _splat_voxels(oracle, a)
    v1 = oracle.density_splat(np.array(a, np.float32), 32, 32, 32, 16, R_PARTICLE, NB_DIST, True, act1)
    v2 = oracle.density_splat(np.array(a[::-1], np.float32), 32, 32, 32, 16, R_PARTICLE, NB_DIST, True, act1)
    assert np.array_equal(v1, v2)


def test_density_finalize_known_answers(oracle):
    """particles/finalize.rs:106-175 (finalize_01 .. 04)."""
    r = 16.0
    vals = np.array([0, round(2.5 * 2.5 / r * 65535.0), 65468, 65535,
                     round(0.9989 * 65535.0), round(0.9991 * 65535.0)], np.float32)
    out = oracle.density_finalize(vals, True, R_PARTICLE, NB_DIST).astype(np.float32) / np.float32(65535.0)
    assert abs(out[0] - 1.0) < 1e-4
    assert abs(out[1] - (1.0 - (0.5 + 2.0) / 6.0)) < 1e-4
    ratio = np.float32(65468.0) / np.float32(65535.0)
    assert abs(out[2] - (1.0 - np.sqrt(ratio * r) / 6.0)) < 1e-4
    assert out[3] == 0.0
    assert out[4] > 0.0 and out[5] == 0.0
    mixed = np.array([((x + y + z) % 17) / 17.0 * 65535.0 for z in range(16) for y in range(16) for x in range(16)])
    fin = oracle.density_finalize(np.round(mixed).astype(np.float32), True, R_PARTICLE, NB_DIST)
    assert fin.min() >= 0 and fin.max() <= 65535


# ---- refinement map (multires/refinement.rs:210-330 tests) ------------------
DOM_BORDER, COARSE_FINE, FINE_COARSE = 1 << 1, 1 << 2, 1 << 3


def test_refinement_known_answers(oracle):
    n = 4
    for lv in (0, 2):  # test_ref_01: uniform maps unchanged
        m = np.full(n ** 3, lv, np.uint8)
        assert np.array_equal(oracle.regularize_refinement_map(m, n, n, n, 3), m)
    m = np.full(n ** 3, 1, np.uint8)  # test_ref_02: a single fine block
    m[21] = 0
    m = oracle.regularize_refinement_map(m, n, n, n, 3)
    flags, fc, _ = oracle.block_topology(m, n, n, n, 3)
    assert m[21] == 0 and flags[21] & FINE_COARSE and not flags[21] & COARSE_FINE
    assert fc[0].tolist() == [21]
    assert m[63] == 1 and not flags[63] & (FINE_COARSE | COARSE_FINE)
    m = np.full(n ** 3, 2, np.uint8)  # test_ref_03: a jump of 2 becomes a staircase
    m[21] = 0
    m = oracle.regularize_refinement_map(m, n, n, n, 3)
    lv = m.reshape(n, n, n)
    for z in range(n):
        for y in range(n):
            for x in range(n):
                nb = lv[max(z - 1, 0):z + 2, max(y - 1, 0):y + 2, max(x - 1, 0):x + 2]
                assert np.abs(nb.astype(int) - int(lv[z, y, x])).max() <= 1
    flags, _, _ = oracle.block_topology(np.zeros(n ** 3, np.uint8), n, n, n, 3)  # test_ref_04
    assert flags[0] & DOM_BORDER and flags[n ** 3 - 1] & DOM_BORDER and not flags[21] & DOM_BORDER
    z = np.zeros(n ** 3, np.uint8)  # test_ref_05 / 06: small level counts, idempotent
    assert np.array_equal(oracle.regularize_refinement_map(z, n, n, n, 1), z)
    assert np.array_equal(oracle.regularize_refinement_map(z, n, n, n, 2), z)
    once = oracle.regularize_refinement_map(z, n, n, n, 3)
    assert np.array_equal(oracle.regularize_refinement_map(once, n, n, n, 3), once)
