"""Particle sorts, P2G and G2P on the GPU against the CPU oracle.

Sorts and G2P are bit-exact.  P2G evaluates every per-particle term exactly
as the reference does (f32, same operation order, same clamped footprint) but
sums the terms in a different fixed order and in FP64.  So it is checked
(1) against the oracle's FP64 sum of the same f32 terms: equal up to 1 ulp of
the f32 result (rounding of two FP64 sums that differ only in order),
(2) against the exact Eq. 6 splat in FP64 weights: within 32 eps of the sum
of |terms| (the f32 weight evaluation error), and (3) against the reference's
own f32 staged splat: within P2G_F32_TOL of the sum of |terms| (the
reference's f32 accumulation error)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = float(np.finfo(np.float32).eps)
P2G_EXACT_TOL = 32 * EPS    # relative to sum |terms|
P2G_F32_TOL = 1e-6          # relative to sum |terms|


def ulp_diff(a, b):
    """|a - b| in units of the f32 spacing at b."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    sp = np.spacing(np.abs(b)).astype(np.float64)
    return np.abs(a.astype(np.float64) - b.astype(np.float64)) / sp


def test_morton3_device(msbg, ctx, oracle):
    r = np.random.default_rng(0)
    xyz = r.integers(0, 1 << 21, (1000, 3)).astype(np.uint64)
    got = msbg.morton3(ctx, xyz)
    want = np.array([oracle.morton3(*map(int, v)) for v in xyz], np.uint64)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n,extent", [(0, 16), (1, 16), (1000, 16), (70000, 64), (300000, 1500), (5000, 2 ** 21 - 1)])
def test_morton_sort_bit_exact(msbg, ctx, oracle, n, extent):
    r = np.random.default_rng(n)
    pos = r.uniform(0, extent, (n, 3)).astype(np.float32)
    if n > 10:
        pos[: n // 10] = pos[n // 10: 2 * (n // 10)]  # duplicate keys exercise stability
    keys, perm = msbg.morton_sort(ctx, pos)
    wk, wp = oracle.morton_sort(pos)
    assert np.array_equal(keys, wk) and np.array_equal(perm, wp)


@pytest.mark.parametrize("n,nb", [(0, 1), (1, 1), (1000, 64), (100000, 4096), (50000, 2 ** 40)])
def test_bucket_indices_bit_exact(msbg, ctx, oracle, n, nb):
    r = np.random.default_rng(n + 1)
    bids = r.integers(0, nb, n).astype(np.uint64)
    plan = msbg.bucket_indices(ctx, bids)
    pb, st, perm = oracle.bucket_indices(bids)
    assert np.array_equal(plan.particle_blocks, pb)
    assert np.array_equal(plan.starts, st)
    assert np.array_equal(plan.perm, perm)


def test_bucket_u64_scale(msbg, ctx):
    bids = np.array([2**32 - 1, 0, 2**32, 0x1_0000_0001, 2**32 - 1], np.uint64)
    plan = msbg.bucket_indices(ctx, bids)
    assert list(plan.particle_blocks) == sorted(set(bids.tolist()))
    i = list(plan.particle_blocks).index(2**32 - 1)
    assert plan.starts[i + 1] - plan.starts[i] == 2


def test_sort_block_list_morton_device(msbg, ctx, oracle):
    r = np.random.default_rng(3)
    nx = ny = nz = 16
    levels = r.integers(0, 3, nx * ny * nz).astype(np.uint8)
    blocks = r.permutation(nx * ny * nz)[:2000]
    got = msbg.sort_block_list_morton(ctx, blocks, nx, ny, levels, 3)
    want = oracle.sort_block_list_morton(blocks, nx, ny, levels, 3)
    assert np.array_equal(got.astype(np.int64), want)


def make_particles(n, s, seed):
    r = np.random.default_rng(seed)
    pos = r.uniform(0.0, s, (n, 3)).astype(np.float32)
    pos = np.minimum(pos, np.float32(s) - np.float32(1e-3))
    vel = r.normal(size=(n, 3)).astype(np.float32)
    mass = r.uniform(0.5, 1.5, n).astype(np.float32)
    return pos, vel, mass


def device_channels(mac, active):
    """[6][n_active][N]: mass x,y,z then velocity x,y,z, as in oracle.p2g."""
    return np.stack([mac.mass(a).read_blocks(active) for a in range(3)] +
                    [mac.velocity(a).read_blocks(active) for a in range(3)])


def check_p2g(msbg, ctx, oracle, pos, vel, mass, s, bsx, r_p):
    mac = msbg.MacGrid(ctx, s, s, s, bsx)
    na = msbg.particles_to_grid(mac, pos, vel, mass, r_p)
    act = mac.active_blocks()
    want_act = oracle.active_blocks(pos, s, s, s, bsx, r_p)
    assert na == len(want_act) and np.array_equal(act.astype(np.int64), want_act)
    got = device_channels(mac, act)
    terms64 = oracle.p2g_terms_f64(pos, vel, mass, s, s, s, bsx, r_p, want_act)
    _, ref32 = oracle.p2g(pos, vel, mass, s, s, s, bsx, r_p, active=want_act, normalize=False)
    exact, absum = oracle.p2g_f64(pos, vel, mass, s, s, s, bsx, r_p, want_act)
    for a in range(3):
        absum[3 + a] = np.maximum(absum[3 + a], 0)
        # (1) mass: the f32 rounding of the FP64 sum of the reference's terms
        m_want = terms64[a].astype(np.float32)
        assert ulp_diff(got[a], m_want).max() <= 1.0, ("mass ulp", a)
        # velocity = f32(P) / f32(M), as normalize_velocity (mac.rs:106-132)
        p_want = terms64[3 + a].astype(np.float32)
        with np.errstate(divide="ignore", invalid="ignore"):
            v_want = np.where(m_want > 0, p_want / np.where(m_want > 0, m_want, 1), 0).astype(np.float32)
        # (FP64 sums in a different order can move a heavily cancelled
        # momentum by more than an ulp of itself, never by more than an ulp
        # of the sum of |terms|.)
        well_conditioned = np.abs(terms64[3 + a]) >= 1e-3 * absum[3 + a]
        assert np.all((ulp_diff(got[3 + a], v_want) <= 3.0) | ~well_conditioned), ("velocity ulp", a)
        mom = got[3 + a].astype(np.float64) * got[a].astype(np.float64)
        assert np.all(np.abs(mom - terms64[3 + a]) <= 4 * EPS * absum[3 + a] + 1e-30), ("momentum", a)
        # (3) against the reference's own f32 staged sums
        err = np.abs(got[a].astype(np.float64) - ref32[a])
        assert np.all(err <= P2G_F32_TOL * absum[a] + 1e-30), ("f32 staged", a, (err / np.maximum(absum[a], 1e-30)).max())
        # (2) against exact-weight FP64: the reference's f32 weight near the
        # edge of the support, w = (1 - d^2/r^2)^3, carries a cancellation
        # error of ~eps * m per term, so the bound has an absolute part.
        err = np.abs(got[a].astype(np.float64) - exact[a])
        assert np.all(err <= P2G_EXACT_TOL * absum[a] + 8 * EPS * mass.max()), ("exact", a, err.max())
    return mac, got


@pytest.mark.parametrize("r_p,bsx,seed", [(2.0, 16, 11), (2.0, 8, 12), (1.5, 16, 13), (3.0, 16, 14)])
def test_p2g_terms_bit_exact(msbg, ctx, oracle, r_p, bsx, seed):
    """Particles on a lattice 8 cells apart, so no two footprints share a
    face: every face sum is a single term, and mass and velocity must equal
    the reference's own staged splat bit for bit.  This pins each term's f32
    operation sequence, which the summed comparisons allow an ulp of slack
    on.  A quarter of the particles have a coordinate exactly on a cell
    centre or a face plane (the footprints of irregular shape)."""
    s = 64
    r = np.random.default_rng(seed)
    lat = np.arange(8) * 8 + 2
    pos = np.stack(np.meshgrid(lat, lat, lat, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    pos += r.uniform(0, 1, pos.shape).astype(np.float32)
    n = len(pos)
    special = r.choice(n, n // 4, replace=False)
    ax = r.integers(0, 3, len(special))
    pos[special, ax] = np.floor(pos[special, ax]) + r.choice(np.array([0.0, 0.5], np.float32), len(special))
    vel = r.normal(size=(n, 3)).astype(np.float32)
    mass = r.uniform(0.5, 1.5, n).astype(np.float32)
    mac = msbg.MacGrid(ctx, s, s, s, bsx)
    msbg.particles_to_grid(mac, pos, vel, mass, r_p)
    act = mac.active_blocks()
    _, want = oracle.p2g(pos, vel, mass, s, s, s, bsx, r_p, active=act.astype(np.int64), normalize=True)
    got = device_channels(mac, act)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("n,s,bsx,r_p,seed", [
    (1, 32, 16, 2.0, 1), (500, 32, 16, 2.0, 2), (20000, 64, 16, 2.0, 3), (20000, 64, 16, 1.5, 4),
    (8000, 48, 8, 2.0, 5), (5000, 64, 16, 3.0, 6),
    # r_p <= 1 (8 tile phases) and r_p 3 on 8^3 blocks (64 phases, one warp per CTA)
    (3000, 32, 16, 1.0, 7), (4000, 32, 8, 3.0, 8),
])
def test_p2g_matches_oracle(msbg, ctx, oracle, n, s, bsx, r_p, seed):
    pos, vel, mass = make_particles(n, s, seed)
    check_p2g(msbg, ctx, oracle, pos, vel, mass, s, bsx, r_p)


def test_p2g_edge_cases(msbg, ctx, oracle):
    """Block seam, domain corner, integer positions (zero-weight boundary faces)."""
    pos = np.array([[15.9, 8, 8], [0.1, 0.1, 0.1], [8, 8, 8], [16, 16, 16], [31.99, 31.99, 0.0], [2, 3, 4]], np.float32)
    vel = np.array([[1, 0, 0], [1, 1, 1], [0, -2, 1], [3, 3, 3], [-1, 0, 2], [0.5, 0.5, 0.5]], np.float32)
    check_p2g(msbg, ctx, oracle, pos, vel, np.ones(len(pos), np.float32), 32, 16, 2.0)


def test_p2g_plane_and_centre_positions(msbg, ctx, oracle):
    """Coordinates exactly on cell centres (x.5) and face planes (integers),
    alone and mixed with regular ones, and one cell holding 300 particles
    (more than a warp stages at once): the cases the r_p = 2 splat sends down
    its general path or across staging refills."""
    r = np.random.default_rng(21)
    base = r.integers(1, 30, (600, 3)).astype(np.float32)
    frac = r.choice(np.array([0.0, 0.5, 0.25, 0.75, 0.9999], np.float32), (600, 3))
    dense = np.float32([9, 9, 9]) + r.uniform(0, 1, (300, 3)).astype(np.float32)
    pos = np.concatenate([base + frac, dense]).astype(np.float32)
    vel = r.normal(size=pos.shape).astype(np.float32)
    mass = r.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    check_p2g(msbg, ctx, oracle, pos, vel, mass, 32, 16, 2.0)
    check_p2g(msbg, ctx, oracle, pos, vel, mass, 32, 8, 2.0)


def test_p2g_deterministic(msbg, ctx):
    pos, vel, mass = make_particles(30000, 64, 9)
    runs = []
    for _ in range(2):
        mac = msbg.MacGrid(ctx, 64, 64, 64, 16)
        msbg.particles_to_grid(mac, pos, vel, mass, 2.0)
        runs.append(device_channels(mac, mac.active_blocks()))
    assert np.array_equal(runs[0], runs[1])


def test_p2g_sorted_input_identical(msbg, ctx):
    """msbg_p2g_sorted_device on Morton-sorted particles == msbg_p2g."""
    import torch
    pos, vel, mass = make_particles(40000, 64, 13)
    mac = msbg.MacGrid(ctx, 64, 64, 64, 16)
    msbg.particles_to_grid(mac, pos, vel, mass, 2.0)
    ref = device_channels(mac, mac.active_blocks())
    keys, perm = msbg.morton_sort(ctx, pos)
    tp, tv, tm = (torch.from_numpy(np.ascontiguousarray(x[perm])).cuda() for x in (pos, vel, mass))
    tk = torch.from_numpy(keys.view(np.int64)).cuda()
    mac2 = msbg.MacGrid(ctx, 64, 64, 64, 16)
    msbg.particles_to_grid_sorted_device(mac2, tp, tv, tm, tk, len(pos), 2.0)
    ctx.synchronize()
    assert np.array_equal(mac2.active_blocks(), mac.active_blocks())
    assert np.array_equal(device_channels(mac2, mac2.active_blocks()), ref)


def test_p2g_permuted_input_identical(msbg, ctx):
    """msbg_p2g_permuted_device on particles in the caller's order with the
    keys and permutation of their Morton sort == msbg_p2g."""
    import torch
    pos, vel, mass = make_particles(40000, 64, 14)
    mac = msbg.MacGrid(ctx, 64, 64, 64, 16)
    msbg.particles_to_grid(mac, pos, vel, mass, 2.0)
    ref = device_channels(mac, mac.active_blocks())
    tp, tv, tm = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (pos, vel, mass))
    tk = torch.empty(len(pos), dtype=torch.int64, device="cuda")
    tperm = torch.empty(len(pos), dtype=torch.int32, device="cuda")
    from msbg_rs_b200._lib import call, ptr
    call("msbg_morton_sort_device", ctx.handle, ptr(tp), len(pos), ptr(tk), ptr(tperm))
    mac2 = msbg.MacGrid(ctx, 64, 64, 64, 16)
    msbg.particles_to_grid_permuted_device(mac2, tp, tv, tm, tk, tperm, len(pos), 2.0)
    ctx.synchronize()
    assert np.array_equal(mac2.active_blocks(), mac.active_blocks())
    assert np.array_equal(device_channels(mac2, mac2.active_blocks()), ref)


def test_p2g_rejects_out_of_domain(msbg, ctx):
    mac = msbg.MacGrid(ctx, 32, 32, 32, 16)
    with pytest.raises(msbg.MsbgError):
        msbg.particles_to_grid(mac, np.array([[40.0, 1, 1]], np.float32), np.zeros((1, 3), np.float32),
                               np.ones(1, np.float32), 2.0)
    assert msbg.particles_to_grid(mac, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32),
                                  np.zeros(0, np.float32), 2.0) == 0


def host_channels(msbg, s, bsx, active, chans):
    grids = []
    for c in range(6):
        g = msbg.HostGrid(f"c{c}", s, s, s, 0.0, 0.0, bsx)
        for k, bid in enumerate(active):
            g.ensure_block(int(bid))
            g.blocks[int(bid)][:] = chans[c][k]
        grids.append(g)
    return grids


@pytest.mark.parametrize("bc", [0, 1, 2])
def test_g2p_bit_exact(msbg, ctx, oracle, bc):
    s, bsx = 48, 16
    pos, vel, mass = make_particles(20000, s, 11)
    mac = msbg.MacGrid(ctx, s, s, s, bsx)
    msbg.particles_to_grid(mac, pos, vel, mass, 2.0)
    act = mac.active_blocks()
    chans = device_channels(mac, act)
    grids = host_channels(msbg, s, bsx, act, chans)
    q = np.concatenate([pos, np.random.default_rng(1).uniform(-3, s + 3, (3000, 3)).astype(np.float32)])
    got = msbg.MacSampler(mac, bc).sample(q)
    want = oracle.mac_sample(grids[3], grids[4], grids[5], q, bc)
    assert np.array_equal(got, want)


def test_p2g_g2p_rigid_translation(msbg, ctx):
    """fluid/p2g.rs:538-557: a rigidly translating cloud round-trips."""
    u = np.array([1.5, -2.0, 0.5], np.float32)
    pos = np.array([[8, 8, 8], [12, 9, 7], [9, 14, 10]], np.float32)
    mac = msbg.MacGrid(ctx, 32, 32, 32, 16)
    msbg.particles_to_grid(mac, pos, np.tile(u, (3, 1)), np.ones(3, np.float32), 2.0)
    got = msbg.MacSampler(mac, msbg.CLAMP).sample(pos)
    np.testing.assert_allclose(got, np.tile(u, (3, 1)), atol=1e-4)


def test_sample_linear_interp_goldens(msbg, ctx, oracle, goldens):
    """tests/difftest_interp.rs trilinear values through the device sampler."""
    from fields import interp_field
    G = goldens["interp"]
    g = msbg.HostGrid("interp", 48, 48, 48, 0.0, 1.0, 16)
    zz, yy, xx = np.meshgrid(np.arange(48), np.arange(48), np.arange(48), indexing="ij")
    dense = interp_field(xx, yy, zz)
    for bid in range(g.n_blocks):
        bx, by, bz = g.get_block_coords_by_id(bid)
        g.ensure_block(bid)
        g.blocks[bid][:] = dense[bz * 16:(bz + 1) * 16, by * 16:(by + 1) * 16, bx * 16:(bx + 1) * 16].reshape(-1)
    dev = msbg.SparseGrid.from_host(ctx, g)
    p = np.array(G["positions"], np.float32)
    got = dev.sample_linear(p, 0, msbg.CLAMP)
    np.testing.assert_allclose(got, [row[0] for row in G["golden"]], atol=G["tol"], rtol=0)
    assert np.array_equal(got, oracle.sample_linear(g, p, 0, msbg.CLAMP))


def test_g2p_blend_device(msbg, ctx, oracle):
    import torch
    r = np.random.default_rng(2)
    a, b, c = (r.normal(size=(1000, 3)).astype(np.float32) for _ in range(3))
    ta, tb, tc = (torch.from_numpy(x).cuda() for x in (a, b, c))
    out = torch.empty_like(ta)
    msbg.g2p_blend_device(ctx, ta, tb, tc, 1000, 0.95, out)
    ctx.synchronize()
    assert np.array_equal(out.cpu().numpy(), oracle.g2p_blend(a, b, c, 0.95))


def test_divergence_and_downsample(msbg, ctx, oracle):
    s = 48
    pos, vel, mass = make_particles(20000, s, 12)
    mac = msbg.MacGrid(ctx, s, s, s, 16)
    msbg.particles_to_grid(mac, pos, vel, mass, 2.0)
    act = mac.active_blocks()
    div = msbg.SparseGrid(ctx, s, s, s, 0.0, 0.0, 16)
    mac.divergence(div, act)
    grids = host_channels(msbg, s, 16, act, device_channels(mac, act))
    want = oracle.divergence(grids[3], grids[4], grids[5], act)
    assert np.array_equal(div.read_blocks(act), want)
    coarse = msbg.SparseGrid(ctx, s // 2, s // 2, s // 2, 0.0, 0.0, 8)
    msbg.downsample_channel_avg(coarse, div)
    assert np.array_equal(coarse.read_blocks(act), oracle.downsample_avg(want, 16))


@pytest.mark.parametrize("with_tilde", [False, True])
def test_g2p_flip_device_equals_sample_then_blend(msbg, ctx, with_tilde):
    """msbg_g2p_flip_device (sample and blend in one pass) gives the bits of
    msbg_g2p_device followed by msbg_g2p_blend_device, with u_tilde the
    sample itself (null) or a caller array; samples outside the domain (the
    boundary gather) included."""
    import torch
    s, bsx = 48, 16
    pos, vel, mass = make_particles(20000, s, 5)
    mac = msbg.MacGrid(ctx, s, s, s, bsx)
    msbg.particles_to_grid(mac, pos, vel, mass, 2.0)
    q = np.concatenate([pos, np.random.default_rng(2).uniform(-3, s + 3, (3000, 3)).astype(np.float32)])
    n = len(q)
    rng = np.random.default_rng(3)
    d_q = torch.from_numpy(q).cuda()
    d_old = torch.from_numpy(rng.standard_normal((n, 3)).astype(np.float32)).cuda()
    d_ut = torch.from_numpy(rng.standard_normal((n, 3)).astype(np.float32)).cuda() if with_tilde else None
    sampler = msbg.MacSampler(mac, msbg.CLAMP)
    u = torch.empty_like(d_old)
    want = torch.empty_like(d_old)
    sampler.sample_device(d_q, n, u)
    msbg.g2p_blend_device(ctx, d_old, u, d_ut if with_tilde else u, n, 0.95, want)
    got = torch.full_like(d_old, 7.0)
    msbg.g2p_flip_device(sampler, d_q, n, d_old, 0.95, got, d_ut)
    ctx.synchronize()
    assert np.array_equal(got.cpu().numpy().view(np.uint32), want.cpu().numpy().view(np.uint32))
