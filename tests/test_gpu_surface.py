"""Surface reconstruction on the device (particles/{sort,splat,finalize}.rs,
particles/mod.rs:279-302): the crate's splat and finalize known answers, and
bit-exact agreement with the oracle's restatement for random clouds (the
splat is a minimum, so the order of the particles does not matter), for the
placement, and for reconstruct_and_smooth (splat, finalize, clamped
mean-curvature sweeps on Density and Density8 storage)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def density_grid(msbg, ctx, s, bsx=16, dtype="u16"):
    return msbg.SparseGrid(ctx, s, s, s, 0.0, 1.0, bsx, dtype, name="surface")


def splat(msbg, ctx, pts, s=32, dtype="u16", bsx=16, r_particle=2.0, nb_dist=2.0):
    g = density_grid(msbg, ctx, s, bsx, dtype)
    cfg = msbg.SurfaceConfig(s, s, s, r_particle=r_particle, nb_dist=nb_dist)
    d = torch.from_numpy(np.ascontiguousarray(pts, np.float32).reshape(-1, 3)).cuda()
    act = msbg.surface.splat_device(g, d, len(d), cfg)
    return g, act, cfg


def voxel(g, act, bsx, x, y, z):
    nb = g.nx
    b = (x // bsx) + (y // bsx) * nb + (z // bsx) * nb * nb
    if b not in set(act.tolist()):
        return 0
    return int(g.read_blocks([b])[0][(x % bsx) + (y % bsx) * bsx + (z % bsx) * bsx * bsx])


def test_splat_known_answers(msbg, ctx):
    """particles/splat.rs:371-459."""
    g, act, _ = splat(msbg, ctx, [[8.0, 8.0, 8.0]])
    assert voxel(g, act, 16, 8, 8, 8) == 3072
    assert voxel(g, act, 16, 5, 8, 8) == round((6.75 / 16.0) * 65535.0)
    assert voxel(g, act, 16, 1, 8, 8) == 65535
    assert voxel(g, act, 16, 0, 8, 8) == 65535
    g, act, _ = splat(msbg, ctx, [[15.5, 8.0, 8.0]])
    assert 1 in act.tolist() and voxel(g, act, 16, 16, 8, 8) == round((1.5 / 16.0) * 65535.0)
    g, act, _ = splat(msbg, ctx, [[0.1, 0.1, 0.1]])
    assert voxel(g, act, 16, 0, 0, 0) != 65535
    g, act, _ = splat(msbg, ctx, [[16.0, 16.0, 16.0]])
    assert voxel(g, act, 16, 21, 16, 16) == 65535 and voxel(g, act, 16, 20, 16, 16) == 65535


@pytest.mark.parametrize("dtype", ["u16", "f32", "u8"])
@pytest.mark.parametrize("bsx,r_particle,nb_dist", [(16, 2.0, 2.0), (8, 1.5, 1.0), (16, 3.0, 4.5)])
def test_splat_and_finalize_match_oracle(msbg, ctx, oracle, dtype, bsx, r_particle, nb_dist):
    s = 64
    r = np.random.default_rng(bsx + int(10 * r_particle))
    pts = np.concatenate([r.uniform(0, s, (20000, 3)),
                          r.integers(0, s, (500, 3)) + r.choice([0.0, 0.5], (500, 3)),
                          np.float32([20, 20, 20]) + r.uniform(0, 1, (3000, 3))]).astype(np.float32)
    pts = np.minimum(pts, np.float32(s) - np.float32(1e-3))
    g, act, cfg = splat(msbg, ctx, pts, s, dtype, bsx, r_particle, nb_dist)
    want_act = oracle.surface_active(pts, s, s, s, bsx, r_particle + nb_dist)
    assert np.array_equal(act.astype(np.int64), want_act)
    want = oracle.density_splat(pts, s, s, s, bsx, r_particle, nb_dist, dtype, want_act)
    got = g.read_blocks(act)
    assert np.array_equal(got, want)
    msbg.surface.finalize(g, act, cfg)
    want_f = oracle.density_finalize(want, dtype, r_particle, nb_dist)
    assert np.array_equal(g.read_blocks(act), want_f)


@pytest.mark.parametrize("dtype", ["u16", "u8"])
def test_reconstruct_and_smooth_matches_oracle(msbg, ctx, oracle, dtype):
    """Density8 smooths through the sqrt-compressed stochastic store of a
    fresh sweeper (seed 0xdeadbeef, 16 lanes)."""
    s, bsx = 64, 16
    r = np.random.default_rng(3)
    # particles on a sphere shell, the kind of cloud the pipeline reconstructs
    d = r.normal(size=(30000, 3))
    pts = (32 + 18 * d / np.linalg.norm(d, axis=1, keepdims=True) + r.uniform(-1, 1, (30000, 3))).astype(np.float32)
    g = density_grid(msbg, ctx, s, bsx, dtype)
    cfg = msbg.SurfaceConfig(s, s, s, r_particle=2.0, nb_dist=2.0, n_smooth_iters=3, smooth_dt=0.05)
    act = msbg.reconstruct_and_smooth(g, pts, cfg)
    want_act = oracle.surface_active(pts, s, s, s, bsx, cfg.r_scan)
    assert np.array_equal(act.astype(np.int64), want_act)
    vals = oracle.density_finalize(oracle.density_splat(pts, s, s, s, bsx, 2.0, 2.0, dtype, want_act), dtype, 2.0, 2.0)
    host = msbg.HostGrid("surface", s, s, s, 0.0, 1.0, bsx, dtype)
    for k, b in enumerate(want_act):
        host.ensure_block(int(b))
        host.blocks[int(b)][:] = vals[k]
    if dtype == "u8":
        oracle.sweep_stochastic(host, want_act, msbg.Stencil.MeanCurvature, cfg.smooth_dt, cfg.n_smooth_iters, True)
    else:
        oracle.sweep(host, want_act, msbg.Stencil.MeanCurvature, cfg.smooth_dt, cfg.n_smooth_iters, True)
    got = g.read_blocks(act)
    for k, b in enumerate(want_act):
        assert np.array_equal(got[k], host.block_array(int(b))), int(b)


def test_place_matches_oracle(msbg, ctx, oracle):
    r = np.random.default_rng(9)
    base = r.uniform(-0.1, 0.2, (300, 3)).astype(np.float32)
    bbox = base.min(axis=0)
    span = float((base.max(axis=0) - bbox).max())
    for s, factor in ((64, 0.1), (48, 0.3)):
        cfg = msbg.SurfaceConfig(s, s, s, instance_scale_factor=factor)
        got = msbg.surface.place(ctx, base, bbox, span, cfg)
        want, _ = oracle.place(base, bbox, span, s, s, s, 16, factor, len(base))
        assert len(got) > 0 and np.array_equal(got, want)
