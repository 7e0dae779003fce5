"""msbg_flip_step: one FLIP transfer step through host arrays.  Its result
must equal, bit for bit, the same step composed from the device-pointer
entry points (each of which is checked against the oracle elsewhere), with
the new velocities returned in the caller's particle order; and the G2P +
blend of the step is checked against the oracle directly on a small case."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

R_P, DT, SWEEPS, ALPHA = 2.0, 0.025, 3, 0.95


def _device_step(msbg, ctx, ft, mac, coarse):
    n = ft.n
    pos = torch.from_numpy(ft.pos).cuda()
    vel = torch.from_numpy(ft.vel).cuda()
    mass = torch.from_numpy(ft.mass).cuda()
    keys = torch.empty(n, dtype=torch.int64, device="cuda")
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    from msbg_rs_b200._lib import call, ptr
    call("msbg_morton_sort_device", ctx.handle, ptr(pos), n, ptr(keys), ptr(perm))
    sp, sv, sm = torch.empty_like(pos), torch.empty_like(vel), torch.empty_like(mass)
    call("msbg_permute_device", ctx.handle, ptr(perm), n, 3, ptr(pos), ptr(sp))
    call("msbg_permute_device", ctx.handle, ptr(perm), n, 3, ptr(vel), ptr(sv))
    call("msbg_permute_device", ctx.handle, ptr(perm), n, 1, ptr(mass), ptr(sm))
    msbg.particles_to_grid_sorted_device(mac, sp, sv, sm, keys, n, R_P)
    act = mac.active_blocks()
    fine = act[ft.levels[act.astype(np.int64)] == 0]
    msbg.downsample_channel_avg(coarse, mac.mass(0))
    msbg.Sweeper(mac.mass(0)).sweep_multires(coarse, ft.levels, fine, msbg.Stencil.MeanCurvature,
                                             msbg.PdeParams(DT, SWEEPS, False))
    u = torch.empty_like(vel)
    msbg.MacSampler(mac, msbg.CLAMP).sample_device(sp, n, u)
    out = torch.empty_like(vel)
    msbg.g2p_blend_device(ctx, sv, u, u, n, ALPHA, out)
    ctx.synchronize()
    res = np.empty_like(ft.vel)
    res[perm.cpu().numpy().astype(np.int64)] = out.cpu().numpy()
    return res, act


@pytest.mark.parametrize("size", [64, 128])
def test_flip_step_equals_device_composition(msbg, ctx, size):
    from msbg_rs_b200 import workloads
    ft = workloads.flip_transfer(size=size, bsx=16, seed=5, ppc=2)
    mac_a = msbg.MacGrid(ctx, size, size, size, 16)
    coarse_a = msbg.SparseGrid(ctx, size // 2, size // 2, size // 2, 0.0, 0.0, 8, name="c")
    want, act_a = _device_step(msbg, ctx, ft, mac_a, coarse_a)
    mac_b = msbg.MacGrid(ctx, size, size, size, 16)
    coarse_b = msbg.SparseGrid(ctx, size // 2, size // 2, size // 2, 0.0, 0.0, 8, name="c")
    fs = msbg.FlipStep(mac_b, coarse_b, ft.levels)
    for _ in range(2):  # the second call reuses the step's device arrays
        got = fs.step(ft.pos, ft.vel, ft.mass, R_P, msbg.Stencil.MeanCurvature, DT, SWEEPS, ALPHA)
        assert np.array_equal(got, want)
    assert np.array_equal(mac_b.active_blocks(), act_a)
    fs.close()


def test_flip_step_against_oracle(msbg, ctx, oracle):
    """Without sweeps the step is P2G, G2P and the blend: checked end to end
    against the oracle's G2P on the oracle-checked grid."""
    from msbg_rs_b200 import workloads
    size = 64
    ft = workloads.flip_transfer(size=size, bsx=16, seed=6, ppc=1)
    mac = msbg.MacGrid(ctx, size, size, size, 16)
    coarse = msbg.SparseGrid(ctx, size // 2, size // 2, size // 2, 0.0, 0.0, 8, name="c")
    fs = msbg.FlipStep(mac, coarse, ft.levels)
    got = fs.step(ft.pos, ft.vel, ft.mass, R_P, msbg.Stencil.MeanCurvature, DT, 0, ALPHA)
    act = mac.active_blocks()
    vg = []
    for a in range(3):
        g = msbg.HostGrid(f"v{a}", size, size, size, 0.0, 0.0, 16)
        data = mac.velocity(a).read_blocks(act)
        for k, b in enumerate(act):
            g.ensure_block(int(b))
            g.blocks[int(b)][:] = data[k]
        vg.append(g)
    u = oracle.mac_sample(vg[0], vg[1], vg[2], ft.pos, msbg.CLAMP)
    want = oracle.g2p_blend(ft.vel, u, u, ALPHA)
    assert np.array_equal(got, want)
    fs.close()
