"""Parity at the benchmark configurations' full sizes.

FLIP transfer, 256^3 (25,427,968 particles, 3 levels): every stage of the
timed step is checked against the oracle, fed with the device's output of
the stage before (so a stage is judged on its own): the Morton sort and the
permutation bit for bit, the P2G active set exactly and the splatted face
masses within 1 ulp of the FP64 sum of the reference's f32 terms over a
Morton-contiguous third of the active blocks, the 10 multires 19-tap sweeps
and G2P + blend bit for bit.

Phase field, 512^3 band: 10 sweeps of the 25-tap stencil on BF16 storage
with [0, 1] clamping, bit for bit against the oracle over every level-0 block.

Pressure solve on the 256^3 layout's level-0 blocks (3.18 M unknowns): the
learned preconditioner, trained on the device, inside CG reaches 1e-6; the
true residual of the FP64 solution is re-measured on the host.

Batched solves: all 64 problems (edges up to 256^3) reach 1e-8, and the FP64
solution of the smallest 256^3 problem is within 1e-6 of the oracle's (both
solutions are 1e-8-residual approximations of the same system).

Tolerances: as stated per check; integer and f32-order-exact stages are
compared bit for bit."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

R_P, DT, SWEEPS, ALPHA = 2.0, 0.025, 10, 0.95


def ulp_diff(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


def host_grid(msbg, name, size, bsx, bids, data):
    g = msbg.HostGrid(name, size, size, size, 0.0, 0.0, bsx)
    for k, b in enumerate(bids):
        g.ensure_block(int(b))
        g.blocks[int(b)][:] = data[k]
    return g


def test_flip_transfer_256_stagewise(msbg, ctx, oracle):
    from msbg_rs_b200 import workloads
    from msbg_rs_b200._lib import call, ptr
    size, bsx = 256, 16
    ft = workloads.flip_transfer(size=size, bsx=bsx, seed=2, ppc=8)
    n = ft.n
    threads = oracle.num_threads()
    pos = torch.from_numpy(ft.pos).cuda()
    vel = torch.from_numpy(ft.vel).cuda()
    mass = torch.from_numpy(ft.mass).cuda()
    keys = torch.empty(n, dtype=torch.int64, device="cuda")
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    call("msbg_morton_sort_device", ctx.handle, ptr(pos), n, ptr(keys), ptr(perm))
    sp, sv, sm = torch.empty_like(pos), torch.empty_like(vel), torch.empty_like(mass)
    call("msbg_permute_device", ctx.handle, ptr(perm), n, 3, ptr(pos), ptr(sp))
    call("msbg_permute_device", ctx.handle, ptr(perm), n, 3, ptr(vel), ptr(sv))
    call("msbg_permute_device", ctx.handle, ptr(perm), n, 1, ptr(mass), ptr(sm))
    ctx.synchronize()
    # 1. Morton sort: bit-exact against the stable CPU sort
    wk, wp = oracle.morton_sort(ft.pos)
    assert np.array_equal(keys.cpu().numpy().view(np.uint64), wk)
    assert np.array_equal(perm.cpu().numpy().view(np.uint32), wp)
    pos_s, vel_s, mass_s = ft.pos[wp], ft.vel[wp], ft.mass[wp]
    assert np.array_equal(sp.cpu().numpy(), pos_s)
    # 2. P2G on the sorted particles
    mac = msbg.MacGrid(ctx, size, size, size, bsx)
    msbg.particles_to_grid_sorted_device(mac, sp, sv, sm, keys, n, R_P)
    act = mac.active_blocks()
    want_act = oracle.active_blocks(pos_s, size, size, size, bsx, R_P)
    assert np.array_equal(act.astype(np.int64), want_act)
    # a Morton-contiguous third of the active blocks
    bx, by, bz = act % (size // bsx), (act // (size // bsx)) % (size // bsx), act // (size // bsx) ** 2
    mk = np.array([oracle.morton3(int(x), int(y), int(z)) for x, y, z in zip(bx, by, bz)], np.uint64)
    third = act[np.argsort(mk, kind="stable")][: len(act) // 3]
    third = np.sort(third)
    terms = oracle.p2g_terms_f64(pos_s, vel_s, mass_s, size, size, size, bsx, R_P, third.astype(np.int64),
                                 threads=threads)
    for a in range(3):
        got = mac.mass(a).read_blocks(third)
        assert ulp_diff(got, terms[a].astype(np.float32)).max() <= 1, ("mass", a)
    # 3. downsample + 10 multires 19-tap sweeps over the level-0 blocks
    fine = act[ft.levels[act.astype(np.int64)] == 0]
    mass_x = mac.mass(0).read_blocks(act)
    coarse = msbg.SparseGrid(ctx, size // 2, size // 2, size // 2, 0.0, 0.0, bsx // 2, name="coarse")
    msbg.downsample_channel_avg(coarse, mac.mass(0))
    msbg.Sweeper(mac.mass(0)).sweep_multires(coarse, ft.levels, fine, msbg.Stencil.MeanCurvature,
                                             msbg.PdeParams(DT, SWEEPS, False))
    got = mac.mass(0).read_blocks(fine)
    hf = host_grid(msbg, "mass_x", size, bsx, act, mass_x)
    hc = host_grid(msbg, "coarse", size // 2, bsx // 2, act, oracle.downsample_avg(mass_x, bsx))
    oracle.sweep_multires(hf, hc, ft.levels, fine.astype(np.int64), 1, DT, SWEEPS, False, threads=threads)
    for k, b in enumerate(fine):
        assert np.array_equal(got[k], hf.blocks[int(b)]), int(b)
    # 4. G2P + FLIP/PIC blend on the splatted velocities
    u = torch.empty_like(vel)
    msbg.MacSampler(mac, msbg.CLAMP).sample_device(sp, n, u)
    out = torch.empty_like(vel)
    msbg.g2p_blend_device(ctx, sv, u, u, n, ALPHA, out)
    ctx.synchronize()
    vg = [host_grid(msbg, f"v{a}", size, bsx, act, mac.velocity(a).read_blocks(act)) for a in range(3)]
    want_u = oracle.mac_sample(vg[0], vg[1], vg[2], pos_s, msbg.CLAMP)
    assert np.array_equal(u.cpu().numpy(), want_u)
    assert np.array_equal(out.cpu().numpy(), oracle.g2p_blend(vel_s, want_u, want_u, ALPHA))


def test_phase_field_512_bf16_25tap(msbg, ctx, oracle):
    from msbg_rs_b200 import workloads
    size = 512
    pf = workloads.phase_field(size, particles=False)
    fine = pf.fine_blocks
    bits = workloads.bf16_bits(pf.phase)
    dev = msbg.SparseGrid(ctx, size, size, size, 0.0, 1.0, 16, dtype="bf16", name="phase")
    dev.write_blocks(fine, bits)
    msbg.Sweeper(dev).sweep(fine, msbg.Stencil.BiLaplacian, msbg.PdeParams(0.01, SWEEPS, True))
    got = dev.read_blocks(fine)
    host = msbg.HostGrid("phase", size, size, size, 0.0, 1.0, 16, "bf16")
    for k, b in enumerate(fine):
        host.ensure_block(int(b))
        host.blocks[int(b)][:] = bits[k]
    oracle.sweep(host, fine.astype(np.int64), msbg.Stencil.BiLaplacian, 0.01, SWEEPS, True,
                 threads=oracle.num_threads())
    for k, b in enumerate(fine):
        assert np.array_equal(got[k], host.block_array(int(b))), int(b)


def test_learned_solve_256_reaches_1e6(msbg, ctx, oracle):
    from msbg_rs_b200 import workloads
    size = 256
    ft = workloads.flip_transfer(size=size, bsx=16, particles=False)
    active = np.unique(ft.fine_blocks)
    b = workloads.smooth_divergence_rhs(size, 16, active, seed=4).reshape(-1).astype(np.float32)
    P = msbg.Poisson(ctx, size, size, size, 16, active)
    net = msbg.UNet(ctx, size, size, size, active, seed=1)
    P.set_preconditioner(net)
    P.train_preconditioner(n_rhs=20, mg_iters=40, steps_per_rhs=40, pool=64, lr=1e-3, target=1, seed=7)
    P.set_network_lead(1)
    # the FP64 solution: rounding x to f32 alone would leave ~1e-5 here
    x64 = torch.zeros(P.n, dtype=torch.float64, device="cuda")
    it, rel, _ = P.solve_device(x64, torch.from_numpy(b).cuda(), method=msbg.LEARNED_LEAD, tol=1e-6, max_iter=200)
    assert rel <= 1e-6 and it < 200
    nb = size // 16
    ax = oracle.poisson_matvec(active.astype(np.int64), nb, nb, nb, 16, x64.cpu().numpy())
    bb = b.astype(np.float64)
    assert np.linalg.norm(bb - ax) / np.linalg.norm(bb) <= 1.5e-6
    P.close()
    net.close()


def test_batched_64_problems_1e8(msbg, ctx, oracle):
    from msbg_rs_b200 import workloads
    probs = workloads.batched_problems(n=64, seed=3)
    B = msbg.Batch(ctx, [(d, bs, a) for d, bs, a, _ in probs], tune=True)
    for p, (_, _, _, b) in enumerate(probs):
        B.set_rhs(p, b)
    its, rel, _ = B.solve(tol=1e-8, iters_per_cycle=8, max_cycles=60)
    assert np.all(rel <= 1e-8), rel.max()
    # the smallest problem on a 256^3 domain against the FP64 oracle
    big = [p for p in range(len(probs)) if probs[p][0][0] == 256]
    assert big
    p = min(big, key=lambda q: len(probs[q][2]) * probs[q][1] ** 3)
    dims, bs, act, b = probs[p]
    n = dims[0] // bs
    xo, _ = oracle.poisson_solve(act.astype(np.int64), n, n, n, bs, b.reshape(-1).astype(np.float64), mode=1,
                                 tol=1e-10, max_iter=200)
    x = B.solution(p)
    err = np.linalg.norm(x - xo) / np.linalg.norm(xo)
    print(f"problem {p}: {len(act)} blocks of {bs}^3, relative error against the FP64 oracle {err:.3g}")
    assert err <= 1e-6
    B.close()
