"""The learned preconditioner inside the pressure solve (methods LEARNED and
HYBRID), trained on the device on pairs the solver generates.

Parity is unpinned (the crate has no solver); what is checked: training
lowers the loss; the trained network's correction lowers the error a V-cycle
leaves (the gain over the method without it, measured on fresh right-hand
sides); learned and hybrid solves reach 1e-6 relative residual, re-measured
in FP64 on the host with the oracle's operator; an untrained network still
converges through the multigrid fallback."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def shell_blocks():
    import sys
    from conftest import load_package
    load_package()
    from msbg_rs_b200 import workloads
    return np.sort(workloads.shell_active_blocks(8, 16, 0.35 * 128, 12.0))


@pytest.fixture(scope="module")
def trained(msbg, ctx):
    act = shell_blocks()
    P = msbg.Poisson(ctx, 128, 128, 128, 16, act)
    net = msbg.UNet(ctx, 128, 128, 128, act, seed=3)
    P.set_preconditioner(net)
    hist = P.train_preconditioner(n_rhs=10, mg_iters=12, steps_per_rhs=30, pool=48, lr=1e-3, target=1, seed=5)
    return act, P, net, hist


def true_rel(oracle, act, x, b):
    ax = oracle.poisson_matvec(act.astype(np.int64), 8, 8, 8, 16, x.astype(np.float64))
    return np.linalg.norm(b - ax) / np.linalg.norm(b)


def test_training_lowers_loss(trained):
    act, P, net, hist = trained
    assert len(hist) == 300 and np.all(np.isfinite(hist))
    assert np.mean(hist[-30:]) < 0.7 * np.mean(hist[:30]), (np.mean(hist[:30]), np.mean(hist[-30:]))


def test_network_correction_beats_vcycle_alone(trained):
    act, P, net, hist = trained
    ev = P.eval_preconditioner(n_rhs=2, mg_iters=8, seed=77)
    assert ev["vcycle_plus_network"] < 0.9 * ev["vcycle"], ev


@pytest.mark.parametrize("method", ["HYBRID", "LEARNED", "LEARNED_MG", "LEARNED_LEAD"])
def test_learned_solves_reach_tolerance(msbg, oracle, trained, method):
    import torch
    act, P, net, hist = trained
    P.set_network_lead(2)
    b = torch.empty(P.n, device="cuda")
    P.rhs(b, seed=12345)
    x = torch.zeros(P.n, device="cuda", dtype=torch.float64)
    it, rel, h = P.solve_device(x, b, method=getattr(msbg, method), tol=1e-6, max_iter=200)
    assert rel <= 1e-6 and it < 200
    assert true_rel(oracle, act, x.cpu().numpy(), b.cpu().numpy().astype(np.float64)) <= 2e-6
    st = P.solve_stats()
    assert st["network"] > 0


def test_untrained_network_falls_back_and_converges(msbg, ctx, oracle):
    import torch
    act = shell_blocks()
    P = msbg.Poisson(ctx, 128, 128, 128, 16, act)
    net = msbg.UNet(ctx, 128, 128, 128, act, seed=11)
    net.set_output_scale(1e3)
    P.set_preconditioner(net)
    b = torch.empty(P.n, device="cuda")
    P.rhs(b, seed=4242)
    x = torch.zeros(P.n, device="cuda", dtype=torch.float64)
    it, rel, h = P.solve_device(x, b, method=msbg.LEARNED, tol=1e-6, max_iter=300)
    assert rel <= 1e-6
    assert true_rel(oracle, act, x.cpu().numpy(), b.cpu().numpy().astype(np.float64)) <= 2e-6


def test_preconditioner_must_match_blocks(msbg, ctx):
    act = shell_blocks()
    P = msbg.Poisson(ctx, 128, 128, 128, 16, act)
    net = msbg.UNet(ctx, 128, 128, 128, act[:-1], seed=1)
    with pytest.raises(msbg.MsbgError):
        P.set_preconditioner(net)
    with pytest.raises(msbg.MsbgError):
        import torch
        b = torch.ones(P.n, device="cuda")
        x = torch.zeros(P.n, device="cuda")
        P.solve_device(x, b, method=msbg.LEARNED)


def test_network_lead_counts_and_restart(msbg, oracle, trained):
    """LEARNED_LEAD applies the network exactly k times, then finishes with
    V-cycles; k = 0 is plain MG-preconditioned CG (same iterations)."""
    import torch
    act, P, net, hist = trained
    b = torch.empty(P.n, device="cuda")
    P.rhs(b, seed=2024)
    x = torch.zeros(P.n, device="cuda", dtype=torch.float64)
    for k in (1, 3, -1):
        x.zero_()
        P.set_network_lead(k)
        it, rel, h = P.solve_device(x, b, method=msbg.LEARNED_LEAD, tol=1e-6, max_iter=200)
        st = P.solve_stats()
        assert rel <= 1e-6 and st["network"] == abs(k), (k, st)
        assert true_rel(oracle, act, x.cpu().numpy(), b.cpu().numpy().astype(np.float64)) <= 2e-6
    x.zero_()
    P.set_network_lead(0)
    it0, rel0, _ = P.solve_device(x, b, method=msbg.LEARNED_LEAD, tol=1e-6, max_iter=200)
    x.zero_()
    it1, rel1, _ = P.solve_device(x, b, method=msbg.PCG, tol=1e-6, max_iter=200)
    assert it0 == it1 and P.solve_stats()["network"] == 0
