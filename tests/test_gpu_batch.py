"""Batched Poisson solves (the whole solve one CUDA graph launch with a
device-side loop over cycles, per-problem CG scalars on the device,
autotuned launch shapes) against the FP64 oracle.

No reference exists (parity unpinned).  Checked per problem: the solve
reaches relative residual 1e-8, re-measured in FP64 on the host with the
oracle's operator; the solution agrees with the oracle's FP64 solve within
1e-6 (relative L2); problems do not leak into each other (a problem solved
alone gives the same solution); a second solve reuses the captured graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problems():
    from conftest import load_package
    load_package()
    from msbg_rs_b200 import workloads
    return workloads.batched_problems(n=7, seed=5, edges=(32, 64), block_sizes=(8, 16), fraction=(0.2, 0.6))


@pytest.fixture(scope="module")
def solved(msbg, ctx, problems):
    B = msbg.Batch(ctx, [(d, bs, a) for d, bs, a, _ in problems], tune=True)
    for p, (_, _, _, b) in enumerate(problems):
        B.set_rhs(p, b)
    its, rel, cyc = B.solve(tol=1e-8, iters_per_cycle=8, max_cycles=40)
    return B, its, rel, cyc


def test_batch_reaches_tolerance_and_matches_oracle(oracle, problems, solved):
    B, its, rel, cyc = solved
    assert cyc > 0 and np.all(rel <= 1e-8), rel
    for p, (dims, bs, act, b) in enumerate(problems):
        n = dims[0] // bs
        x = B.solution(p)
        a64 = act.astype(np.int64)
        ax = oracle.poisson_matvec(a64, n, n, n, bs, x)
        bb = b.reshape(-1).astype(np.float64)
        assert np.linalg.norm(bb - ax) / np.linalg.norm(bb) <= 2e-8
        xo, _ = oracle.poisson_solve(a64, n, n, n, bs, bb, mode=1, tol=1e-12, max_iter=400)
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-6


def test_tuning_is_reported(solved):
    B = solved[0]
    for g in range(B.n_groups):
        cfg, cells = B.tuning(g)
        assert len(cfg) == len(cells) >= 2
        assert np.all((cfg[:, :2] >= 0) & (cfg[:, :2] < 8))
        assert np.all(np.isin(cfg[:, 2], [0, 2, 4, 8, 16]))
        assert np.all(np.diff(cells.astype(np.int64)) <= 0)
    # a group of 16^3 blocks tunes the tile kernel's depth on its finest level
    assert any(B.tuning(g)[0][0, 2] in (2, 4, 8, 16) for g in range(B.n_groups))


def test_problems_are_independent(msbg, ctx, problems, solved):
    """Problem 0 solved alone through the single-problem solver gives the
    same solution as inside the batch."""
    import torch
    B = solved[0]
    dims, bs, act, b = problems[0]
    P = msbg.Poisson(ctx, *dims, bs, act)
    x = torch.zeros(P.n, dtype=torch.float64, device="cuda")
    P.solve_device(x, torch.from_numpy(b.reshape(-1)).cuda(), method=msbg.PCG, tol=1e-10, max_iter=200)
    xs = x.cpu().numpy()
    assert np.linalg.norm(B.solution(0) - xs) / np.linalg.norm(xs) <= 1e-6


def test_second_solve_reuses_graph(problems, solved):
    B = solved[0]
    rng = np.random.default_rng(9)
    for p, (_, _, _, b) in enumerate(problems):
        B.set_rhs(p, rng.uniform(-1, 1, b.size).astype(np.float32))
    its, rel, cyc = B.solve(tol=1e-8, iters_per_cycle=8, max_cycles=40)
    assert np.all(rel <= 1e-8) and cyc > 0


def test_device_loop_stops_at_the_cycle_limit(msbg, ctx, problems):
    """The loop's test runs on the device: with a limit of 0 no cycle runs,
    with a limit of 1 exactly one runs and the problems stay unconverged;
    the cycles it reports are the ones it ran (a resumed solve finishes)."""
    B = msbg.Batch(ctx, [(d, bs, a) for d, bs, a, _ in problems], tune=False)
    for p, (_, _, _, b) in enumerate(problems):
        B.set_rhs(p, b)
    its, rel, cyc = B.solve(tol=1e-8, iters_per_cycle=2, max_cycles=0)
    assert cyc == 0 and np.all(rel > 1e-8) and np.all(its == 0)
    its, rel, cyc = B.solve(tol=1e-8, iters_per_cycle=2, max_cycles=1)
    assert cyc == 1 and np.all(rel > 1e-8) and np.all(its > 0)
    its, rel, cyc = B.solve(tol=1e-8, iters_per_cycle=2, max_cycles=200, zero_x=False)
    assert cyc > 1 and np.all(rel <= 1e-8)
    B.close()


def test_single_problem_and_single_block(msbg, ctx, oracle):
    """A batch of one problem, and a problem of one block next to a larger one."""
    rng = np.random.default_rng(21)
    probs = [((32, 32, 32), 8, np.array([13], np.uint64)), ((64, 64, 64), 16, np.array([0, 1, 2, 5, 6], np.uint64))]
    for subset in ([probs[0]], probs):
        B = msbg.Batch(ctx, subset, tune=False)
        rhs = []
        for p, (dims, bs, act) in enumerate(subset):
            b = rng.uniform(-1, 1, len(act) * bs ** 3).astype(np.float32)
            rhs.append(b)
            B.set_rhs(p, b)
        its, rel, cyc = B.solve(tol=1e-8, iters_per_cycle=4, max_cycles=50)
        assert np.all(rel <= 1e-8)
        for p, (dims, bs, act) in enumerate(subset):
            n = dims[0] // bs
            x = B.solution(p)
            ax = oracle.poisson_matvec(act.astype(np.int64), n, n, n, bs, x)
            bb = rhs[p].astype(np.float64)
            assert np.linalg.norm(bb - ax) / np.linalg.norm(bb) <= 2e-8
        B.close()
