"""Refinement map on the device (multires/refinement.rs:63-208): the crate's
known answers, and bit-exact agreement with the oracle on random maps (2:1
regularisation, block flags, FINE_COARSE lists in block order, EXISTS count),
including the 4-level map of the phase-field layout."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_refinement_known_answers_on_device(msbg, ctx):
    from msbg_rs_b200 import multires as mr
    n = 4
    m = np.full(n ** 3, 1, np.uint8)
    m[21] = 0
    m = mr.regularize_refinement_map(ctx, m, n, n, n, 3)
    flags, fc, _ = mr.block_topology(ctx, m, n, n, n, 3)
    assert m[21] == 0 and flags[21] & mr.FINE_COARSE and not flags[21] & mr.COARSE_FINE
    assert fc[0].tolist() == [21]
    assert m[63] == 1 and not flags[63] & (mr.FINE_COARSE | mr.COARSE_FINE)
    flags, _, _ = mr.block_topology(ctx, np.zeros(n ** 3, np.uint8), n, n, n, 3)
    assert flags[0] & mr.DOM_BORDER and flags[63] & mr.DOM_BORDER and not flags[21] & mr.DOM_BORDER


@pytest.mark.parametrize("dims,n_levels", [((8, 8, 8), 3), ((17, 9, 13), 4), ((32, 32, 32), 5), ((5, 7, 3), 2)])
def test_refinement_matches_oracle(msbg, ctx, oracle, dims, n_levels):
    from msbg_rs_b200 import multires as mr
    nx, ny, nz = dims
    r = np.random.default_rng(nx * ny + n_levels)
    m = r.integers(0, n_levels, nx * ny * nz).astype(np.uint8)
    got = mr.regularize_refinement_map(ctx, m, nx, ny, nz, n_levels)
    want = oracle.regularize_refinement_map(m, nx, ny, nz, n_levels)
    assert np.array_equal(got, want)
    user = (r.random(len(m)) < 0.3).astype(np.uint16) << 12
    f, fc, ex = mr.block_topology(ctx, got, nx, ny, nz, n_levels, user)
    wf, wfc, wex = oracle.block_topology(want, nx, ny, nz, n_levels, user)
    assert np.array_equal(f, wf) and ex == wex
    assert all(np.array_equal(a.astype(np.int64), b) for a, b in zip(fc, wfc))


def test_phase_field_layout_map(msbg, ctx, oracle):
    """The 4-level map of the 512^3 phase-field layout (32^3 blocks), regularised."""
    from msbg_rs_b200 import workloads
    lv = workloads.block_levels(512, 16, 0.3 * 512, bands=(16.0, 48.0)).astype(np.uint8)
    lv = np.minimum(lv + (lv == 2) * np.uint8(1), 3).astype(np.uint8)  # a level-3 band outside
    got = msbg.multires.regularize_refinement_map(ctx, lv, 32, 32, 32, 4)
    assert np.array_equal(got, oracle.regularize_refinement_map(lv, 32, 32, 32, 4))
