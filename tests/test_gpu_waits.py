"""Bounded device waits: a wait on counts that nothing publishes gives up after
its time limit, the call returns MSBG_ERR_TIMEOUT with the status word
cleared, and the same context then sorts correctly.  The waiting CTA reads a
flag that is never set (no fault, no trap), as the radix-sort look-back does
when a predecessor tile is late."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_lookback_wait_times_out_and_context_recovers(msbg, ctx, oracle):
    lib = msbg._lib.lib()
    st = lib.msbg_test_sort_lookback_timeout(ctx.handle, C.c_uint64(2_000_000))  # 2 ms
    assert st == msbg._lib.MSBG_ERR_TIMEOUT
    assert b"radix-sort look-back" in lib.msbg_last_error()
    # the status word was cleared: a normal sort on the same context succeeds
    pos = np.random.default_rng(11).uniform(0.0, 200.0, (30000, 3)).astype(np.float32)
    keys, perm = msbg.morton_sort(ctx, pos)
    want_k, want_p = oracle.morton_sort(pos)
    assert np.array_equal(keys, want_k) and np.array_equal(perm, want_p)


def test_lookback_timeout_limit_is_checked(msbg, ctx):
    lib = msbg._lib.lib()
    assert lib.msbg_test_sort_lookback_timeout(ctx.handle, C.c_uint64(10)) == msbg._lib.MSBG_ERR_ARG
