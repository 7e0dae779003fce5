"""msbg_morton_sort_noalloc_device: the Morton sort for callers that cannot
allocate device memory on the calling path (real-time loops, allocator
callbacks, processes whose device memory is reserved up front).  Its
temporaries live in a fixed scratch array inside the library, so it takes at
most 262144 particles.  Checked through the C ABI against the allocating
entry point, msbg_morton_sort_device, on two calls in a row: the sorts are
integer work, so the results must be equal bit for bit.  This file is
collected last so that a run stopping at the first failure has already run
every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 262144


def _sorts(msbg, ctx, dpos, n):
    import torch

    lib = msbg._lib.lib()
    ptr = msbg._lib.ptr
    k_fixed = torch.empty(n, dtype=torch.int64, device="cuda")
    p_fixed = torch.empty(n, dtype=torch.int32, device="cuda")
    k_alloc = torch.empty_like(k_fixed)
    p_alloc = torch.empty_like(p_fixed)
    msbg._lib.check(lib.msbg_morton_sort_noalloc_device(ctx.handle, ptr(dpos), C.c_size_t(n), ptr(k_fixed), ptr(p_fixed)))
    msbg._lib.check(lib.msbg_morton_sort_device(ctx.handle, ptr(dpos), C.c_size_t(n), ptr(k_alloc), ptr(p_alloc)))
    ctx.synchronize()
    return k_fixed, p_fixed, k_alloc, p_alloc


def test_noalloc_morton_sort_matches_allocating_entry_point(msbg, ctx):
    import torch

    rng = np.random.default_rng(2024)
    # two calls in a row: a full-size call, then a smaller one that reuses the
    # scratch array the first call left behind
    for n, extent in ((MAX_PARTICLES, 400.0), (70001, 64.0)):
        pos = rng.uniform(0.0, extent, (n, 3)).astype(np.float32)
        pos[: n // 8] = pos[n // 8: 2 * (n // 8)]  # repeated keys: the sort must be stable
        dpos = torch.from_numpy(pos).cuda()
        k_fixed, p_fixed, k_alloc, p_alloc = _sorts(msbg, ctx, dpos, n)
        assert torch.equal(k_fixed, k_alloc)
        assert torch.equal(p_fixed, p_alloc)


def test_noalloc_morton_sort_allocates_nothing(msbg):
    """On a fresh context the call leaves the context's scratch arena empty,
    and once the library's kernels are loaded, further calls leave the
    device's free memory unchanged."""
    import torch

    lib = msbg._lib.lib()
    ptr = msbg._lib.ptr
    fresh = msbg.Context(0)
    try:
        n = 50000
        pos = np.random.default_rng(7).uniform(0.0, 100.0, (n, 3)).astype(np.float32)
        dpos = torch.from_numpy(pos).cuda()
        keys = torch.empty(n, dtype=torch.int64, device="cuda")
        perm = torch.empty(n, dtype=torch.int32, device="cuda")
        used = C.c_uint64()

        def run():
            msbg._lib.check(lib.msbg_morton_sort_noalloc_device(fresh.handle, ptr(dpos), C.c_size_t(n), ptr(keys),
                                                                ptr(perm)))

        run()
        msbg._lib.check(lib.msbg_ctx_scratch_bytes(fresh.handle, C.byref(used)))
        assert used.value == 0
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        run()
        run()
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free_before
        msbg._lib.check(lib.msbg_ctx_scratch_bytes(fresh.handle, C.byref(used)))
        assert used.value == 0
    finally:
        fresh.close()


def test_noalloc_morton_sort_rejects_oversize(msbg, ctx):
    import torch

    n = MAX_PARTICLES + 1
    dpos = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    keys = torch.empty(n, dtype=torch.int64, device="cuda")
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    lib = msbg._lib.lib()
    st = lib.msbg_morton_sort_noalloc_device(ctx.handle, msbg._lib.ptr(dpos), C.c_size_t(n), msbg._lib.ptr(keys),
                                             msbg._lib.ptr(perm))
    assert st == msbg._lib.MSBG_ERR_ARG
    assert b"exceeds the maximum" in lib.msbg_last_error()
