"""Payload gather of a sort permutation (the gather of bucket_particles,
fluid/mod.rs:71-91): msbg_permute_device for rows of 1, 3 and 5 floats,
bit-exact against numpy indexing."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("width", [1, 3, 5])
@pytest.mark.parametrize("n", [1, 1000, 300001])
def test_permute_rows(msbg, ctx, n, width):
    import torch
    rng = np.random.default_rng(n + width)
    perm = rng.permutation(n).astype(np.uint32)
    src = rng.standard_normal((n, width)).astype(np.float32)
    d_perm = torch.from_numpy(perm.view(np.int32)).cuda()
    d_src = torch.from_numpy(src).cuda()
    d_dst = torch.empty_like(d_src)
    msbg._lib.call("msbg_permute_device", ctx.handle, msbg._lib.ptr(d_perm), n, width, msbg._lib.ptr(d_src),
                   msbg._lib.ptr(d_dst))
    ctx.synchronize()
    assert np.array_equal(d_dst.cpu().numpy().view(np.uint32), src[perm].view(np.uint32))
