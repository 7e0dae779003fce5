"""Input fields and grids of the reference's own tests, restated for the parity
tests (the formulas are the reference's; the values are generated here)."""
from __future__ import annotations

import numpy as np


def stencil_field(x, y, z):
    """tests/difftest_stencil.rs:25-32 (f32 arithmetic)."""
    f = np.float32
    u = (np.asarray(x, np.int32) - 24).astype(f)
    v = (np.asarray(y, np.int32) - 24).astype(f)
    w = (np.asarray(z, np.int32) - 24).astype(f)
    q = f(0.01) * (u * u + f(2.0) * v * v + f(3.0) * w * w + u * v)
    r = f(0.001) * (u * u * u * u + v * v * v * v + w * w * w * w)
    return (q + r).astype(f)


def smoother_field(x, y, z):
    """tests/difftest_smoother.rs:22-24: sin(0.1x) cos(0.08y) sin(0.06z) in f32."""
    f = np.float32
    x = np.asarray(x, f)
    y = np.asarray(y, f)
    z = np.asarray(z, f)
    a = np.sin((f(0.1) * x).astype(f)).astype(f)
    b = np.cos((f(0.08) * y).astype(f)).astype(f)
    c = np.sin((f(0.06) * z).astype(f)).astype(f)
    return ((a * b).astype(f) * c).astype(f)


def interp_field(x, y, z):
    """tests/difftest_interp.rs:15-19 (f32, left-to-right)."""
    f = np.float32
    x = np.asarray(x, f)
    y = np.asarray(y, f)
    z = np.asarray(z, f)
    t = f(0.002) * x * x
    t = t + f(0.003) * y * y
    t = t + f(0.004) * z * z
    t = t + f(0.005) * x * y
    t = t + f(0.006) * x * z
    t = t + f(0.007) * y * z
    t = t + f(0.1) * x
    t = t + f(0.05) * y
    t = t - f(0.02) * z
    t = t + f(0.75)
    return t.astype(f)


def dense_grid(HostGrid, size, fn, bsx=16, empty=0.0, full=1.0, name="g"):
    """All blocks of a size^3 domain allocated with fn(x, y, z) in each voxel."""
    g = HostGrid(name, size, size, size, empty, full, bsx)
    b = bsx
    zz, yy, xx = np.meshgrid(np.arange(b), np.arange(b), np.arange(b), indexing="ij")
    for bid in range(g.n_blocks):
        bx, by, bz = g.get_block_coords_by_id(bid)
        g.ensure_block(bid)
        g.blocks[bid][:] = fn(bx * b + xx, by * b + yy, bz * b + zz).reshape(-1)
    return g
