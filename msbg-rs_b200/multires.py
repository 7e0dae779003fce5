"""Multiresolution helpers on the device: downsample_channel_avg
(multires/downsample.rs:13-59), the 2^3 box-average restriction of one level's
blocks to the next coarser level, and the refinement map
(multires/refinement.rs): 2:1 regularisation and block topology."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call, ptr
from .grid import Context, SparseGrid

DOM_BORDER, COARSE_FINE, FINE_COARSE, EXISTS = 1 << 1, 1 << 2, 1 << 3, 1 << 12


def regularize_refinement_map(ctx: Context, levels: np.ndarray, nx: int, ny: int, nz: int, n_levels: int) -> np.ndarray:
    """regularize_refinement_map (refinement.rs:63-107) of a per-block level
    map; returns the regularised copy."""
    m = np.ascontiguousarray(levels, np.uint8).copy()
    call("msbg_regularize_refinement_map", ctx.handle, ptr(m), nx, ny, nz, int(n_levels))
    return m


def block_topology(ctx: Context, levels: np.ndarray, nx: int, ny: int, nz: int, n_levels: int, user_flags=None):
    """compute_block_topology (refinement.rs:124-208): (flags [n] u16,
    FINE_COARSE block lists per level in block order, EXISTS count)."""
    m = np.ascontiguousarray(levels, np.uint8)
    n = len(m)
    u = None if user_flags is None else np.ascontiguousarray(user_flags, np.uint16)
    flags = np.zeros(n, np.uint16)
    fc = np.zeros((n_levels, n), np.uint64)
    cnt = np.zeros(n_levels, np.uint64)
    ex = C.c_uint64()
    call("msbg_block_topology", ctx.handle, ptr(m), nx, ny, nz, int(n_levels), ptr(u), ptr(flags), ptr(fc), ptr(cnt),
         C.byref(ex))
    return flags, [fc[l, : int(cnt[l])].copy() for l in range(n_levels)], ex.value


def downsample_channel_avg(dst: SparseGrid, src: SparseGrid) -> None:
    """Every value block of src gets a dst block (half the block size) holding
    the 2^3 mean."""
    call("msbg_downsample_avg", dst.handle, src.handle)
