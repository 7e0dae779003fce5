"""Particle sorting on the device: morton3 (multires/sort.rs:20-22), the
per-particle Morton sort, bucket_indices (particles/sort.rs:174-269) and
sort_block_list_morton (multires/sort.rs:35-57)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import call, ptr
from .grid import Context


def morton3_host(x: int, y: int, z: int) -> int:
    """63-bit Morton code, 21 bits per axis (multires/sort.rs:8-22), on the host."""

    def spread(v: int) -> int:
        v &= 0x1FFFFF
        v = (v | (v << 32)) & 0x001F00000000FFFF
        v = (v | (v << 16)) & 0x001F0000FF0000FF
        v = (v | (v << 8)) & 0x100F00F00F00F00F
        v = (v | (v << 4)) & 0x10C30C30C30C30C3
        v = (v | (v << 2)) & 0x1249249249249249
        return v

    return spread(x) | (spread(y) << 1) | (spread(z) << 2)


def morton3(ctx: Context, xyz: np.ndarray) -> np.ndarray:
    """morton3 for an [n][3] u64 array, computed on the device."""
    a = np.ascontiguousarray(xyz, np.uint64).reshape(-1, 3)
    out = np.empty(len(a), np.uint64)
    call("msbg_morton3", ctx.handle, ptr(a), len(a), ptr(out))
    return out


def morton_sort(ctx: Context, pos: np.ndarray):
    """Stable sort of particles by morton3(trunc(p)): returns (sorted keys, perm)."""
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    keys = np.empty(len(p), np.uint64)
    perm = np.empty(len(p), np.uint32)
    call("msbg_morton_sort", ctx.handle, ptr(p), len(p), ptr(keys), ptr(perm))
    return keys, perm


@dataclass
class BucketPlan:
    """particles/sort.rs:163-167"""

    particle_blocks: np.ndarray
    starts: np.ndarray
    perm: np.ndarray


def bucket_indices(ctx: Context, bids) -> BucketPlan:
    """bucket_indices (particles/sort.rs:174-269); intra-block order = input order."""
    b = np.ascontiguousarray(bids, np.uint64)
    n = len(b)
    blocks = np.empty(max(n, 1), np.uint64)
    starts = np.empty(n + 1, np.uint64)
    perm = np.empty(max(n, 1), np.uint32)
    nb = C.c_size_t()
    call("msbg_bucket_indices", ctx.handle, ptr(b), n, ptr(blocks), ptr(starts), ptr(perm), C.byref(nb))
    k = nb.value
    return BucketPlan(blocks[:k].copy(), starts[: k + 1].copy(), perm[:n].copy())


def sort_block_list_morton(ctx: Context, blocks, nx: int, ny: int, levels: np.ndarray, n_levels: int) -> np.ndarray:
    """sort_block_list_morton (multires/sort.rs:35-57)."""
    b = np.array(blocks, np.uint64)
    lv = np.ascontiguousarray(levels, np.uint8)
    call("msbg_sort_block_list_morton", ctx.handle, ptr(b), len(b), int(nx), int(ny), ptr(lv), lv.size, int(n_levels))
    return b
