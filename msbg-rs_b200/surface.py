"""Surface reconstruction from particles on the device (particles/mod.rs:113-302):
SurfaceConfig, the instanced placement `place` (particles/sort.rs:31-144),
the min-splat of normalised squared distances (particles/splat.rs:92-319),
`finalize` (particles/finalize.rs:35-71) and reconstruct_and_smooth.  The
density grid is a SparseGrid of Density (u16), Density8 (u8) or f32 values with empty value
0 and full value 1 (the crate's D::empty() and D::full())."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import call, ptr
from .grid import Context, SparseGrid


@dataclass
class SurfaceConfig:
    """SurfaceConfig (particles/mod.rs:113-163)."""
    sx: int
    sy: int
    sz: int
    n_instances: int = 0
    instance_scale_factor: float = 0.01
    r_particle: float = 2.0
    nb_dist: float = 2.0
    n_smooth_iters: int = 5
    smooth_dt: float = 0.05

    @property
    def r_scan(self) -> float:
        return self.r_particle + self.nb_dist


def place(ctx: Context, base: np.ndarray, bbox_min, span_max: float, cfg: SurfaceConfig) -> np.ndarray:
    """Instanced placement of the base cloud (particles/sort.rs:31-144):
    positions [n][3] f32, instance-major; n_instances 0 means one instance per
    base point."""
    b = np.ascontiguousarray(base, np.float32).reshape(-1, 3)
    bb = np.ascontiguousarray(bbox_min, np.float32).reshape(3)
    n_inst = cfg.n_instances or len(b)
    n = C.c_size_t()
    call("msbg_place_instances", ctx.handle, ptr(b), len(b), ptr(bb), float(span_max), cfg.sx, cfg.sy, cfg.sz,
         float(cfg.instance_scale_factor), n_inst, None, 0, C.byref(n))
    out = np.empty((n.value, 3), np.float32)
    call("msbg_place_instances", ctx.handle, ptr(b), len(b), ptr(bb), float(span_max), cfg.sx, cfg.sy, cfg.sz,
         float(cfg.instance_scale_factor), n_inst, ptr(out), n.value, C.byref(n))
    return out


def splat_device(grid: SparseGrid, d_pos, n: int, cfg: SurfaceConfig) -> np.ndarray:
    """splat (particles/splat.rs:92-319) of device positions [n][3]: allocates
    the footprint blocks, fills them with the full value and takes the minimum
    of the quantised dist_sq / r_scan^2; returns the active bids."""
    act = np.empty(grid.n_blocks, np.uint64)
    na = C.c_size_t()
    call("msbg_surface_splat_device", grid.handle, ptr(d_pos), int(n), float(cfg.r_particle), float(cfg.nb_dist),
         ptr(act), len(act), C.byref(na))
    return act[: na.value].copy()


def finalize(grid: SparseGrid, active, cfg: SurfaceConfig) -> None:
    """finalize (particles/finalize.rs:35-71) of the listed blocks, in place."""
    a = np.ascontiguousarray(active, np.uint64)
    call("msbg_surface_finalize", grid.handle, ptr(a), len(a), float(cfg.r_particle), float(cfg.nb_dist))


def reconstruct_and_smooth(grid: SparseGrid, positions: np.ndarray, cfg: SurfaceConfig) -> np.ndarray:
    """Splat, finalize and cfg.n_smooth_iters mean-curvature sweeps with
    [0, 1] clamping (particles/mod.rs:279-302) of host positions; returns the
    active bids."""
    p = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    act = np.empty(grid.n_blocks, np.uint64)
    na = C.c_size_t()
    call("msbg_reconstruct_and_smooth", grid.handle, ptr(p), len(p), float(cfg.r_particle), float(cfg.nb_dist),
         int(cfg.n_smooth_iters), float(cfg.smooth_dt), ptr(act), len(act), C.byref(na))
    return act[: na.value].copy()
