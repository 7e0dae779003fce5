"""In-place 8-colour PDE smoothing: the device counterpart of solver.rs:141-267.

`Sweeper(grid).sweep(active, Stencil.X, PdeParams(dt, iterations, clamp))`
runs `iterations` full 8-colour sweeps on the GPU.  Semantics follow the
reference: colour = bx&1 | (by&1)<<1 | (bz&1)<<2, Neumann boundary, blocks
of `active` that are not value blocks are skipped, Gauss-Seidel across
colours and Jacobi inside a block on the staged halo snapshot.  The call
enqueues the sweep on the grid's context stream and returns.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import call, ptr
from .grid import SparseGrid


class Stencil(enum.IntEnum):
    """solver.rs:44-51"""

    Laplacian = _lib.MSBG_LAPLACIAN
    MeanCurvature = _lib.MSBG_MEAN_CURVATURE
    BiLaplacian = _lib.MSBG_BILAPLACIAN


class Fence(enum.Enum):
    """solver.rs:68-80.  Kept for API parity: on the GPU consecutive colour
    phases are ordered by the stream, so every variant behaves like Sfence."""

    Sfence = "sfence"
    Mfence = "mfence"
    None_ = "none"


@dataclass
class PdeParams:
    """solver.rs:53-61"""

    dt: float
    iterations: int
    do_constr_zero_one: bool = False


class Sweeper:
    """Sweeper::new(grid, num_threads, fence) (solver.rs:154-160)."""

    def __init__(self, grid: SparseGrid, num_threads: int = 0, fence: Fence = Fence.Sfence,
                 seed: int = 0xDEADBEEF, lanes: int = 16):
        """`seed` and `lanes` set the Density8 store's generator: the slot of
        the reference's first sweeping thread is SimdRng::<LANES>::seed(
        0xdeadbeef) (solver.rs:109-119), LANES the build's SIMD width."""
        self.grid = grid
        self.fence = fence
        self.seed = int(seed) & 0xFFFFFFFF
        self.lanes = int(lanes)
        self.stream_pos = 0  # generator draws taken so far (Density8 only)

    def sweep(self, active, stencil: Stencil, params: PdeParams) -> None:
        """Sweeper::sweep (solver.rs:166-185); a Density8 grid continues this
        sweeper's generator stream across calls."""
        a = np.ascontiguousarray(active, np.uint64)
        pos = C.c_uint64(self.stream_pos)
        call("msbg_sweep_stochastic", self.grid.handle, ptr(a), len(a), int(stencil), float(params.dt),
             int(params.iterations), int(bool(params.do_constr_zero_one)), self.seed, self.lanes, C.byref(pos))
        self.stream_pos = pos.value

    def sweep_multires(self, coarse: SparseGrid, levels: np.ndarray, active, stencil: Stencil, params: PdeParams) -> None:
        """Sweep whose halos sample coarser neighbours from `coarse`
        (fill_multires, multires/halo.rs:187-358)."""
        a = np.ascontiguousarray(active, np.uint64)
        lv = np.ascontiguousarray(levels, np.uint8)
        assert lv.size >= self.grid.n_blocks
        call("msbg_sweep_multires", self.grid.handle, coarse.handle, ptr(lv), ptr(a), len(a), int(stencil),
             float(params.dt), int(params.iterations), int(bool(params.do_constr_zero_one)))


def apply_pde(grid: SparseGrid, active, stencil: Stencil, params: PdeParams, num_threads: int = 0,
              fence: Fence = Fence.Sfence) -> None:
    """apply_pde (solver.rs:228-240)."""
    Sweeper(grid, num_threads, fence).sweep(active, stencil, params)
