"""Sampler (math/sample.rs:600-649): a grid bound to an alignment and a
boundary condition, sampled with trilinear or cubic B-spline reconstruction
(values, gradients, the cubic Hessian) on the device."""
from __future__ import annotations

import numpy as np

from .grid import SparseGrid

LINEAR, CUBIC_BSPLINE = 0, 1  # Interpolation (math/boundary.rs)
CORNER, CELL_CENTERED = 0, 1  # GridAlignment


class Sampler:
    """Sampler::new(grid, align, bc) with sample::<IP>, gradient::<IP> and
    hessian.  Cubic reconstruction is cell-centred whatever the alignment,
    as in the crate."""

    def __init__(self, grid: SparseGrid, align: int, bc: int):
        self.grid, self.align, self.bc = grid, int(align), int(bc)

    def sample(self, pos, interp: int = LINEAR) -> np.ndarray:
        if interp == LINEAR:
            return self.grid.sample_linear(pos, self.align, self.bc)
        return self.grid.sample_ext(pos, 0, self.align, self.bc)

    def gradient(self, pos, interp: int = LINEAR) -> np.ndarray:
        return self.grid.sample_ext(pos, 3 if interp == LINEAR else 1, self.align, self.bc)

    def hessian(self, pos) -> np.ndarray:
        """[n][6]: fxx, fyy, fzz, fxy, fxz, fyz."""
        return self.grid.sample_ext(pos, 2, self.align, self.bc)
