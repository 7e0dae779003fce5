"""msbg-rs_b200: the msbg-rs sparse-grid hot path on B200 (sm_100a).

Host-side mirror of the crate's API over the C ABI in include/msbg_cuda.h:
sparse grids and halo gathers (sparse_grid.rs, multires/halo.rs), the
8-colour smoother (solver.rs), Morton/bucket sorts (multires/sort.rs,
particles/sort.rs), P2G/G2P on the MAC grid (fluid/) and the 2^3 downsample
(multires/downsample.rs).  All compute runs in libmsbg_cuda.so; importing the
package does not load it, the first call does (and fails loudly when it has
not been built).

The package directory name contains a hyphen, so it is loaded under the
module name `msbg_rs_b200` (see load_package in tests/conftest.py, bench.py).
"""
from . import _lib
from .grid import Context, HostGrid, SparseGrid
from .solver import Fence, PdeParams, Stencil, Sweeper, apply_pde
from .particles import BucketPlan, bucket_indices, morton3, morton3_host, morton_sort, sort_block_list_morton
from .fluid import (FlipStep, MacGrid, MacSampler, X, Y, Z, g2p_blend, g2p_blend_device, g2p_flip_device,
                    particles_to_grid, particles_to_grid_device, particles_to_grid_sorted_device,
                    particles_to_grid_permuted_device)
from .multires import downsample_channel_avg
from .sampler import CELL_CENTERED, CORNER, CUBIC_BSPLINE, LINEAR, Sampler
from . import surface
from .surface import SurfaceConfig, reconstruct_and_smooth
from .poisson import HYBRID, LEARNED, LEARNED_LEAD, LEARNED_MG, MG, PCG, Poisson
from .learned import UNet
from .batch import Batch
from .blockmap import BlockMap

MsbgError = _lib.MsbgError
CLAMP, NEUMANN, DIRICHLET = _lib.MSBG_CLAMP, _lib.MSBG_NEUMANN, _lib.MSBG_DIRICHLET

__all__ = [
    "Context", "HostGrid", "SparseGrid", "Fence", "PdeParams", "Stencil", "Sweeper", "apply_pde",
    "BucketPlan", "bucket_indices", "morton3", "morton3_host", "morton_sort", "sort_block_list_morton",
    "FlipStep", "MacGrid", "MacSampler", "X", "Y", "Z", "g2p_blend", "g2p_blend_device", "g2p_flip_device",
    "particles_to_grid",
    "particles_to_grid_device", "particles_to_grid_sorted_device", "particles_to_grid_permuted_device", "downsample_channel_avg", "MsbgError", "CLAMP", "NEUMANN", "DIRICHLET",
    "surface", "SurfaceConfig", "reconstruct_and_smooth", "Sampler", "LINEAR", "CUBIC_BSPLINE", "CORNER", "CELL_CENTERED",
    "Poisson", "MG", "PCG", "LEARNED", "HYBRID", "LEARNED_MG", "LEARNED_LEAD", "UNet", "Batch", "BlockMap",
]
