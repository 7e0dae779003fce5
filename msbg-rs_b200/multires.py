"""Multiresolution helper on the device: downsample_channel_avg
(multires/downsample.rs:13-59), the 2^3 box-average restriction of one level's
blocks to the next coarser level."""
from __future__ import annotations

from ._lib import call
from .grid import SparseGrid


def downsample_channel_avg(dst: SparseGrid, src: SparseGrid) -> None:
    """Every value block of src gets a dst block (half the block size) holding
    the 2^3 mean."""
    call("msbg_downsample_avg", dst.handle, src.handle)
