"""Sparse block grid: the host-side mirror of `SparseGrid` (sparse_grid.rs:61-435)
and its device-resident counterpart behind the C ABI.

`HostGrid` keeps the crate's semantics on the host with numpy blocks: absent
blocks read the empty value, the full dummy the full value, value blocks their
data.  It builds inputs and inspects results.  `SparseGrid` owns an
`msbg_grid` (payload arena + block table in HBM) and moves blocks between the
two.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import call, ptr

DTYPES = {"f32": (_lib.MSBG_F32, np.float32), "u16": (_lib.MSBG_U16, np.uint16), "bf16": (_lib.MSBG_BF16, np.uint16),
          "u8": (_lib.MSBG_U8, np.uint8), "f16": (_lib.MSBG_F16, np.uint16)}


def _log2(v: int) -> int:
    assert v > 0 and (v & (v - 1)) == 0, "block size must be a power of two"
    return v.bit_length() - 1


class Context:
    """One CUDA device + stream (msbg_ctx)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        call("msbg_ctx_create", device, C.byref(h))
        self.handle = h
        self.device = device

    def synchronize(self) -> None:
        call("msbg_ctx_synchronize", self.handle)

    def stream(self) -> int:
        s = C.c_void_p()
        call("msbg_ctx_stream", self.handle, C.byref(s))
        return s.value or 0

    def kernel_launches(self) -> int:
        v = C.c_uint64()
        call("msbg_ctx_kernel_launches", self.handle, C.byref(v))
        return v.value

    def close(self) -> None:
        if self.handle:
            call("msbg_ctx_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HostGrid:
    """Host mirror of SparseGrid (sparse_grid.rs:61-435), numpy blocks."""

    def __init__(self, name, sx, sy, sz, empty_value=0.0, full_value=1.0, bsx=16, dtype="f32"):
        self.name = name
        self.sx, self.sy, self.sz = int(sx), int(sy), int(sz)
        self.bsx = int(bsx)
        self.log2 = _log2(self.bsx)
        self.nx = (self.sx + self.bsx - 1) >> self.log2
        self.ny = (self.sy + self.bsx - 1) >> self.log2
        self.nz = (self.sz + self.bsx - 1) >> self.log2
        self.nxy = self.nx * self.ny
        self.n_blocks = self.nxy * self.nz
        self.N = self.bsx ** 3
        self.dtype = dtype
        self.np_dtype = DTYPES[dtype][1]
        self.empty_value = float(empty_value)
        self.full_value = float(full_value)
        self.blocks: dict[int, np.ndarray] = {}
        self.full: set[int] = set()

    # sparse_grid.rs:157-175
    def get_block_id(self, x, y, z) -> int:
        return (x >> self.log2) + (y >> self.log2) * self.nx + (z >> self.log2) * self.nxy

    def get_voxel_id(self, x, y, z) -> int:
        m = self.bsx - 1
        return (x & m) | ((y & m) << self.log2) | ((z & m) << (2 * self.log2))

    def get_block_coords_by_id(self, bid):
        return bid % self.nx, (bid // self.nx) % self.ny, bid // self.nxy

    def _stored(self, v: float):
        if self.dtype == "f32":
            return np.float32(v)
        if self.dtype == "u16":
            r = np.floor(np.abs(np.float32(v) * np.float32(65535.0)) + 0.5) * np.sign(v)
            return np.uint16(min(max(r, 0.0), 65535.0))
        if self.dtype == "u8":  # Density8 from_unit (channel.rs:378-382)
            r = np.floor(np.abs(np.float32(v) * np.float32(255.0)) + 0.5) * np.sign(v)
            return np.uint8(min(max(r, 0.0), 255.0))
        if self.dtype == "f16":  # binary16 bits, round to nearest even
            return np.array([v], np.float32).astype(np.float16).view(np.uint16)[0]
        b = np.array([v], np.float32).view(np.uint32)[0]
        b = (int(b) + 0x7FFF + ((int(b) >> 16) & 1)) >> 16
        return np.uint16(b)

    def ensure_block(self, bid: int) -> None:
        """ensure_block (sparse_grid.rs:310-322)."""
        if bid not in self.blocks:
            self.full.discard(bid)
            self.blocks[bid] = np.full(self.N, self._stored(self.empty_value), self.np_dtype)

    def set_full_block(self, bid: int) -> None:
        assert bid not in self.blocks
        self.full.add(bid)

    def set_empty_block(self, bid: int) -> None:
        assert bid not in self.blocks
        self.full.discard(bid)

    def set_empty_value(self, v: float) -> None:
        self.empty_value = float(v)

    def set_full_value(self, v: float) -> None:
        self.full_value = float(v)

    def set_voxel(self, x, y, z, v) -> None:
        bid = self.get_block_id(x, y, z)
        self.ensure_block(bid)
        self.blocks[bid][self.get_voxel_id(x, y, z)] = v

    def get_voxel(self, x, y, z):
        bid = self.get_block_id(x, y, z)
        if bid in self.blocks:
            return self.blocks[bid][self.get_voxel_id(x, y, z)]
        return self._stored(self.full_value if bid in self.full else self.empty_value)

    def get_block_data(self, bid):
        return self.blocks.get(bid)

    def value_block_ids(self) -> list[int]:
        return sorted(self.blocks)

    def block_array(self, bid) -> np.ndarray:
        """Block contents as get_value_in_block sees them (dummies constant)."""
        if bid in self.blocks:
            return self.blocks[bid]
        return np.full(self.N, self._stored(self.full_value if bid in self.full else self.empty_value), self.np_dtype)

    def dense(self) -> np.ndarray:
        """Dense [sz][sy][sx] float array of get_voxel over the domain."""
        out = np.empty((self.nz * self.bsx, self.ny * self.bsx, self.nx * self.bsx), self.np_dtype)
        b = self.bsx
        for bz in range(self.nz):
            for by in range(self.ny):
                for bx in range(self.nx):
                    bid = bx + by * self.nx + bz * self.nxy
                    out[bz * b:(bz + 1) * b, by * b:(by + 1) * b, bx * b:(bx + 1) * b] = self.block_array(bid).reshape(b, b, b)
        return out[: self.sz, : self.sy, : self.sx]

    def table_and_data(self):
        """Dense block table (slot, -1 empty, -2 full) + [slots][N] payload."""
        table = np.full(self.n_blocks, -1, np.int32)
        ids = self.value_block_ids()
        data = np.zeros((max(len(ids), 1), self.N), self.np_dtype)
        for s, bid in enumerate(ids):
            table[bid] = s
            data[s] = self.blocks[bid]
        for bid in self.full:
            table[bid] = -2
        return table, data, ids

    def copy(self) -> "HostGrid":
        g = HostGrid(self.name, self.sx, self.sy, self.sz, self.empty_value, self.full_value, self.bsx, self.dtype)
        g.blocks = {k: v.copy() for k, v in self.blocks.items()}
        g.full = set(self.full)
        return g


class SparseGrid:
    """Device-resident sparse grid (msbg_grid): payload arena + block table in HBM."""

    def __init__(self, ctx: Context, sx, sy, sz, empty_value=0.0, full_value=1.0, bsx=16, dtype="f32", name="grid"):
        self.ctx = ctx
        self.name = name
        self.sx, self.sy, self.sz, self.bsx = int(sx), int(sy), int(sz), int(bsx)
        self.dtype = dtype
        self.np_dtype = DTYPES[dtype][1]
        self.N = self.bsx ** 3
        h = C.c_void_p()
        call("msbg_grid_create", ctx.handle, self.sx, self.sy, self.sz, self.bsx, DTYPES[dtype][0],
             float(empty_value), float(full_value), C.byref(h))
        self.handle = h
        self._owned = True
        d = self.dims()
        self.nx, self.ny, self.nz, self.n_blocks = d[3], d[4], d[5], d[6]
        self.nxy = self.nx * self.ny

    @classmethod
    def borrowed(cls, ctx: Context, handle, sx, sy, sz, bsx, dtype="f32", name="channel") -> "SparseGrid":
        g = cls.__new__(cls)
        g.ctx, g.name, g.handle, g._owned = ctx, name, handle, False
        g.sx, g.sy, g.sz, g.bsx, g.dtype = sx, sy, sz, bsx, dtype
        g.np_dtype = DTYPES[dtype][1]
        g.N = bsx ** 3
        d = g.dims()
        g.nx, g.ny, g.nz, g.n_blocks = d[3], d[4], d[5], d[6]
        g.nxy = g.nx * g.ny
        return g

    @classmethod
    def from_host(cls, ctx: Context, host: HostGrid) -> "SparseGrid":
        g = cls(ctx, host.sx, host.sy, host.sz, host.empty_value, host.full_value, host.bsx, host.dtype, host.name)
        ids = np.array(host.value_block_ids(), np.uint64)
        if len(ids):
            g.write_blocks(ids, np.stack([host.blocks[int(b)] for b in ids]))
        if host.full:
            full = np.array(sorted(host.full), np.uint64)
            call("msbg_grid_set_full_blocks", g.handle, ptr(full), len(full))
        return g

    def to_host(self) -> HostGrid:
        d = self.dims()
        h = HostGrid(self.name, self.sx, self.sy, self.sz, 0.0, 0.0, self.bsx, self.dtype)
        ids = self.value_block_ids()
        if len(ids):
            data = self.read_blocks(ids)
            for k, bid in enumerate(ids):
                h.blocks[int(bid)] = data[k].copy()
        del d
        return h

    def dims(self):
        out = (C.c_uint64 * 8)()
        call("msbg_grid_dims", self.handle, out)
        return [int(v) for v in out]

    def n_value_blocks(self) -> int:
        return self.dims()[7]

    def ensure_blocks(self, bids) -> None:
        b = np.ascontiguousarray(bids, np.uint64)
        call("msbg_grid_ensure_blocks", self.handle, ptr(b), len(b))

    def set_full_blocks(self, bids) -> None:
        b = np.ascontiguousarray(bids, np.uint64)
        call("msbg_grid_set_full_blocks", self.handle, ptr(b), len(b))

    def set_empty_blocks(self, bids) -> None:
        b = np.ascontiguousarray(bids, np.uint64)
        call("msbg_grid_set_empty_blocks", self.handle, ptr(b), len(b))

    def write_blocks(self, bids, payload: np.ndarray) -> None:
        b = np.ascontiguousarray(bids, np.uint64)
        p = np.ascontiguousarray(payload, self.np_dtype).reshape(len(b), self.N)
        call("msbg_grid_write_blocks", self.handle, ptr(b), len(b), ptr(p))

    def read_blocks(self, bids) -> np.ndarray:
        b = np.ascontiguousarray(bids, np.uint64)
        out = np.empty((len(b), self.N), self.np_dtype)
        call("msbg_grid_read_blocks", self.handle, ptr(b), len(b), ptr(out))
        return out

    def fill_blocks(self, bids, value: float) -> None:
        b = np.ascontiguousarray(bids, np.uint64)
        call("msbg_grid_fill_blocks", self.handle, ptr(b), len(b), float(value))

    def value_block_ids(self) -> np.ndarray:
        n = C.c_size_t()
        call("msbg_grid_value_block_ids", self.handle, None, 0, C.byref(n))
        out = np.empty(n.value, np.uint64)
        call("msbg_grid_value_block_ids", self.handle, ptr(out), n.value, C.byref(n))
        return out

    def payload_device_ptr(self):
        p = C.c_void_p()
        n = C.c_uint64()
        call("msbg_grid_payload", self.handle, C.byref(p), C.byref(n))
        return p.value or 0, n.value

    def slots(self, bids) -> np.ndarray:
        b = np.ascontiguousarray(bids, np.uint64)
        out = np.empty(len(b), np.int32)
        call("msbg_grid_slots", self.handle, ptr(b), len(b), ptr(out))
        return out

    def halo_gather(self, bids, halo: int, full: bool, bc: int) -> np.ndarray:
        """HaloBlock::fill (multires/halo.rs:31-170) for each bid: [n][HSX^3] f32."""
        b = np.ascontiguousarray(bids, np.uint64)
        hsx = self.bsx + 2 * halo
        out = np.empty((len(b), hsx ** 3), np.float32)
        call("msbg_halo_gather", self.handle, ptr(b), len(b), int(halo), int(bool(full)), int(bc), ptr(out))
        return out

    def sample_linear(self, pos: np.ndarray, align: int, bc: int) -> np.ndarray:
        """Sampler::sample::<Linear> (math/sample.rs:494-512)."""
        p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        out = np.empty(len(p), np.float32)
        call("msbg_sample_linear", self.handle, ptr(p), len(p), int(align), int(bc), ptr(out))
        return out

    def ensure_blocks_device(self, d_bids, d_slots_out=None) -> None:
        """ensure_blocks_parallel (sparse_grid.rs:326-355) from a device (torch)
        array of block ids; optionally writes every id's slot."""
        call("msbg_grid_ensure_blocks_device", self.handle, ptr(d_bids), int(d_bids.numel()), ptr(d_slots_out))

    def sample_ext(self, pos: np.ndarray, mode: int, align: int, bc: int) -> np.ndarray:
        """Cubic value (mode 0), cubic gradient (1), Hessian (2) or trilinear
        gradient (3) (math/sample.rs:493-649)."""
        p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        w = {0: 1, 1: 3, 2: 6, 3: 3}[int(mode)]
        out = np.empty((len(p), w), np.float32)
        call("msbg_sample_ext", self.handle, ptr(p), len(p), int(mode), int(align), int(bc), ptr(out))
        return out[:, 0] if w == 1 else out

    def close(self) -> None:
        if self.handle and self._owned:
            call("msbg_grid_destroy", self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
