"""BlockMap (blockmap.rs:35-209) in device memory: block id -> u32 value,
with insert, update (the counting form), get, remove and sorted_pairs over
batches of device (torch) arrays or host (numpy) arrays."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call, ptr
from .grid import Context


class BlockMap:
    def __init__(self, ctx: Context, capacity: int = 4):
        self.ctx = ctx
        h = C.c_void_p()
        call("msbg_blockmap_create", ctx.handle, int(capacity), C.byref(h))
        self.handle = h

    @staticmethod
    def _dev(a, dtype):
        import torch
        if isinstance(a, torch.Tensor):
            return a
        return torch.from_numpy(np.ascontiguousarray(a, dtype)).cuda()

    def __len__(self) -> int:
        n = C.c_uint64()
        call("msbg_blockmap_len", self.handle, C.byref(n), None)
        return n.value

    def capacity(self) -> int:
        c = C.c_uint64()
        call("msbg_blockmap_len", self.handle, None, C.byref(c))
        return c.value

    def insert(self, keys, vals) -> None:
        k, v = self._dev(keys, np.uint64), self._dev(vals, np.uint32)
        call("msbg_blockmap_insert_device", self.handle, ptr(k), ptr(v), len(k))

    def update_add(self, keys) -> None:
        """update(key, 1, |c| c + 1) for every key (a histogram)."""
        k = self._dev(keys, np.uint64)
        call("msbg_blockmap_update_add_device", self.handle, ptr(k), len(k))

    def get(self, keys, missing: int = 0xFFFFFFFF) -> np.ndarray:
        import torch
        k = self._dev(keys, np.uint64)
        out = torch.empty(len(k), dtype=torch.int32, device=k.device)
        call("msbg_blockmap_get_device", self.handle, ptr(k), len(k), C.c_uint32(missing), ptr(out))
        return out.cpu().numpy().view(np.uint32)

    def remove(self, keys) -> None:
        k = self._dev(keys, np.uint64)
        call("msbg_blockmap_remove_device", self.handle, ptr(k), len(k))

    def sorted_pairs(self):
        import torch
        n = C.c_size_t()
        call("msbg_blockmap_sorted_pairs_device", self.handle, None, None, 0, C.byref(n))
        k = torch.empty(max(n.value, 1), dtype=torch.int64, device="cuda")
        v = torch.empty(max(n.value, 1), dtype=torch.int32, device="cuda")
        call("msbg_blockmap_sorted_pairs_device", self.handle, ptr(k), ptr(v), len(k), C.byref(n))
        return k[: n.value].cpu().numpy().view(np.uint64), v[: n.value].cpu().numpy().view(np.uint32)

    def close(self) -> None:
        if self.handle:
            call("msbg_blockmap_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
