"""The learned preconditioner's network (the C ABI's msbg_unet_*): a
block-sparse 3D U-Net over the level-0 blocks of a Poisson solve, trained and
applied on the device.  No counterpart in the crate, which has no pressure
solver."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call, ptr
from .grid import Context


class UNet:
    def __init__(self, ctx: Context, sx, sy, sz, active, seed: int = 1):
        self.ctx = ctx
        a = np.unique(np.asarray(active, np.uint64))
        self.active = a
        h = C.c_void_p()
        call("msbg_unet_create", ctx.handle, int(sx), int(sy), int(sz), ptr(a), len(a), int(seed), C.byref(h))
        self.handle = h
        n = C.c_size_t()
        call("msbg_unet_num_params", h, C.byref(n))
        self.n_params = n.value
        self.n = len(a) * 4096

    def layers(self) -> np.ndarray:
        out = np.zeros(8 * 16, np.int64)
        n = C.c_size_t()
        call("msbg_unet_layers", self.handle, ptr(out), len(out), C.byref(n))
        return out[: 8 * n.value].reshape(n.value, 8)

    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        call("msbg_unet_get_params", self.handle, ptr(out))
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        call("msbg_unet_set_params", self.handle, ptr(p))

    def grads(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        call("msbg_unet_get_grads", self.handle, ptr(out))
        return out

    def set_output_scale(self, s: float) -> None:
        call("msbg_unet_set_output_scale", self.handle, float(s))

    def apply(self, d_r, d_z) -> None:
        call("msbg_unet_apply_device", self.handle, ptr(d_r), ptr(d_z))

    def forward_raw(self, d_r, d_y) -> None:
        call("msbg_unet_forward_raw_device", self.handle, ptr(d_r), ptr(d_y))

    def train_step(self, d_r, d_e, lr: float = 1e-3, update: bool = True) -> float:
        loss = C.c_double()
        call("msbg_unet_train_step_device", self.handle, ptr(d_r), ptr(d_e), float(lr), int(bool(update)),
             C.byref(loss))
        return loss.value

    def close(self):
        if self.handle:
            call("msbg_unet_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
