"""Poisson pressure solve on the device (the C ABI's msbg_poisson_*).

The crate specifies but does not implement the solve (docs/roadmap.md:608-702):
7-point operator y = D x - sum_nb x with D = 6, weighted-Jacobi relaxation,
zero Dirichlet values outside the active blocks.  Vectors are [n][bsx^3] f32
in ascending block-id order.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call, ptr
from .grid import Context

MG, PCG = 0, 1


class Poisson:
    def __init__(self, ctx: Context, sx, sy, sz, bsx, active):
        self.ctx = ctx
        a = np.unique(np.asarray(active, np.uint64))
        self.active = a
        self.bsx = int(bsx)
        h = C.c_void_p()
        call("msbg_poisson_create", ctx.handle, int(sx), int(sy), int(sz), self.bsx, ptr(a), len(a), C.byref(h))
        self.handle = h
        self.n = len(a) * self.bsx ** 3

    def levels(self) -> np.ndarray:
        out = np.zeros(64, np.uint64)
        n = C.c_size_t()
        call("msbg_poisson_levels", self.handle, ptr(out), 64, C.byref(n))
        return out[: n.value].astype(np.int64)

    def set_smoother(self, nu1=2, nu2=2, omega=2.0 / 3.0):
        call("msbg_poisson_set_smoother", self.handle, int(nu1), int(nu2), float(omega))

    def matvec(self, d_x, d_y):
        call("msbg_poisson_matvec_device", self.handle, ptr(d_x), ptr(d_y))

    def jacobi(self, d_x, d_b, omega=2.0 / 3.0, sweeps=1):
        call("msbg_poisson_jacobi_device", self.handle, ptr(d_x), ptr(d_b), float(omega), int(sweeps))

    def residual(self, d_x, d_b, d_r) -> float:
        nrm = C.c_double()
        call("msbg_poisson_residual_device", self.handle, ptr(d_x), ptr(d_b), ptr(d_r), C.byref(nrm))
        return nrm.value

    def vcycle(self, d_x, d_b):
        call("msbg_poisson_vcycle_device", self.handle, ptr(d_x), ptr(d_b))

    def dot(self, d_a, d_b) -> float:
        out = C.c_double()
        call("msbg_poisson_dot_device", self.handle, ptr(d_a), ptr(d_b), C.byref(out))
        return out.value

    def solve_device(self, d_x, d_b, method=PCG, tol=1e-6, max_iter=100):
        it = C.c_int()
        rel = C.c_double()
        hist = np.zeros(max(max_iter, 1), np.float64)
        call("msbg_poisson_solve_device", self.handle, int(method), ptr(d_x), ptr(d_b), float(tol), int(max_iter),
             C.byref(it), C.byref(rel), ptr(hist))
        return it.value, rel.value, hist[: it.value]

    def solve(self, b: np.ndarray, x0=None, method=PCG, tol=1e-6, max_iter=100):
        """Host arrays in, host solution out."""
        bb = np.ascontiguousarray(b, np.float32).reshape(-1)
        x = np.zeros_like(bb) if x0 is None else np.array(x0, np.float32).reshape(-1)
        it = C.c_int()
        rel = C.c_double()
        hist = np.zeros(max(max_iter, 1), np.float64)
        call("msbg_poisson_solve", self.handle, int(method), ptr(x), ptr(bb), float(tol), int(max_iter), C.byref(it),
             C.byref(rel), ptr(hist))
        return x, it.value, rel.value, hist[: it.value]

    def close(self):
        if self.handle:
            call("msbg_poisson_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
