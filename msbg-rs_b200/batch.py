"""Batched Poisson solves (the C ABI's msbg_batch_*): many independent sparse
problems solved together in one CUDA graph launch whose device-side loop runs
solver cycles until every problem converges, launch shapes autotuned per
level.  No counterpart in the crate, which has no
pressure solver."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call, ptr
from .grid import Context


class Batch:
    def __init__(self, ctx: Context, problems, tune: bool = True):
        """problems: sequence of (dims (sx, sy, sz), bsx, active block ids)."""
        self.ctx = ctx
        n = len(problems)
        self.bsx = np.array([int(p[1]) for p in problems], np.int32)
        self.dims = np.array([[int(d) for d in p[0]] for p in problems], np.uint64).reshape(-1)
        self._active = [np.unique(np.asarray(p[2], np.uint64)) for p in problems]
        ptrs = (C.c_void_p * n)(*[a.ctypes.data for a in self._active])
        counts = np.array([len(a) for a in self._active], np.uint64)
        h = C.c_void_p()
        call("msbg_batch_create", ctx.handle, n, ptr(self.bsx), ptr(self.dims), ptrs, ptr(counts), int(bool(tune)),
             C.byref(h))
        self.handle = h
        self.n = n
        ng = C.c_int()
        call("msbg_batch_groups", h, C.byref(ng))
        self.n_groups = ng.value

    def layout(self, p):
        """(group, first cell, cells) of problem p in its group's vectors."""
        g, off, cnt = C.c_int(), C.c_uint64(), C.c_uint64()
        call("msbg_batch_problem", self.handle, int(p), C.byref(g), C.byref(off), C.byref(cnt))
        return g.value, off.value, cnt.value

    def buffers(self, g):
        """(device f32 rhs pointer, device FP64 solution pointer, cells, bsx) of group g."""
        b, x, n, bs = C.c_void_p(), C.c_void_p(), C.c_uint64(), C.c_int()
        call("msbg_batch_buffers", self.handle, int(g), C.byref(b), C.byref(x), C.byref(n), C.byref(bs))
        return b.value, x.value, n.value, bs.value

    def set_rhs(self, p, b: np.ndarray) -> None:
        bb = np.ascontiguousarray(b, np.float32).reshape(-1)
        assert bb.size == self.layout(p)[2]
        call("msbg_batch_set_rhs", self.handle, int(p), ptr(bb))

    def solution(self, p) -> np.ndarray:
        out = np.empty(self.layout(p)[2], np.float64)
        call("msbg_batch_get_solution", self.handle, int(p), ptr(out))
        return out

    def tuning(self, g):
        """Per level of group g: the chosen (Jacobi shape index, residual shape
        index, tile z-planes or 0) and the level's cells."""
        cfg = np.zeros(3 * 64, np.int32)
        cells = np.zeros(64, np.uint64)
        n = C.c_size_t()
        call("msbg_batch_tuning", self.handle, int(g), ptr(cfg), ptr(cells), 64, C.byref(n))
        return cfg[: 3 * n.value].reshape(-1, 3), cells[: n.value]

    def solve(self, tol=1e-8, iters_per_cycle=8, max_cycles=100, zero_x=True):
        """(iterations per problem, relative residual per problem, cycles)."""
        its = np.zeros(self.n, np.int32)
        rel = np.zeros(self.n, np.float64)
        cyc = C.c_int()
        call("msbg_batch_solve", self.handle, float(tol), int(iters_per_cycle), int(max_cycles), int(bool(zero_x)),
             ptr(its), ptr(rel), C.byref(cyc))
        return its, rel, cyc.value

    def close(self):
        if self.handle:
            call("msbg_batch_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
