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

MG, PCG, LEARNED, HYBRID, LEARNED_MG, LEARNED_LEAD = 0, 1, 2, 3, 4, 5


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

    def autotune(self) -> np.ndarray:
        """Times the launch choices of every level but the coarsest and keeps
        the fastest; per level (Jacobi shape, residual shape, tile or 0)."""
        cfg = np.zeros(3 * 64, np.int32)
        n = C.c_size_t()
        call("msbg_poisson_autotune", self.handle, ptr(cfg), cfg.size, C.byref(n))
        return cfg[: 3 * n.value].reshape(-1, 3)

    def set_tuning(self, cfg) -> None:
        """Per level (Jacobi shape, residual shape, tile or 0), as autotune returns it."""
        c = np.ascontiguousarray(cfg, np.int32).reshape(-1, 3)
        call("msbg_poisson_set_tuning", self.handle, ptr(c), len(c))

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
        """Device solve; d_x f32 or float64 (the FP64 solution is kept as is)."""
        it = C.c_int()
        rel = C.c_double()
        hist = np.zeros(max(max_iter, 1), np.float64)
        fn = "msbg_poisson_solve_f64_device" if str(getattr(d_x, "dtype", "")) == "torch.float64" else \
            "msbg_poisson_solve_device"
        call(fn, self.handle, int(method), ptr(d_x), ptr(d_b), float(tol), int(max_iter), C.byref(it), C.byref(rel),
             ptr(hist))
        self.last_history = hist[: it.value]
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

    # ---- learned preconditioner ------------------------------------------------
    def set_preconditioner(self, net) -> None:
        """Network for methods LEARNED (2) and HYBRID (3); None clears it."""
        self._net = net
        call("msbg_poisson_set_preconditioner", self.handle, net.handle if net is not None else None)

    def set_network_lead(self, k: int) -> None:
        """Method LEARNED_LEAD (5): the first |k| preconditioner applications
        are HYBRID's (V-cycle, network, V-cycle; no last V-cycle for k < 0),
        then CG restarts with plain V-cycles."""
        call("msbg_poisson_set_network_lead", self.handle, int(k))

    def solve_stats(self) -> dict:
        """Preconditioner applications of the last solve and its fallback:
        reason 0 none, 1 stall, 2 p.Ap <= 0, 3 r.z <= 0."""
        out = np.zeros(4, np.int32)
        call("msbg_poisson_solve_stats", self.handle, ptr(out))
        return {"vcycles": int(out[0]), "network": int(out[1]), "fallback": int(out[2]), "fallback_iter": int(out[3])}

    def rhs(self, d_b, seed: int, n_blobs: int = 32) -> None:
        call("msbg_poisson_rhs_device", self.handle, int(seed), int(n_blobs), ptr(d_b))

    def train_preconditioner(self, n_rhs=16, mg_iters=20, steps_per_rhs=20, pool=64, lr=1e-3, target=1, seed=1):
        hist = np.zeros(max(1, n_rhs * steps_per_rhs), np.float64)
        steps = C.c_int64()
        call("msbg_poisson_train_preconditioner", self.handle, int(n_rhs), int(mg_iters), int(steps_per_rhs), int(pool),
             float(lr), int(target), int(seed), ptr(hist), len(hist), C.byref(steps))
        return hist[: steps.value]

    def eval_preconditioner(self, n_rhs=2, mg_iters=10, seed=99) -> dict:
        out = np.zeros(3, np.float64)
        call("msbg_poisson_eval_preconditioner", self.handle, int(n_rhs), int(mg_iters), int(seed), ptr(out))
        return {"network": out[0], "vcycle": out[1], "vcycle_plus_network": out[2]}

    def close(self):
        if self.handle:
            call("msbg_poisson_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
