"""MAC-grid fluid transfer on the device: MacGrid (fluid/mac.rs),
particles_to_grid (fluid/p2g.rs:141-164), MacSampler (fluid/g2p.rs:11-33)
and g2p_blend (fluid/g2p.rs:42-45)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call, ptr
from .grid import Context, SparseGrid

X, Y, Z = 0, 1, 2


class MacGrid:
    """MacGrid::new (mac.rs:35-45): three face-velocity and three face-mass channels."""

    def __init__(self, ctx: Context, sx, sy, sz, bsx=16):
        self.ctx = ctx
        self.sx, self.sy, self.sz, self.bsx = int(sx), int(sy), int(sz), int(bsx)
        h = C.c_void_p()
        call("msbg_mac_create", ctx.handle, self.sx, self.sy, self.sz, self.bsx, C.byref(h))
        self.handle = h
        self._ch = []
        for c in range(6):
            g = C.c_void_p()
            call("msbg_mac_channel", h, c, C.byref(g))
            self._ch.append(SparseGrid.borrowed(ctx, g, self.sx, self.sy, self.sz, self.bsx, "f32", f"ch{c}"))

    def velocity(self, a: int) -> SparseGrid:
        return self._ch[a]

    def mass(self, a: int) -> SparseGrid:
        return self._ch[3 + a]

    def zero_blocks(self, active) -> None:
        """MacGrid::zero_blocks (mac.rs:95-102)."""
        b = np.ascontiguousarray(active, np.uint64)
        call("msbg_mac_zero_blocks", self.handle, ptr(b), len(b))

    def normalize_velocity(self, active) -> None:
        """MacGrid::normalize_velocity (mac.rs:106-132)."""
        b = np.ascontiguousarray(active, np.uint64)
        call("msbg_mac_normalize_velocity", self.handle, ptr(b), len(b))

    def divergence(self, dst: SparseGrid, active) -> None:
        """MacGrid::divergence (mac.rs:137-171)."""
        b = np.ascontiguousarray(active, np.uint64)
        call("msbg_mac_divergence", self.handle, dst.handle, ptr(b), len(b))

    def active_blocks(self) -> np.ndarray:
        n = C.c_size_t()
        call("msbg_mac_active_blocks", self.handle, None, 0, C.byref(n))
        out = np.empty(n.value, np.uint64)
        call("msbg_mac_active_blocks", self.handle, ptr(out), n.value, C.byref(n))
        return out

    def close(self) -> None:
        if self.handle:
            call("msbg_mac_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def particles_to_grid(mac: MacGrid, positions, velocities, mass, r_p: float) -> int:
    """particles_to_grid (fluid/p2g.rs:141-164) from host arrays; returns the
    number of active blocks.  positions/velocities are [n][3], mass [n]."""
    p = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    v = np.ascontiguousarray(velocities, np.float32).reshape(-1, 3)
    m = np.ascontiguousarray(mass, np.float32).reshape(-1)
    assert len(p) == len(v) == len(m)
    na = C.c_size_t()
    call("msbg_p2g", mac.handle, ptr(p), ptr(v), ptr(m), len(p), float(r_p), C.byref(na))
    return na.value


def particles_to_grid_device(mac: MacGrid, d_pos, d_vel, d_mass, n: int, r_p: float) -> int:
    """Same as particles_to_grid with device arrays (torch tensors or raw pointers)."""
    na = C.c_size_t()
    call("msbg_p2g_device", mac.handle, ptr(d_pos), ptr(d_vel), ptr(d_mass), int(n), float(r_p), C.byref(na))
    return na.value


def particles_to_grid_sorted_device(mac: MacGrid, d_pos, d_vel, d_mass, d_keys, n: int, r_p: float) -> int:
    """particles_to_grid for Morton-sorted device arrays with their sorted keys."""
    na = C.c_size_t()
    call("msbg_p2g_sorted_device", mac.handle, ptr(d_pos), ptr(d_vel), ptr(d_mass), ptr(d_keys), int(n), float(r_p),
         C.byref(na))
    return na.value


def particles_to_grid_permuted_device(mac: MacGrid, d_pos, d_vel, d_mass, d_keys, d_perm, n: int, r_p: float) -> int:
    """particles_to_grid for device arrays in the caller's order, with the sorted
    keys and the permutation of a Morton sort of their positions."""
    na = C.c_size_t()
    call("msbg_p2g_permuted_device", mac.handle, ptr(d_pos), ptr(d_vel), ptr(d_mass), ptr(d_keys), ptr(d_perm), int(n),
         float(r_p), C.byref(na))
    return na.value


class MacSampler:
    """MacSampler::new(mac, bc) + sample::<Linear> (fluid/g2p.rs:15-32)."""

    def __init__(self, mac: MacGrid, bc: int):
        self.mac = mac
        self.bc = int(bc)

    def sample(self, positions) -> np.ndarray:
        p = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        out = np.empty_like(p)
        call("msbg_g2p", self.mac.handle, ptr(p), len(p), self.bc, ptr(out))
        return out

    def sample_device(self, d_pos, n: int, d_out) -> None:
        call("msbg_g2p_device", self.mac.handle, ptr(d_pos), int(n), self.bc, ptr(d_out))


def g2p_flip_device(sampler: "MacSampler", d_pos, n: int, d_u_old, alpha: float, d_out, d_u_tilde=None) -> None:
    """MacSampler::sample then g2p_blend (fluid/g2p.rs:26-45) in one pass on
    device [n][3] arrays; d_u_tilde None: the sample is its own u_tilde."""
    call("msbg_g2p_flip_device", sampler.mac.handle, ptr(d_pos), int(n), sampler.bc, ptr(d_u_old), ptr(d_u_tilde),
         float(alpha), ptr(d_out))


def g2p_blend_device(ctx: Context, d_u_old, d_u, d_u_tilde, n: int, alpha: float, d_out) -> None:
    """g2p_blend (fluid/g2p.rs:42-45) on device [n][3] arrays."""
    call("msbg_g2p_blend_device", ctx.handle, ptr(d_u_old), ptr(d_u), ptr(d_u_tilde), int(n), float(alpha), ptr(d_out))


def g2p_blend(u_old: np.ndarray, u: np.ndarray, u_tilde: np.ndarray, alpha: float) -> np.ndarray:
    """g2p_blend (fluid/g2p.rs:42-45) on host arrays (f32, component-wise)."""
    a = np.float32(alpha)
    delta = (u.astype(np.float32) - u_tilde.astype(np.float32)).astype(np.float32)
    return ((u_old.astype(np.float32) + delta) * a + u.astype(np.float32) * (np.float32(1.0) - a)).astype(np.float32)


class FlipStep:
    """One FLIP transfer step through host arrays (msbg_flip_step): Morton
    sort, particles_to_grid (fluid/p2g.rs:141-164), `sweeps` multires sweeps
    of the x-face mass over the level-0 blocks (solver.rs:166-185),
    MacSampler::sample + g2p_blend (fluid/g2p.rs:15-45), with the copies in
    the call.  `levels` holds one level per block of the MAC grid; `coarse`
    has half its block size."""

    def __init__(self, mac: MacGrid, coarse: SparseGrid, levels):
        self.mac, self.coarse = mac, coarse
        self.levels = np.ascontiguousarray(levels, np.uint8)
        h = C.c_void_p()
        call("msbg_flip_create", mac.handle, coarse.handle, ptr(self.levels), len(self.levels), C.byref(h))
        self.handle = h

    def step_ptrs(self, pos_ptr: int, vel_ptr: int, mass_ptr: int, n: int, r_p: float, stencil: int, dt: float,
                  sweeps: int, alpha: float, out_ptr: int) -> None:
        """Host addresses (e.g. of page-locked buffers); out gets [n][3]."""
        call("msbg_flip_step", self.handle, C.c_void_p(pos_ptr), C.c_void_p(vel_ptr), C.c_void_p(mass_ptr), int(n),
             float(r_p), int(stencil), float(dt), int(sweeps), float(alpha), C.c_void_p(out_ptr))

    def step(self, positions, velocities, mass, r_p: float, stencil: int, dt: float, sweeps: int,
             alpha: float) -> np.ndarray:
        p = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        v = np.ascontiguousarray(velocities, np.float32).reshape(-1, 3)
        m = np.ascontiguousarray(mass, np.float32).reshape(-1)
        out = np.empty_like(v)
        self.step_ptrs(p.ctypes.data, v.ctypes.data, m.ctypes.data, len(p), r_p, stencil, dt, sweeps, alpha,
                       out.ctypes.data)
        return out

    def close(self) -> None:
        if self.handle:
            call("msbg_flip_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
