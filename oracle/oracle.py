"""ctypes binding of the CPU oracle (oracle/msbg_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA library and the
timed CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg use it.  Each wrapper names the reference function it restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libmsbg_oracle.so")


class OracleGrid(C.Structure):
    _fields_ = [
        ("sx", C.c_int64), ("sy", C.c_int64), ("sz", C.c_int64),
        ("bsx", C.c_int32), ("_pad", C.c_int32),
        ("nx", C.c_int64), ("ny", C.c_int64), ("nz", C.c_int64), ("nxy", C.c_int64),
        ("table", C.c_void_p), ("data", C.c_void_p),
        ("empty_value", C.c_float), ("full_value", C.c_float),
    ]


_lib = None


def build() -> None:
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.or_morton3.restype = C.c_uint64
        _lib.or_morton3.argtypes = [C.c_uint64] * 3
        _lib.or_bucket_indices.restype = C.c_int64
        _lib.or_active_blocks.restype = C.c_int64
        _lib.or_active_blocks.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_float, C.c_void_p]
        _lib.or_kernel.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_int, C.c_void_p]
        _lib.or_sweep.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int]
        _lib.or_sweep_multires.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int,
                                           C.c_float, C.c_int, C.c_int, C.c_int]
        _lib.or_halo_fill.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_void_p]
        _lib.or_fill_multires.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_void_p]
        _lib.or_p2g.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int,
                                C.c_float, C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_int]
        _lib.or_p2g_terms_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                                          C.c_int, C.c_float, C.c_void_p, C.c_int64, C.c_void_p, C.c_int]
        _lib.or_p2g_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int,
                                    C.c_float, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        _lib.or_mac_sample.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_void_p]
        _lib.or_sample_linear.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p]
        _lib.or_sample_ext.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_void_p]
        _lib.or_regularize_refinement_map.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int]
        _lib.or_block_topology.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p]
        _lib.or_block_topology.restype = C.c_uint64
        _lib.or_place.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_float, C.c_int64, C.c_int64, C.c_int64, C.c_int,
                                  C.c_float, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
        _lib.or_place.restype = C.c_int64
        _lib.or_surface_active.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_float,
                                           C.c_void_p]
        _lib.or_surface_active.restype = C.c_int64
        _lib.or_density_splat.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_float,
                                          C.c_float, C.c_int, C.c_void_p, C.c_int64, C.c_void_p]
        _lib.or_density_finalize.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_float, C.c_float]
        _lib.or_g2p_blend.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_void_p]
        _lib.or_divergence.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
        _lib.or_downsample_avg.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p]
        _lib.or_sort_block_list_morton.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_int]
        _lib.or_morton_sort.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        _lib.or_bucket_indices.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.or_poisson_matvec.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_double,
                                           C.c_void_p, C.c_void_p]
        _lib.or_poisson_jacobi.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_double,
                                           C.c_double, C.c_int, C.c_void_p, C.c_void_p]
        _lib.or_poisson_solve.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int,
                                          C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.or_poisson_solve.restype = C.c_int
        _lib.or_poisson_levels.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_void_p]
        _lib.or_poisson_levels.restype = C.c_int
        _lib.or_num_threads.restype = C.c_int
        _lib.or_sweep_stochastic.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_float, C.c_int,
                                             C.c_int, C.c_uint32, C.c_int, C.c_uint64]
        _lib.or_sweep_stochastic.restype = C.c_uint64
        _lib.or_f32_to_f16.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        _lib.or_f16_to_f32.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        _lib.or_density8_store_sr.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
        _lib.or_lane_rng.argtypes = [C.c_uint32, C.c_int, C.c_int64, C.c_void_p]
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else C.c_void_p(0)


class GridView:
    """Dense-table view of a HostGrid (f32 data) that the oracle reads/writes."""

    def __init__(self, host, data_override=None):
        self.host = host
        self.table, data, self.ids = host.table_and_data()
        if data_override is not None:
            data = data_override
        self.data = np.ascontiguousarray(data)
        self.s = OracleGrid(host.sx, host.sy, host.sz, host.bsx, 0, host.nx, host.ny, host.nz, host.nxy,
                            self.table.ctypes.data, self.data.ctypes.data, host.empty_value, host.full_value)

    def ref(self):
        return C.byref(self.s)

    def write_back(self):
        for s, bid in enumerate(self.ids):
            self.host.blocks[bid][:] = self.data[s]


def halo_fill(host, bid: int, halo: int, full: bool, bc: int) -> np.ndarray:
    """HaloBlock::fill (multires/halo.rs:31-170)."""
    v = GridView(host)
    hsx = host.bsx + 2 * halo
    out = np.zeros(hsx ** 3, np.float32)
    lib().or_halo_fill(v.ref(), int(bid), int(halo), int(bool(full)), int(bc), _p(out))
    return out


def fill_multires(fine, coarse, levels, bid, halo, full, bc) -> np.ndarray:
    """fill_multires (multires/halo.rs:187-358)."""
    vf, vc = GridView(fine), GridView(coarse)
    lv = np.ascontiguousarray(levels, np.uint8)
    hsx = fine.bsx + 2 * halo
    out = np.zeros(hsx ** 3, np.float32)
    lib().or_fill_multires(vf.ref(), vc.ref(), _p(lv), int(bid), int(halo), int(bool(full)), int(bc), _p(out))
    return out


def kernel(stencil: int, halo: np.ndarray, bsx: int, dt: float, clamp01: bool) -> np.ndarray:
    """kernel_laplacian / kernel_meancurv / kernel_bilaplacian on a staged halo."""
    h = np.ascontiguousarray(halo, np.float32)
    out = np.empty(bsx ** 3, np.float32)
    lib().or_kernel(int(stencil), _p(h), int(bsx), float(dt), int(bool(clamp01)), _p(out))
    return out


_ELEM = {"f32": 0, "u16": 1, "bf16": 2, "u8": 3, "f16": 4}


def sweep(host, active, stencil: int, dt: float, iterations: int, clamp01: bool, threads: int = 1) -> None:
    """Serial colour-ordered sweep (solver.rs:187-217, 290-331); in place on host."""
    v = GridView(host)
    a = np.ascontiguousarray(active, np.int64)
    lib().or_sweep(v.ref(), _p(v.data), _ELEM[host.dtype], _p(a), len(a), int(stencil), float(dt), int(iterations),
                   int(bool(clamp01)), int(threads))
    v.write_back()


def sweep_stochastic(host, active, stencil: int, dt: float, iterations: int, clamp01: bool, seed: int = 0xDEADBEEF,
                     lanes: int = 16, stream_pos: int = 0) -> int:
    """Sweeper::sweep on Density8 storage (solver.rs:166-217) with the one
    sweeping thread's generator SimdRng::<lanes>::seed(seed) after
    `stream_pos` draws (stencil.rs:103-132, 176-192); in place on host.
    Returns the draws taken after the call."""
    assert host.dtype == "u8"
    v = GridView(host)
    a = np.ascontiguousarray(active, np.int64)
    pos = lib().or_sweep_stochastic(v.ref(), _p(v.data), _p(a), len(a), int(stencil), float(dt), int(iterations),
                                    int(bool(clamp01)), int(seed) & 0xFFFFFFFF, int(lanes), int(stream_pos))
    v.write_back()
    return int(pos)


def f32_to_f16(x) -> np.ndarray:
    """IEEE binary16 bits of f32 values, round to nearest even."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty(x.shape, np.uint16)
    lib().or_f32_to_f16(_p(x), x.size, _p(out))
    return out


def f16_to_f32(bits) -> np.ndarray:
    b = np.ascontiguousarray(bits, np.uint16)
    out = np.empty(b.shape, np.float32)
    lib().or_f16_to_f32(_p(b), b.size, _p(out))
    return out


def density8_store_sr(v, u) -> np.ndarray:
    """Density8 StoreBack of values v against draws u (stencil.rs:176-192)."""
    v = np.ascontiguousarray(v, np.float32)
    u = np.ascontiguousarray(u, np.float32)
    out = np.empty(v.shape, np.uint8)
    lib().or_density8_store_sr(_p(v), _p(u), v.size, _p(out))
    return out


def lane_rng(seed: int, lanes: int, draws: int) -> np.ndarray:
    """The first `draws` outputs of SimdRng::<lanes>::seed(seed), [draws][lanes]."""
    out = np.empty((draws, lanes), np.float32)
    lib().or_lane_rng(int(seed) & 0xFFFFFFFF, int(lanes), int(draws), _p(out))
    return out


def sweep_multires(fine, coarse, levels, active, stencil, dt, iterations, clamp01, threads=1) -> None:
    vf, vc = GridView(fine), GridView(coarse)
    lv = np.ascontiguousarray(levels, np.uint8)
    a = np.ascontiguousarray(active, np.int64)
    lib().or_sweep_multires(vf.ref(), _p(vf.data), vc.ref(), _p(lv), _p(a), len(a), int(stencil), float(dt),
                            int(iterations), int(bool(clamp01)), int(threads))
    vf.write_back()


def morton3(x, y, z) -> int:
    return int(lib().or_morton3(int(x), int(y), int(z)))


def sort_block_list_morton(blocks, nx, ny, levels, n_levels) -> np.ndarray:
    b = np.array(blocks, np.int64)
    lv = np.ascontiguousarray(levels, np.uint8)
    lib().or_sort_block_list_morton(_p(b), len(b), int(nx), int(ny), _p(lv), int(n_levels))
    return b


def bucket_indices(bids):
    """Stable dense counting sort (particles/sort.rs:455-490)."""
    b = np.ascontiguousarray(bids, np.uint64)
    n = len(b)
    pb = np.empty(max(n, 1), np.uint64)
    st = np.empty(n + 1, np.uint64)
    perm = np.empty(max(n, 1), np.uint32)
    nb = lib().or_bucket_indices(_p(b), n, _p(pb), _p(st), _p(perm))
    if n == 0:
        return np.empty(0, np.uint64), np.zeros(1, np.uint64), np.empty(0, np.uint32)
    return pb[:nb].copy(), st[: nb + 1].copy(), perm[:n].copy()


def morton_sort(pos):
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    keys = np.empty(len(p), np.uint64)
    perm = np.empty(len(p), np.uint32)
    lib().or_morton_sort(_p(p), len(p), _p(keys), _p(perm))
    return keys, perm


def active_blocks(pos, sx, sy, sz, bsx, r_p) -> np.ndarray:
    """fluid/p2g.rs:104-136 (reach r_p + 1)."""
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    n = lib().or_active_blocks(_p(p), len(p), sx, sy, sz, bsx, float(r_p), None)
    out = np.empty(n, np.int64)
    lib().or_active_blocks(_p(p), len(p), sx, sy, sz, bsx, float(r_p), _p(out))
    return out


def p2g(pos, vel, mass, sx, sy, sz, bsx, r_p, active=None, normalize=True, threads=1):
    """particles_to_grid with the staged splat in the reference's order.
    Returns (active, channels[6][n_active][N]) with channels = mass x,y,z then
    velocity x,y,z (momentum when normalize is False)."""
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    v = np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
    m = np.ascontiguousarray(mass, np.float32).reshape(-1)
    if active is None:
        active = active_blocks(p, sx, sy, sz, bsx, r_p)
    a = np.ascontiguousarray(active, np.int64)
    out = np.zeros((6, len(a), bsx ** 3), np.float32)
    lib().or_p2g(_p(p), _p(v), _p(m), len(p), sx, sy, sz, bsx, float(r_p), _p(a), len(a), int(bool(normalize)), _p(out),
                 int(threads))
    return a, out


def p2g_terms_f64(pos, vel, mass, sx, sy, sz, bsx, r_p, active, threads=1):
    """The reference's f32 per-particle terms summed in FP64 (mass, momentum)."""
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    v = np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
    m = np.ascontiguousarray(mass, np.float32).reshape(-1)
    a = np.ascontiguousarray(active, np.int64)
    out = np.zeros((6, len(a), bsx ** 3), np.float64)
    lib().or_p2g_terms_f64(_p(p), _p(v), _p(m), len(p), sx, sy, sz, bsx, float(r_p), _p(a), len(a), _p(out),
                           int(threads))
    return out


def p2g_f64(pos, vel, mass, sx, sy, sz, bsx, r_p, active):
    """Exact Eq. 6 splat in FP64 (unnormalised) + per-face sums of |terms|."""
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    v = np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
    m = np.ascontiguousarray(mass, np.float32).reshape(-1)
    a = np.ascontiguousarray(active, np.int64)
    out = np.zeros((6, len(a), bsx ** 3), np.float64)
    ab = np.zeros((6, len(a), bsx ** 3), np.float64)
    lib().or_p2g_f64(_p(p), _p(v), _p(m), len(p), sx, sy, sz, bsx, float(r_p), _p(a), len(a), _p(out), _p(ab))
    return out, ab


def sample_linear(host, pos, align, bc) -> np.ndarray:
    v = GridView(host)
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    out = np.empty(len(p), np.float32)
    lib().or_sample_linear(v.ref(), _p(p), len(p), int(align), int(bc), _p(out))
    return out


SAMPLE_WIDTH = {0: 1, 1: 3, 2: 6, 3: 3}


def sample_ext(host, pos, mode, bc, align=0) -> np.ndarray:
    """Sample for SparseGrid (math/sample.rs:493-649): mode 0 cubic value,
    1 cubic gradient [n][3], 2 cubic Hessian [n][6] (fxx, fyy, fzz, fxy, fxz,
    fyz), 3 trilinear gradient [n][3] at `align` (0 Corner, 1 CellCentered)."""
    v = GridView(host)
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    out = np.empty((len(p), SAMPLE_WIDTH[mode]), np.float32)
    lib().or_sample_ext(v.ref(), _p(p), len(p), int(mode), int(align), int(bc), _p(out))
    return out[:, 0] if mode == 0 else out


def regularize_refinement_map(levels, nx, ny, nz, n_levels) -> np.ndarray:
    """multires/refinement.rs:63-107 (a copy is regularised)."""
    m = np.ascontiguousarray(levels, np.uint8).copy()
    lib().or_regularize_refinement_map(_p(m), nx, ny, nz, int(n_levels))
    return m


def block_topology(levels, nx, ny, nz, n_levels, user_flags=None):
    """multires/refinement.rs:124-208: (flags [n] u16, fine-coarse lists per
    level, EXISTS count)."""
    m = np.ascontiguousarray(levels, np.uint8)
    n = len(m)
    u = None if user_flags is None else np.ascontiguousarray(user_flags, np.uint16)
    flags = np.zeros(n, np.uint16)
    fc = np.zeros((n_levels, n), np.int64)
    cnt = np.zeros(n_levels, np.int64)
    n_act = lib().or_block_topology(_p(m), nx, ny, nz, int(n_levels), None if u is None else _p(u), _p(flags), _p(fc),
                                    _p(cnt))
    return flags, [fc[l, : cnt[l]].copy() for l in range(n_levels)], int(n_act)


def domain_bounds(sx, sy, sz):
    """DomainBounds::new (particles/mod.rs): align24(0.005), align24(size - 0.005)."""
    scale = 16_777_215.0 / 32_768.0

    def align24(x):
        return np.float32(np.floor(scale * x + 0.5) / scale)

    return (np.array([align24(0.005)] * 3, np.float32),
            np.array([align24(float(v) - 0.005) for v in (sx, sy, sz)], np.float32))


def place(base, bbox_min, span_max, sx, sy, sz, bsx, factor, n_instances):
    """particles/sort.rs:31-144 place: (positions [n][3] f32, centre bids)."""
    b = np.ascontiguousarray(base, np.float32).reshape(-1, 3)
    bb = np.ascontiguousarray(bbox_min, np.float32)
    lo, hi = domain_bounds(sx, sy, sz)
    n = lib().or_place(_p(b), len(b), _p(bb), float(span_max), sx, sy, sz, bsx, float(factor), int(n_instances),
                       _p(lo), _p(hi), None, None, 0)
    pos = np.zeros((n, 3), np.float32)
    bids = np.zeros(n, np.int64)
    lib().or_place(_p(b), len(b), _p(bb), float(span_max), sx, sy, sz, bsx, float(factor), int(n_instances), _p(lo),
                   _p(hi), _p(pos), _p(bids), n)
    return pos, bids


def surface_active(pos, sx, sy, sz, bsx, r_scan) -> np.ndarray:
    """Footprint block union of the surface splat (reach r_scan)."""
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    c = lib().or_surface_active(_p(p), len(p), sx, sy, sz, bsx, float(r_scan), None)
    out = np.zeros(c, np.int64)
    lib().or_surface_active(_p(p), len(p), sx, sy, sz, bsx, float(r_scan), _p(out))
    return out


_QMAX = {"f32": (0, np.float32), "u16": (65535, np.uint16), "u8": (255, np.uint8)}


def _quant(density):
    """Storage of a surface grid: True/"u16" Density, "u8" Density8, False/"f32"."""
    if density is True:
        density = "u16"
    elif density is False:
        density = "f32"
    return _QMAX[density]


def density_splat(pos, sx, sy, sz, bsx, r_particle, nb_dist, density, active) -> np.ndarray:
    """particles/splat.rs:92-319 min-splat into the active blocks (filled with
    the full value first): [n_active][bsx^3] in the grid's storage type
    (`density`: True or "u16" Density, "u8" Density8, False or "f32")."""
    qmax, dt = _quant(density)
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    a = np.ascontiguousarray(active, np.int64)
    out = np.zeros((len(a), bsx ** 3), np.float32)
    lib().or_density_splat(_p(p), len(p), sx, sy, sz, bsx, float(r_particle), float(nb_dist), qmax, _p(a),
                           len(a), _p(out))
    return out.astype(dt)


def density_finalize(vals, density, r_particle, nb_dist) -> np.ndarray:
    """particles/finalize.rs:35-71 on splatted values (storage as in density_splat)."""
    qmax, dt = _quant(density)
    v = np.ascontiguousarray(vals, np.float32).copy()
    lib().or_density_finalize(_p(v), v.size, qmax, float(r_particle), float(nb_dist))
    return v.astype(dt)


def mac_sample(vx, vy, vz, pos, bc) -> np.ndarray:
    """MacSampler::sample::<Linear> (fluid/g2p.rs:26-32) over three HostGrids."""
    views = [GridView(g) for g in (vx, vy, vz)]
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    out = np.empty((len(p), 3), np.float32)
    lib().or_mac_sample(views[0].ref(), views[1].ref(), views[2].ref(), _p(p), len(p), int(bc), _p(out))
    return out


def g2p_blend(u_old, u, u_tilde, alpha) -> np.ndarray:
    a, b, c = (np.ascontiguousarray(x, np.float32) for x in (u_old, u, u_tilde))
    out = np.empty_like(a)
    lib().or_g2p_blend(_p(a), _p(b), _p(c), a.size // 3, float(alpha), _p(out))
    return out


def divergence(ux, uy, uz, active) -> np.ndarray:
    """MacGrid::divergence (mac.rs:137-171) over three HostGrids."""
    views = [GridView(g) for g in (ux, uy, uz)]
    a = np.ascontiguousarray(active, np.int64)
    out = np.zeros((len(a), ux.N), np.float32)
    lib().or_divergence(views[0].ref(), views[1].ref(), views[2].ref(), _p(a), len(a), _p(out))
    return out


def downsample_avg(fine_blocks: np.ndarray, bsx: int) -> np.ndarray:
    """downsample_channel_avg (multires/downsample.rs:13-59) of [n][bsx^3] blocks."""
    f = np.ascontiguousarray(fine_blocks, np.float32)
    n = f.shape[0]
    out = np.empty((n, (bsx // 2) ** 3), np.float32)
    lib().or_downsample_avg(_p(f), n, int(bsx), _p(out))
    return out


def num_threads() -> int:
    return int(lib().or_num_threads())


# ---- FP64 Poisson oracle (no reference implementation) -----------------------
def poisson_matvec(active, nx, ny, nz, bs, x, scale=1.0):
    a = np.ascontiguousarray(active, np.int64)
    xx = np.ascontiguousarray(x, np.float64)
    y = np.empty_like(xx)
    lib().or_poisson_matvec(_p(a), len(a), nx, ny, nz, bs, float(scale), _p(xx), _p(y))
    return y


def poisson_jacobi(active, nx, ny, nz, bs, x, b, omega, sweeps, scale=1.0):
    a = np.ascontiguousarray(active, np.int64)
    xx = np.array(x, np.float64)
    bb = np.ascontiguousarray(b, np.float64)
    lib().or_poisson_jacobi(_p(a), len(a), nx, ny, nz, bs, float(scale), float(omega), int(sweeps), _p(xx), _p(bb))
    return xx


def poisson_levels(active, nx, ny, nz, bs, max_levels=32):
    a = np.ascontiguousarray(np.unique(np.asarray(active, np.int64)))
    cells = np.zeros(64, np.int64)
    n = lib().or_poisson_levels(_p(a), len(a), nx, ny, nz, bs, max_levels, _p(cells))
    return cells[:n]


def poisson_solve(active, nx, ny, nz, bs, b, mode=0, tol=1e-6, max_iter=200, nu1=2, nu2=2, omega=2.0 / 3.0,
                  max_levels=32):
    """FP64 V-cycle (mode 0) or MG-preconditioned CG (mode 1); unknowns in
    ascending block-id order."""
    a = np.ascontiguousarray(np.unique(np.asarray(active, np.int64)))
    bb = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(bb)
    hist = np.zeros(max_iter + 1, np.float64)
    it = lib().or_poisson_solve(_p(a), len(a), nx, ny, nz, bs, max_levels, nu1, nu2, float(omega), int(mode),
                                float(tol), int(max_iter), _p(x), _p(bb), _p(hist))
    return x, hist[:it]
