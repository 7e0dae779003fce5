"""Seeded synthetic inputs with the shapes of the benchmark configurations.

There is no public dataset for this path: every input is generated here from a
seed (numpy PCG64, seed = configuration index + 1), following the
configuration rules stated beside each generator.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def shell_active_blocks(n_per_axis: int, bsx: int, radius: float, thickness: float) -> np.ndarray:
    """Blocks whose bounding box meets the spherical shell
    | |x - c| - radius | <= thickness / 2, c = the domain centre."""
    c = n_per_axis * bsx / 2.0
    b = np.arange(n_per_axis)
    bz, by, bx = np.meshgrid(b, b, b, indexing="ij")
    lo = np.stack([bx, by, bz], -1).astype(np.float64) * bsx
    hi = lo + bsx
    dmin = np.linalg.norm(np.clip(c, lo, hi) - c, axis=-1)
    dmax = np.linalg.norm(np.maximum(np.abs(lo - c), np.abs(hi - c)), axis=-1)
    hit = (dmin <= radius + thickness / 2) & (dmax >= radius - thickness / 2)
    return np.nonzero(hit.reshape(-1))[0].astype(np.uint64)


@dataclass
class ShellProblem:
    """Single-level shell: 16^3 blocks of a size^3 domain intersecting the
    shell of radius 0.35*size and thickness 12 cells, U[-1, 1] values."""

    size: int
    bsx: int
    active: np.ndarray
    values: np.ndarray  # [n_active][bsx^3] f32


def shell_problem(size: int = 128, bsx: int = 16, seed: int = 1, radius_frac: float = 0.35, thickness: float = 12.0,
                  values: bool = True) -> ShellProblem:
    n = size // bsx
    active = shell_active_blocks(n, bsx, radius_frac * size, thickness)
    vals = None
    if values:
        rng = np.random.default_rng(seed)
        vals = rng.uniform(-1.0, 1.0, (len(active), bsx ** 3)).astype(np.float32)
    return ShellProblem(size, bsx, active, vals)


@dataclass
class FlipTransfer:
    """FLIP transfer workload: size^3 domain of bsx^3 blocks, 3 levels by the
    distance of a block centre to the sphere |x - c| = 0.35*size (< 16 cells
    -> level 0, < 48 -> level 1, else 2); 8 particles per level-0 cell,
    uniformly jittered inside the cell; velocities N(0, 1), mass 1."""

    size: int
    bsx: int
    levels: np.ndarray      # [n_blocks] u8
    fine_blocks: np.ndarray  # level-0 block ids
    pos: np.ndarray          # [n][3] f32
    vel: np.ndarray          # [n][3] f32
    mass: np.ndarray         # [n] f32

    @property
    def n(self) -> int:
        return len(self.mass)


def block_levels(size: int, bsx: int, radius: float, bands=(16.0, 48.0)) -> np.ndarray:
    n = size // bsx
    b = np.arange(n)
    bz, by, bx = np.meshgrid(b, b, b, indexing="ij")
    centre = (np.stack([bx, by, bz], -1).astype(np.float64) + 0.5) * bsx
    d = np.abs(np.linalg.norm(centre - size / 2.0, axis=-1) - radius).reshape(-1)
    lv = np.full(d.shape, 2, np.uint8)
    lv[d < bands[1]] = 1
    lv[d < bands[0]] = 0
    return lv


def flip_transfer(size: int = 256, bsx: int = 16, seed: int = 2, ppc: int = 8, radius_frac: float = 0.35,
                  particles: bool = True) -> FlipTransfer:
    levels = block_levels(size, bsx, radius_frac * size)
    fine = np.nonzero(levels == 0)[0].astype(np.uint64)
    if not particles:
        e = np.empty((0, 3), np.float32)
        return FlipTransfer(size, bsx, levels, fine, e, e, np.empty(0, np.float32))
    n_per_axis = size // bsx
    rng = np.random.default_rng(seed)
    cells = np.arange(bsx ** 3)
    lx, ly, lz = cells % bsx, (cells // bsx) % bsx, cells // (bsx * bsx)
    bx = (fine % n_per_axis).astype(np.int64)
    by = ((fine // n_per_axis) % n_per_axis).astype(np.int64)
    bz = (fine // (n_per_axis * n_per_axis)).astype(np.int64)
    cx = (bx[:, None] * bsx + lx[None, :]).reshape(-1)
    cy = (by[:, None] * bsx + ly[None, :]).reshape(-1)
    cz = (bz[:, None] * bsx + lz[None, :]).reshape(-1)
    origin = np.repeat(np.stack([cx, cy, cz], -1).astype(np.float32), ppc, axis=0)
    jitter = rng.random(origin.shape, dtype=np.float32)
    pos = origin + jitter
    # origin + jitter can round up to the next cell in f32: keep it inside
    pos = np.minimum(pos, np.nextafter(origin + 1, origin, dtype=np.float32))
    vel = rng.standard_normal(origin.shape, dtype=np.float32)
    mass = np.ones(len(pos), np.float32)
    return FlipTransfer(size, bsx, levels, fine, pos.astype(np.float32), vel, mass)


def block_cell_centres(size: int, bsx: int, bids: np.ndarray) -> np.ndarray:
    """Cell-centre coordinates [n_blocks][bsx^3][3] (f64) of the given blocks in
    the payload order x | y<<lg | z<<2lg."""
    n = size // bsx
    bids = np.asarray(bids, np.int64)
    cells = np.arange(bsx ** 3)
    lx, ly, lz = cells % bsx, (cells // bsx) % bsx, cells // (bsx * bsx)
    bx, by, bz = bids % n, (bids // n) % n, bids // (n * n)
    return np.stack([(bx[:, None] * bsx + lx[None, :]) + 0.5, (by[:, None] * bsx + ly[None, :]) + 0.5,
                     (bz[:, None] * bsx + lz[None, :]) + 0.5], -1)


def smooth_divergence_rhs(size: int, bsx: int, active: np.ndarray, seed: int = 4, n_blobs: int = 32,
                          sigma=(4.0, 16.0)) -> np.ndarray:
    """Right-hand side of the learned-preconditioner configuration: the
    divergence of a random smooth velocity field u = sum_i a_i g_i(x),
    g_i = exp(-|x - c_i|^2 / (2 sigma_i^2)), amplitudes a_i ~ N(0, 1)^3, sigma_i
    uniform in [4, 16] cells, centres at random cells of the active blocks.
    div u = sum_i -(a_i . (x - c_i)) / sigma_i^2 g_i(x), evaluated at cell
    centres.  Returns [n_active][bsx^3] f32 for the active blocks in ascending
    block-id order (the Poisson vector layout)."""
    rng = np.random.default_rng(seed)
    bids = np.unique(np.asarray(active, np.uint64)).astype(np.int64)
    x = block_cell_centres(size, bsx, bids).reshape(-1, 3)
    centres = x[rng.integers(0, len(x), n_blobs)]
    sig = rng.uniform(sigma[0], sigma[1], n_blobs)
    amp = rng.standard_normal((n_blobs, 3))
    out = np.zeros(len(x), np.float64)
    chunk = 1 << 20
    for s in range(0, len(x), chunk):
        xs = x[s:s + chunk]
        acc = np.zeros(len(xs), np.float64)
        for i in range(n_blobs):
            d = xs - centres[i]
            r2 = np.einsum("ij,ij->i", d, d)
            acc += -(d @ amp[i]) / sig[i] ** 2 * np.exp(-r2 / (2.0 * sig[i] ** 2))
        out[s:s + chunk] = acc
    return out.astype(np.float32).reshape(len(bids), bsx ** 3)


def batched_problems(n: int = 64, seed: int = 3, edges=(32, 64, 128, 256), block_sizes=(8, 16),
                     fraction=(0.05, 0.6)):
    """The batched-solve configuration: n problems, each a cube of edge drawn
    from `edges`, blocks of 8^3 or 16^3, an active fraction uniform in
    `fraction` made of the blocks closest to a random sphere surface (a shell
    of that volume fraction), right-hand side uniform in [-1, 1] with its
    mean removed.  Returns [(dims, bsx, active, rhs)], rhs [n_active][bsx^3]
    f32 in ascending block-id order."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        edge = int(rng.choice(edges))
        bsx = int(rng.choice(block_sizes))
        nb = edge // bsx
        f = rng.uniform(*fraction)
        b = np.arange(nb)
        bz, by, bx = np.meshgrid(b, b, b, indexing="ij")
        centre = (np.stack([bx, by, bz], -1).reshape(-1, 3) + 0.5) * bsx
        c = rng.uniform(0.3, 0.7, 3) * edge
        r = rng.uniform(0.2, 0.45) * edge
        d = np.abs(np.linalg.norm(centre - c, axis=1) - r)
        k = max(1, int(np.ceil(f * nb ** 3)))
        active = np.sort(np.argsort(d, kind="stable")[:k]).astype(np.uint64)
        rhs = rng.uniform(-1.0, 1.0, (k, bsx ** 3))
        rhs -= rhs.mean()
        out.append(((edge, edge, edge), bsx, active, rhs.astype(np.float32)))
    return out


def value_noise(p: np.ndarray, seed: int, octaves: int = 3, base: float = 64.0, amplitude: float = 10.0) -> np.ndarray:
    """Value noise at points p [n][3]: random values on lattices of spacing
    base / 2^o (o < octaves), trilinearly interpolated, amplitudes halving per
    octave, scaled so the octaves together span +-amplitude."""
    rng = np.random.default_rng(seed)
    out = np.zeros(len(p), np.float64)
    norm = sum(0.5 ** o for o in range(octaves))
    for o in range(octaves):
        h = base / 2 ** o
        q = p / h
        i0 = np.floor(q).astype(np.int64)
        f = q - i0
        m = int(np.max(i0)) + 2
        lat = rng.uniform(-1.0, 1.0, (m + 1, m + 1, m + 1))
        acc = np.zeros(len(p))
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    w = (f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) * (f[:, 2] if dz else 1 - f[:, 2])
                    acc += w * lat[np.clip(i0[:, 0] + dx, 0, m), np.clip(i0[:, 1] + dy, 0, m), np.clip(i0[:, 2] + dz, 0, m)]
        out += acc * (0.5 ** o)
    return out * (amplitude / norm)


@dataclass
class PhaseField:
    """The full phase-field FLIP step: size^3 domain of 16^3 blocks, a sphere
    of radius 0.3 size perturbed by 3-octave value noise of amplitude 10
    cells; 4 levels by the distance of a block centre to the surface (< 16
    cells: level 0, < 48: 1, < 112: 2, else 3); 8 particles per cell within
    12 cells of the surface (a band of width 24), velocities N(0, 1), mass 1;
    the phase field 0.5 (1 - tanh(phi / 2)) on the level-0 blocks."""

    size: int
    levels: np.ndarray      # [n_blocks] u8
    fine_blocks: np.ndarray
    phase: np.ndarray       # [n_fine][4096] f32
    pos: np.ndarray
    vel: np.ndarray
    mass: np.ndarray

    @property
    def n(self) -> int:
        return len(self.mass)


def phase_field(size: int = 512, seed: int = 5, ppc: int = 8, band: float = 12.0, particles: bool = True) -> PhaseField:
    bsx = 16
    nb = size // bsx
    c = size / 2.0
    r0 = 0.3 * size

    def phi(p):
        d = p - c
        rr = np.linalg.norm(d, axis=1)
        return rr - (r0 + value_noise(p, seed))

    b = np.arange(nb)
    bz, by, bx = np.meshgrid(b, b, b, indexing="ij")
    centre = (np.stack([bx, by, bz], -1).reshape(-1, 3) + 0.5) * bsx
    dist = np.abs(phi(centre))
    lv = np.full(nb ** 3, 3, np.uint8)
    lv[dist < 112] = 2
    lv[dist < 48] = 1
    lv[dist < 16] = 0
    fine = np.nonzero(lv == 0)[0].astype(np.uint64)
    cells = np.arange(bsx ** 3)
    lx, ly, lz = cells % bsx, (cells // bsx) % bsx, cells // (bsx * bsx)
    fb = fine.astype(np.int64)
    cx = ((fb % nb)[:, None] * bsx + lx[None, :]).reshape(-1)
    cy = (((fb // nb) % nb)[:, None] * bsx + ly[None, :]).reshape(-1)
    cz = ((fb // (nb * nb))[:, None] * bsx + lz[None, :]).reshape(-1)
    cc = np.stack([cx, cy, cz], -1).astype(np.float64) + 0.5
    ph = np.empty(len(cc))
    chunk = 1 << 21
    for s in range(0, len(cc), chunk):
        ph[s:s + chunk] = phi(cc[s:s + chunk])
    phase = (0.5 * (1.0 - np.tanh(ph / 2.0))).astype(np.float32).reshape(len(fine), bsx ** 3)
    if not particles:
        e = np.empty((0, 3), np.float32)
        return PhaseField(size, lv, fine, phase, e, e, np.empty(0, np.float32))
    inband = np.abs(ph) < band
    origin = np.repeat(cc[inband] - 0.5, ppc, axis=0).astype(np.float32)
    rng = np.random.default_rng(seed + 1)
    pos = origin + rng.random(origin.shape, dtype=np.float32)
    pos = np.minimum(pos, np.nextafter(origin + 1, origin, dtype=np.float32))
    vel = rng.standard_normal(origin.shape, dtype=np.float32)
    mass = np.ones(len(pos), np.float32)
    order = rng.permutation(len(pos))
    return PhaseField(size, lv, fine, phase, pos[order], vel[order], mass[order])


def bf16_bits(a: np.ndarray) -> np.ndarray:
    """f32 -> bf16 bit patterns, round to nearest even (the device store rule)."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    nan = (u & 0x7FFFFFFF) > 0x7F800000
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return np.where(nan, ((u >> 16) | 0x40).astype(np.uint16), r)
