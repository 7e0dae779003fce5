"""CPU oracle (test infrastructure only) for the learned preconditioner: the
block-sparse 3x3x3 convolution, its data and weight gradients, pooling,
upsampling and the U-Net built from them, in numpy FP64 with the same bf16
rounding points as the device network.

The crate has no learned preconditioner (it has no pressure solver at all),
so there is no reference to pin this against: parity is unpinned, and the
oracle restates the operations from their definitions.  Layouts follow the
device: a level's feature map is [cells][C] with cells in block order (block
k holds cells k*bs^3 ... (k+1)*bs^3 - 1, payload order x | y<<lg | z<<2lg),
blocks of the active set in ascending id order, absent neighbours zero.
Weights are [27][Cout][Cin], tap t = (dx+1) + 3 (dy+1) + 9 (dz+1).
"""
from __future__ import annotations

import numpy as np


# ---- bf16 ---------------------------------------------------------------------
def bf16_bits(a: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even f32 -> bf16 bit patterns (uint16)."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    nan = (u & 0x7FFFFFFF) > 0x7F800000
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return np.where(nan, ((u >> 16) | 0x40).astype(np.uint16), r)


def bf16_value(bits: np.ndarray) -> np.ndarray:
    return (np.asarray(bits, np.uint16).astype(np.uint32) << 16).view(np.float32)


def bf16_round(a: np.ndarray) -> np.ndarray:
    return bf16_value(bf16_bits(a)).astype(np.float64)


# ---- block neighbourhoods -----------------------------------------------------
def nbr27(active: np.ndarray, n_per_axis: int) -> np.ndarray:
    """[n][27] slot of each neighbour block (ascending-id slots), -1 if absent."""
    a = np.asarray(active, np.int64)
    slot = {int(b): i for i, b in enumerate(a)}
    n = n_per_axis
    out = np.full((len(a), 27), -1, np.int32)
    for i, b in enumerate(a):
        bx, by, bz = b % n, (b // n) % n, b // (n * n)
        for t in range(27):
            dx, dy, dz = t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1
            x, y, z = bx + dx, by + dy, bz + dz
            if 0 <= x < n and 0 <= y < n and 0 <= z < n:
                out[i, t] = slot.get(int(x + y * n + z * n * n), -1)
    return out


def tap_index(nbr: np.ndarray, lg: int) -> np.ndarray:
    """[cells][27] source cell of each tap, -1 outside the active blocks."""
    bs = 1 << lg
    nb = len(nbr)
    v = np.arange(bs ** 3)
    cx, cy, cz = v & (bs - 1), (v >> lg) & (bs - 1), v >> (2 * lg)
    out = np.full((nb * bs ** 3, 27), -1, np.int64)
    for t in range(27):
        dx, dy, dz = t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1
        gx, gy, gz = cx + dx, cy + dy, cz + dz
        ox = np.where(gx < 0, 0, np.where(gx >= bs, 2, 1))
        oy = np.where(gy < 0, 0, np.where(gy >= bs, 2, 1))
        oz = np.where(gz < 0, 0, np.where(gz >= bs, 2, 1))
        code = ox + 3 * oy + 9 * oz
        vv = (gx & (bs - 1)) | ((gy & (bs - 1)) << lg) | ((gz & (bs - 1)) << (2 * lg))
        kk = nbr[:, code]  # [nb][bs^3]
        src = kk.astype(np.int64) * bs ** 3 + vv[None, :]
        out[:, t] = np.where(kk >= 0, src, -1).reshape(-1)
    return out


def gather_taps(x: np.ndarray, taps: np.ndarray) -> np.ndarray:
    """[cells][27][C] shifted inputs (zero outside)."""
    xp = np.concatenate([x, np.zeros((1, x.shape[1]), x.dtype)], 0)
    idx = np.where(taps >= 0, taps, len(x))
    return xp[idx]


# ---- convolution --------------------------------------------------------------
def conv3(x: np.ndarray, w: np.ndarray, b, taps: np.ndarray) -> np.ndarray:
    """y[c][o] = b[o] + sum_t sum_i w[t][o][i] x[c + d(t)][i]  (FP64)."""
    g = gather_taps(np.asarray(x, np.float64), taps)  # [cells][27][Cin]
    y = np.einsum("cti,toi->co", g, np.asarray(w, np.float64), optimize=True)
    if b is not None:
        y = y + np.asarray(b, np.float64)[None, :]
    return y


def conv3_wgrad(x: np.ndarray, dy: np.ndarray, taps: np.ndarray) -> np.ndarray:
    """dw[t][o][i] = sum_c x[c + d(t)][i] dy[c][o]  (FP64)."""
    g = gather_taps(np.asarray(x, np.float64), taps)
    return np.einsum("cti,co->toi", g, np.asarray(dy, np.float64), optimize=True)


def conv3_dgrad(dy: np.ndarray, w: np.ndarray, taps: np.ndarray) -> np.ndarray:
    """dx[c'][i] = sum_t sum_o w[t][o][i] dy[c' - d(t)][o]: the forward
    convolution with the taps mirrored and the weights transposed."""
    wt = np.transpose(np.asarray(w, np.float64)[::-1], (0, 2, 1))
    return conv3(dy, wt, None, taps)
