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


# ---- the network ----------------------------------------------------------------
# layer table (level, cin, cout, cin_real, cout_real, relu), the device order
LAYERS = [(0, 16, 16, 1, 16, True), (1, 16, 32, 16, 32, True), (2, 32, 64, 32, 64, True), (2, 64, 64, 64, 64, True),
          (2, 64, 32, 64, 32, False), (1, 32, 32, 32, 32, True), (1, 32, 16, 32, 16, False), (0, 16, 16, 16, 1, False)]
L0A, L1A, L2A, L2B, L2C, L1C, L1D, L0C = range(8)


def param_offsets():
    offs, o = [], 0
    for (_, ci, co, _, _, _) in LAYERS:
        offs.append((o, o + 27 * ci * co))
        o += 27 * ci * co + co
    return offs, o


def children(nb: int, lgc: int) -> np.ndarray:
    """[coarse cells][8] index of each child at level lgc+1 (same block)."""
    bc, lgf = 1 << lgc, lgc + 1
    v = np.arange(bc ** 3)
    cx, cy, cz = v & (bc - 1), (v >> lgc) & (bc - 1), v >> (2 * lgc)
    out = np.empty((nb * bc ** 3, 8), np.int64)
    for d in range(8):
        fx, fy, fz = 2 * cx + (d & 1), 2 * cy + ((d >> 1) & 1), 2 * cz + (d >> 2)
        f = fx | (fy << lgf) | (fz << (2 * lgf))
        out[:, d] = (np.arange(nb)[:, None] * (8 * bc ** 3) + f[None, :]).reshape(-1)
    return out


class UNet:
    """The device network restated in numpy.  With rounding=True every value
    the device stores in bf16 is rounded to bf16 here too (the rest is FP64);
    with rounding=False everything is FP64 (for finite-difference checks)."""

    def __init__(self, nbr: np.ndarray, params: np.ndarray, out_scale: float = 1.0, rounding: bool = True):
        self.nb = len(nbr)
        self.taps = [tap_index(nbr, 4 - l) for l in range(3)]
        self.kids = [None, children(self.nb, 3), children(self.nb, 2)]  # kids[l]: level-l cells -> level l-1
        self.offs, self.n_params = param_offsets()
        self.params = np.asarray(params, np.float64)
        self.S = float(out_scale)
        self.rounding = rounding

    def r(self, a):
        return bf16_round(a) if self.rounding else np.asarray(a, np.float64)

    def w(self, i):
        (o, ob), (_, ci, co, _, _, _) = self.offs[i], LAYERS[i]
        w = self.params[o:o + 27 * ci * co].reshape(27, co, ci)
        return self.r(w), self.params[ob:ob + co]

    def pool(self, a, lc, scale):
        return self.r(a[self.kids[lc]].sum(1) * scale)

    def up(self, c, lf):
        """copy coarse values (level lf+1) to the 8 children at level lf"""
        out = np.empty((len(c) * 8, c.shape[1]))
        out[self.kids[lf + 1]] = c[:, None, :]
        return out

    def conv(self, i, x, relu):
        w, b = self.w(i)
        y = conv3(x, w, b, self.taps[LAYERS[i][0]])
        return np.maximum(y, 0) if relu else y

    def forward(self, r):
        r = np.asarray(r, np.float32)
        s_in = np.sqrt(np.mean(r.astype(np.float64) ** 2))
        x = np.zeros((len(r), 16))
        x[:, 0] = (r * np.float32(1.0 / s_in)).astype(np.float32) if self.rounding else r / s_in
        x0 = self.r(x)
        a0 = self.r(self.conv(L0A, x0, True))
        p1 = self.pool(a0, 1, 0.125)
        a1 = self.r(self.conv(L1A, p1, True))
        p2 = self.pool(a1, 2, 0.125)
        a2 = self.r(self.conv(L2A, p2, True))
        a3 = self.r(self.conv(L2B, a2, True))
        c2 = self.r(self.conv(L2C, a3, False))
        u1 = self.r(np.maximum(self.up(c2, 1) + a1, 0))
        a4 = self.r(self.conv(L1C, u1, True))
        c1 = self.r(self.conv(L1D, a4, False))
        u0 = self.r(np.maximum(self.up(c1, 0) + a0, 0))
        y = self.conv(L0C, u0, False)[:, 0]
        self.cache = dict(s_in=s_in, x0=x0, a0=a0, p1=p1, a1=a1, p2=p2, a2=a2, a3=a3, c2=c2, u1=u1, a4=a4, c1=c1, u0=u0)
        return y

    def loss(self, r, e):
        y = self.forward(r)
        eh = np.asarray(e, np.float64) / self.cache["s_in"]
        d = self.S * y - eh
        return np.sum(d * d) / np.sum(eh * eh), y, eh

    def grads(self, r, e):
        """(loss, flat gradient) of the loss w.r.t. the parameters."""
        L, y, eh = self.loss(r, e)
        c = self.cache
        g = np.zeros(self.n_params)
        dy = np.zeros((len(y), 16))
        dy[:, 0] = 2 * self.S * (self.S * y - eh) / np.sum(eh * eh)
        dy = self.r(dy)

        def wgrad(i, x, d):
            (o, ob), (lv, ci, co, cir, cor, _) = self.offs[i], LAYERS[i]
            gw = conv3_wgrad(x, d, self.taps[lv])
            gw[:, cor:, :] = 0
            gw[:, :, cir:] = 0
            g[o:o + 27 * ci * co] = gw.reshape(-1)
            gb = d.sum(0)
            gb[cor:] = 0
            g[ob:ob + co] = gb

        def dgrad(i, d, mask):
            w, _ = self.w(i)
            out = conv3_dgrad(d, w, self.taps[LAYERS[i][0]])
            return out if mask is None else np.where(mask > 0, out, 0.0)

        wgrad(L0C, c["u0"], dy)
        du0m = self.r(dgrad(L0C, dy, c["u0"]))
        dc1 = self.pool(du0m, 1, 1.0)
        wgrad(L1D, c["a4"], dc1)
        da4m = self.r(dgrad(L1D, dc1, c["a4"]))
        wgrad(L1C, c["u1"], da4m)
        du1m = self.r(dgrad(L1C, da4m, c["u1"]))
        dc2 = self.pool(du1m, 2, 1.0)
        wgrad(L2C, c["a3"], dc2)
        da3m = self.r(dgrad(L2C, dc2, c["a3"]))
        wgrad(L2B, c["a2"], da3m)
        da2m = self.r(dgrad(L2B, da3m, c["a2"]))
        wgrad(L2A, c["p2"], da2m)
        dp2 = dgrad(L2A, da2m, None)
        da1m = self.r(np.where(c["a1"] > 0, du1m + 0.125 * self.up(dp2, 1), 0.0))
        wgrad(L1A, c["p1"], da1m)
        dp1 = dgrad(L1A, da1m, None)
        da0m = self.r(np.where(c["a0"] > 0, du0m + 0.125 * self.up(dp1, 0), 0.0))
        wgrad(L0A, c["x0"], da0m)
        return L, g
