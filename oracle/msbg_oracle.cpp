// msbg_oracle.cpp -- CPU restatement of the msbg-rs sparse-grid hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the CUDA
// library and the timed multi-core CPU baseline.  Nothing in the product path
// links, loads or calls it.  Every function restates a reference function and
// cites the reference file:line it follows (paths are relative to the msbg-rs
// source tree).  Arithmetic follows the reference operation by operation:
// left-associative `+` chains, an explicit fmaf() wherever the reference calls
// `mul_add`, IEEE division and square root, no contraction (the Makefile
// builds with -ffp-contract=off).
//
// Parity status: the restated A-rows (grid semantics, halo, three stencils,
// 8-colour sweep, Morton key, bucket sort, P2G, MAC ops, trilinear G2P,
// downsample) are pinned against the reference's golden vectors in
// tests/test_oracle_golden.py.  The FP64 Poisson oracle (matvec, weighted
// Jacobi, V-cycle, PCG) has no reference implementation: parity unpinned.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// Grid view.  The reference's SparseGrid (sparse_grid.rs:61-435) keeps a hash
// map bid -> block; the oracle uses a dense table with the same meaning:
// table[bid] >= 0 is a value-block slot, -1 is absent/empty, -2 the full dummy.
// ---------------------------------------------------------------------------
struct Grid {
    int64_t sx, sy, sz;
    int32_t bsx;
    int64_t nx, ny, nz, nxy;
    const int32_t* table;
    float* data;  // [slots][bsx^3]
    float empty_value, full_value;
};

inline int ilog2(int v) { int l = 0; while ((1 << l) < v) ++l; return l; }

// boundary.rs:7-56
enum BC { BC_CLAMP = 0, BC_NEUMANN = 1, BC_DIRICHLET = 2 };

inline int32_t reflect_axis(int32_t g, int32_t max) {
    int32_t period = 2 * (max + 1);
    int32_t r = g % period;
    if (r < 0) r += period;
    return r > max ? period - 1 - r : r;
}

// boundary.rs:33-42 resolve_axis: returns false only for Dirichlet out of range.
inline bool resolve_axis(int32_t g, int32_t max, int bc, int32_t* out) {
    if (g >= 0 && g <= max) { *out = g; return true; }
    if (bc == BC_CLAMP) { *out = g < 0 ? 0 : max; return true; }
    if (bc == BC_NEUMANN) { *out = reflect_axis(g, max); return true; }
    return false;
}

struct Dummies {
    std::vector<float> empty, full;
    Dummies(const Grid& g) {
        size_t n = (size_t)g.bsx * g.bsx * g.bsx;
        empty.assign(n, g.empty_value);
        full.assign(n, g.full_value);
    }
};

// sparse_grid.rs:402-411 block_data_ptr: absent -> empty dummy, full -> full dummy.
inline const float* block_data_ptr(const Grid& g, const Dummies& d, int64_t bid) {
    int32_t s = g.table[bid];
    if (s >= 0) return g.data + (size_t)s * g.bsx * g.bsx * g.bsx;
    if (s == -2) return d.full.data();
    return d.empty.data();
}

// ---------------------------------------------------------------------------
// halo.rs:31-170 HaloBlock::fill::<HALO, FULL>
// ---------------------------------------------------------------------------
void halo_fill(const Grid& g, const Dummies& dm, int64_t bid, int HALO, bool FULL, int bc,
               float* dst) {
    const int bsx = g.bsx, lg = ilog2(bsx), mask = bsx - 1, HSX = bsx + 2 * HALO;
    const int32_t nx = (int32_t)g.nx, ny = (int32_t)g.ny, nz = (int32_t)g.nz;
    const int32_t sx = (int32_t)g.sx, sy = (int32_t)g.sy, sz = (int32_t)g.sz;
    const float empty = g.empty_value;
    const int32_t bx0 = (int32_t)(bid % g.nx), by0 = (int32_t)((bid / g.nx) % g.ny),
                  bz0 = (int32_t)(bid / g.nxy);
    const int32_t x0 = bx0 * bsx;
    const int n = 2 * HALO + 1;
    const float* ptrs[125];
    for (int dz = 0; dz < n; ++dz)
        for (int dy = 0; dy < n; ++dy)
            for (int dx = 0; dx < n; ++dx) {
                int32_t bx = bx0 + dx - HALO, by = by0 + dy - HALO, bz = bz0 + dz - HALO;
                const float* p = dm.empty.data();
                if (bx >= 0 && bx < nx && by >= 0 && by < ny && bz >= 0 && bz < nz)
                    p = block_data_ptr(g, dm, (int64_t)bx + (int64_t)by * g.nx + (int64_t)bz * g.nxy);
                ptrs[dx + n * dy + n * n * dz] = p;
            }
    auto read = [&](int32_t x, int32_t y, int32_t z) -> float {
        int idx = ((x >> lg) - bx0 + HALO) + n * ((y >> lg) - by0 + HALO) +
                  n * n * ((z >> lg) - bz0 + HALO);
        int vid = (x & mask) | ((y & mask) << lg) | ((z & mask) << (2 * lg));
        return ptrs[idx][vid];
    };
    int32_t rxl[2], rxr[2];
    bool okl[2], okr[2];
    for (int j = 0; j < HALO; ++j) {
        okl[j] = resolve_axis(x0 - HALO + j, sx - 1, bc, &rxl[j]);
        okr[j] = resolve_axis(x0 + bsx + j, sx - 1, bc, &rxr[j]);
    }
    for (int z = 0; z < HSX; ++z) {
        int32_t rz; bool okz = resolve_axis(bz0 * bsx + z - HALO, sz - 1, bc, &rz);
        for (int y = 0; y < HSX; ++y) {
            int32_t ry; bool oky = resolve_axis(by0 * bsx + y - HALO, sy - 1, bc, &ry);
            float* row = dst + (size_t)z * HSX * HSX + (size_t)y * HSX;
            if (oky && okz && x0 + bsx <= sx) {
                int idx = HALO + n * ((ry >> lg) - by0 + HALO) + n * n * ((rz >> lg) - bz0 + HALO);
                const float* p = ptrs[idx];
                int vid = ((ry & mask) << lg) | ((rz & mask) << (2 * lg));
                for (int i = 0; i < bsx; ++i) row[HALO + i] = p[vid + i];
            } else if (oky && okz) {
                for (int i = 0; i < bsx; ++i) {
                    int32_t rx;
                    row[HALO + i] = resolve_axis(x0 + i, sx - 1, bc, &rx) ? read(rx, ry, rz) : empty;
                }
            } else {
                for (int i = 0; i < bsx; ++i) row[HALO + i] = empty;
            }
            if (FULL || (y >= HALO && y < HALO + bsx && z >= HALO && z < HALO + bsx)) {
                for (int j = 0; j < HALO; ++j) {
                    row[j] = (okl[j] && oky && okz) ? read(rxl[j], ry, rz) : empty;
                    row[HALO + bsx + j] = (okr[j] && oky && okz) ? read(rxr[j], ry, rz) : empty;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// halo.rs:187-358 fill_multires: same-level neighbours from `fine`, coarser
// neighbours (levels[b] > levels[bid]) ghost-sampled from `coarse` at >>1.
// The empty value is 0.0 here (halo.rs:211).
// ---------------------------------------------------------------------------
void fill_multires(const Grid& fine, const Grid& coarse, const uint8_t* levels, int64_t bid,
                   int HALO, bool FULL, int bc, float* dst) {
    const int bsx = fine.bsx, lg = ilog2(bsx), mask = bsx - 1, HSX = bsx + 2 * HALO;
    const int bsc = coarse.bsx, clg = ilog2(bsc), cmask = bsc - 1;
    const int32_t nx = (int32_t)fine.nx, ny = (int32_t)fine.ny, nz = (int32_t)fine.nz;
    const int32_t sx = (int32_t)fine.sx, sy = (int32_t)fine.sy, sz = (int32_t)fine.sz;
    const float empty = 0.0f;
    const int32_t bx0 = (int32_t)(bid % fine.nx), by0 = (int32_t)((bid / fine.nx) % fine.ny),
                  bz0 = (int32_t)(bid / fine.nxy);
    const int32_t x0 = bx0 * bsx;
    const uint8_t lvl = levels[bid];
    std::vector<float> zf((size_t)bsx * bsx * bsx, 0.0f), zc((size_t)bsc * bsc * bsc, 0.0f);
    const int n = 2 * HALO + 1;
    const float* ptrs[125];
    const float* cptrs[125];
    for (int i = 0; i < 125; ++i) { ptrs[i] = zf.data(); cptrs[i] = nullptr; }
    for (int dz = 0; dz < n; ++dz)
        for (int dy = 0; dy < n; ++dy)
            for (int dx = 0; dx < n; ++dx) {
                int idx = dx + n * dy + n * n * dz;
                int32_t bx = bx0 + dx - HALO, by = by0 + dy - HALO, bz = bz0 + dz - HALO;
                if (bx >= 0 && bx < nx && by >= 0 && by < ny && bz >= 0 && bz < nz) {
                    int64_t b = (int64_t)bx + (int64_t)by * fine.nx + (int64_t)bz * fine.nxy;
                    if (levels[b] > lvl) {
                        int32_t s = coarse.table[b];
                        cptrs[idx] = s >= 0 ? coarse.data + (size_t)s * bsc * bsc * bsc : zc.data();
                    } else {
                        int32_t s = fine.table[b];
                        ptrs[idx] = s >= 0 ? fine.data + (size_t)s * bsx * bsx * bsx : zf.data();
                    }
                }
            }
    auto read = [&](int32_t x, int32_t y, int32_t z) -> float {
        int idx = ((x >> lg) - bx0 + HALO) + n * ((y >> lg) - by0 + HALO) +
                  n * n * ((z >> lg) - bz0 + HALO);
        if (cptrs[idx]) {
            int vid = ((x >> 1) & cmask) | (((y >> 1) & cmask) << clg) | (((z >> 1) & cmask) << (2 * clg));
            return cptrs[idx][vid];
        }
        int vid = (x & mask) | ((y & mask) << lg) | ((z & mask) << (2 * lg));
        return ptrs[idx][vid];
    };
    int32_t rxl[2], rxr[2];
    bool okl[2], okr[2];
    for (int j = 0; j < HALO; ++j) {
        okl[j] = resolve_axis(x0 - HALO + j, sx - 1, bc, &rxl[j]);
        okr[j] = resolve_axis(x0 + bsx + j, sx - 1, bc, &rxr[j]);
    }
    for (int z = 0; z < HSX; ++z) {
        int32_t rz; bool okz = resolve_axis(bz0 * bsx + z - HALO, sz - 1, bc, &rz);
        for (int y = 0; y < HSX; ++y) {
            int32_t ry; bool oky = resolve_axis(by0 * bsx + y - HALO, sy - 1, bc, &ry);
            float* row = dst + (size_t)z * HSX * HSX + (size_t)y * HSX;
            if (oky && okz && x0 + bsx <= sx) {
                int idx = HALO + n * ((ry >> lg) - by0 + HALO) + n * n * ((rz >> lg) - bz0 + HALO);
                if (cptrs[idx]) {
                    for (int i = 0; i < bsx; ++i) {
                        int32_t rx;
                        row[HALO + i] = resolve_axis(x0 + i, sx - 1, bc, &rx) ? read(rx, ry, rz) : empty;
                    }
                } else {
                    int vid = ((ry & mask) << lg) | ((rz & mask) << (2 * lg));
                    for (int i = 0; i < bsx; ++i) row[HALO + i] = ptrs[idx][vid + i];
                }
            } else if (oky && okz) {
                for (int i = 0; i < bsx; ++i) {
                    int32_t rx;
                    row[HALO + i] = resolve_axis(x0 + i, sx - 1, bc, &rx) ? read(rx, ry, rz) : empty;
                }
            } else {
                for (int i = 0; i < bsx; ++i) row[HALO + i] = empty;
            }
            if (FULL || (y >= HALO && y < HALO + bsx && z >= HALO && z < HALO + bsx)) {
                for (int j = 0; j < HALO; ++j) {
                    row[j] = (okl[j] && oky && okz) ? read(rxl[j], ry, rz) : empty;
                    row[HALO + bsx + j] = (okr[j] && oky && okz) ? read(rxr[j], ry, rz) : empty;
                }
            }
        }
    }
}

inline float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// laplacian.rs:16-70 (7 taps; mul_add at :53, :58, :60)
void kernel_laplacian(const float* h, int bsx, float dt, bool clamp01, float* out) {
    const int HSX = bsx + 2, dy = HSX, dz = HSX * HSX;
    int o = 0;
    for (int z = 1; z <= bsx; ++z)
        for (int y = 1; y <= bsx; ++y)
            for (int x = 1; x <= bsx; ++x, ++o) {
                int i = z * dz + y * dy + x;
                float c = h[i], lx = h[i - 1], rx = h[i + 1], dyu = h[i - dy], dyd = h[i + dy],
                      dzb = h[i - dz], dzf = h[i + dz];
                float nb = lx + rx;
                nb = nb + dyu; nb = nb + dyd; nb = nb + dzb; nb = nb + dzf;
                float lap = fmaf(c, -6.0f, nb);
                float fx = (rx - lx) * 0.5f, fy = (dyd - dyu) * 0.5f, fz = (dzf - dzb) * 0.5f;
                float g = sqrtf(fmaf(fx, fx, fmaf(fy, fy, fz * fz)));
                float nv = fmaf(dt * lap, g, c);
                out[o] = clamp01 ? clampf(nv, 0.0f, 1.0f) : nv;
            }
}

// meancurv.rs:17-107 (19 taps; mul_add at :84-92)
void kernel_meancurv(const float* h, int bsx, float dt, bool clamp01, float* out) {
    const int HSX = bsx + 2, dy = HSX, dz = HSX * HSX;
    int o = 0;
    for (int z = 1; z <= bsx; ++z)
        for (int y = 1; y <= bsx; ++y)
            for (int x = 1; x <= bsx; ++x, ++o) {
                int i = z * dz + y * dy + x;
                float f0 = h[i], f1 = h[i - 1], f2 = h[i + 1], f3 = h[i - dy], f4 = h[i + dy],
                      f5 = h[i - dz], f6 = h[i + dz];
                float fx = (f2 - f1) * 0.5f, fy = (f4 - f3) * 0.5f, fz = (f6 - f5) * 0.5f;
                float fxx = (f1 + f2) - 2.0f * f0, fyy = (f3 + f4) - 2.0f * f0,
                      fzz = (f5 + f6) - 2.0f * f0;
                float d1 = h[i + 1 + dy], d2 = h[i + 1 - dy], d3 = h[i - 1 + dy], d4 = h[i - 1 - dy];
                float d5 = h[i + 1 + dz], d6 = h[i + 1 - dz], d7 = h[i - 1 + dz], d8 = h[i - 1 - dz];
                float d9 = h[i + dy + dz], d10 = h[i + dy - dz], d11 = h[i - dy + dz],
                      d12 = h[i - dy - dz];
                float fyx = (((d1 - d2) - d3) + d4) * 0.25f;
                float fzx = (((d5 - d6) - d7) + d8) * 0.25f;
                float fzy = (((d9 - d10) - d11) + d12) * 0.25f;
                float cross = (fx * (fy * fyx) + fx * (fz * fzx)) + fy * (fz * fzy);
                float hnum = fmaf(fy * fy + fz * fz, fxx,
                                  fmaf(fx * fx + fz * fz, fyy, fmaf(fx * fx + fy * fy, fzz, -2.0f * cross)));
                float grad = fmaf(fx, fx, fmaf(fy, fy, fz * fz));
                float hc = grad > 1e-7f ? hnum / grad : 0.0f;
                float d = clampf(dt * hc, -0.1f, 0.1f);
                float nv = f0 + d;
                out[o] = clamp01 ? clampf(nv, 0.0f, 1.0f) : nv;
            }
}

// bilaplacian.rs:15-97 (25 taps; mul_add at :82)
void kernel_bilaplacian(const float* h, int bsx, float dt, bool clamp01, float* out) {
    const int HSX = bsx + 4, dy = HSX, dz = HSX * HSX;
    int o = 0;
    for (int z = 2; z <= bsx + 1; ++z)
        for (int y = 2; y <= bsx + 1; ++y)
            for (int x = 2; x <= bsx + 1; ++x, ++o) {
                int i = z * dz + y * dy + x;
                float f0 = h[i], f1 = h[i - 1], f2 = h[i + 1], f3 = h[i - dy], f4 = h[i + dy],
                      f5 = h[i - dz], f6 = h[i + dz];
                float g1 = h[i - 2], g2 = h[i + 2], g3 = h[i - 2 * dy], g4 = h[i + 2 * dy],
                      g5 = h[i - 2 * dz], g6 = h[i + 2 * dz];
                float s1 = f1 + f2; s1 = s1 + f3; s1 = s1 + f4; s1 = s1 + f5; s1 = s1 + f6;
                float s2 = g1 + g2; s2 = s2 + g3; s2 = s2 + g4; s2 = s2 + g5; s2 = s2 + g6;
                float sd = h[i + 1 + dy] + h[i + 1 - dy];
                sd = sd + h[i - 1 + dy]; sd = sd + h[i - 1 - dy];
                sd = sd + h[i + 1 + dz]; sd = sd + h[i + 1 - dz];
                sd = sd + h[i - 1 + dz]; sd = sd + h[i - 1 - dz];
                sd = sd + h[i + dy + dz]; sd = sd + h[i + dy - dz];
                sd = sd + h[i - dy + dz]; sd = sd + h[i - dy - dz];
                float hv = ((42.0f * f0 - 12.0f * s1) + s2) + 2.0f * sd;
                float fx = (f2 - f1) * 0.5f, fy = (f4 - f3) * 0.5f, fz = (f6 - f5) * 0.5f;
                float g = sqrtf(fmaf(fx, fx, fmaf(fy, fy, fz * fz)));
                float upd = (dt * hv) * g;
                float d = clampf(-upd, -0.1f, 0.1f);
                float nv = f0 + d;
                out[o] = clamp01 ? clampf(nv, 0.0f, 1.0f) : nv;
            }
}

// multires/sort.rs:8-22
inline uint64_t spread(uint64_t v) {
    v &= 0x1fffffULL;
    v = (v | (v << 32)) & 0x001f00000000ffffULL;
    v = (v | (v << 16)) & 0x001f0000ff0000ffULL;
    v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
    v = (v | (v << 2)) & 0x1249249249249249ULL;
    return v;
}
inline uint64_t morton3(uint64_t x, uint64_t y, uint64_t z) {
    return spread(x) | (spread(y) << 1) | (spread(z) << 2);
}

// Storage element conversions (stencil.rs:142-192 StoreBack, sample.rs:45-70 Dequant).
enum DType { DT_F32 = 0, DT_U16 = 1, DT_BF16 = 2, DT_U8 = 3, DT_F16 = 4 };
inline float bf16_to_f32(uint16_t b) { uint32_t u = (uint32_t)b << 16; float f; memcpy(&f, &u, 4); return f; }
inline uint16_t f32_to_bf16_rn(float f) {
    uint32_t u; memcpy(&u, &f, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40);  // quiet NaN
    uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return (uint16_t)(u >> 16);
}
// stencil.rs:160-174: round(v * 65535) half away from zero, then u16.
inline uint16_t f32_to_density(float v) {
    float r = roundf(v * 65535.0f);
    if (!(r > 0.0f)) r = 0.0f;
    if (r > 65535.0f) r = 65535.0f;
    return (uint16_t)r;
}
inline float density_to_f32(uint16_t v) { return (float)v * (1.0f / 65535.0f); }

// Density8 (channel.rs:155-190): read linearly, q / 255 (sample.rs:64-70);
// a plain write rounds half away from zero and saturates (from_unit,
// channel.rs:378-382).
inline float density8_to_f32(uint8_t q) { return (float)q * (1.0f / 255.0f); }
inline uint8_t f32_to_density8(float v) {
    float r = roundf(v * 255.0f);
    if (!(r > 0.0f)) r = 0.0f;
    if (r > 255.0f) r = 255.0f;
    return (uint8_t)r;
}
// The smoother's Density8 write-back (stencil.rs:176-192): sqrt compression,
// then floor + 1 when the draw u lies below the fraction.  The float -> i32
// conversion is the x86 one (NaN or out of range gives INT_MIN) and the
// i32 -> u8 cast wraps.
inline uint8_t density8_store_sr(float v, float u) {
    float vf = sqrtf(v) * 255.0f;
    float fl = floorf(vf);
    float frac = vf - fl;
    float r = u < frac ? fl + 1.0f : fl;
    int32_t i = (r >= -2147483648.0f && r < 2147483648.0f) ? (int32_t)r : INT32_MIN;
    return (uint8_t)(i & 0xff);
}

// SimdRng<W> (stencil.rs:103-132): W lanes seeded by a murmur finaliser of
// seed ^ lane * 0x9e3779b9 (zero replaced by 0xdeadbeef); each draw
// multiplies every lane by 16807 and maps state >> 9 into [1, 2), minus 1.
struct LaneRng {
    uint32_t s[16];
    int w;
    LaneRng(uint32_t seed, int lanes) : w(lanes) {
        for (int l = 0; l < 16; ++l) {
            uint32_t h = seed ^ ((uint32_t)l * 0x9e3779b9u);
            h ^= h >> 16;
            h *= 0x85ebca6bu;
            h ^= h >> 13;
            h *= 0xc2b2ae35u;
            h ^= h >> 16;
            s[l] = h ? h : 0xdeadbeefu;
        }
    }
    void next(float* u) {
        for (int l = 0; l < w; ++l) {
            s[l] *= 16807u;
            uint32_t bits = (s[l] >> 9) | 0x3f800000u;
            float f;
            memcpy(&f, &bits, 4);
            u[l] = f - 1.0f;
        }
    }
};

// IEEE 754 binary16, written from the format: 1 sign, 5 exponent (bias 15),
// 10 fraction bits; conversions from f32 round to nearest, ties to even.
inline uint16_t f32_to_f16_rn(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u, ax = x & 0x7fffffffu;
    if (ax > 0x7f800000u) return (uint16_t)(sign | 0x7e00u);   // NaN
    if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);  // >= 65520 rounds to infinity
    if (ax >= 0x38800000u) {                                    // normal: >= 2^-14
        const uint32_t e = (ax >> 23) - 127 + 15, m = ax & 0x7fffffu;
        uint32_t h = (e << 10) | (m >> 13);
        const uint32_t rem = m & 0x1fffu;
        if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) ++h;  // a carry moves into the exponent
        return (uint16_t)(sign | h);
    }
    const uint32_t e = ax >> 23;  // subnormal result, unit 2^-24
    if (e == 0) return (uint16_t)sign;
    const uint32_t m = (ax & 0x7fffffu) | 0x800000u;  // value m * 2^(e - 150)
    const uint32_t shift = 126 - e;                  // m * 2^(e - 126) units; shift >= 14
    if (shift >= 32) return (uint16_t)sign;
    uint32_t h = m >> shift;
    const uint32_t rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1);
    if (rem > half || (rem == half && (h & 1u))) ++h;
    return (uint16_t)(sign | h);
}
inline float f16_to_f32(uint16_t h) {
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    uint32_t bits;
    if (e == 0) {
        const float v = ldexpf((float)m, -24);
        memcpy(&bits, &v, 4);
        bits |= sign;
    } else if (e == 31) {
        bits = sign | 0x7f800000u | (m << 13);
    } else {
        bits = sign | ((e - 15 + 127) << 23) | (m << 13);
    }
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

}  // namespace

extern "C" {

// -------------------------------------------------------------------------
// Exported oracle entry points (called from oracle/oracle.py via ctypes).
// -------------------------------------------------------------------------
struct OracleGrid {  // mirrors Grid, C layout for ctypes
    int64_t sx, sy, sz;
    int32_t bsx, _pad;
    int64_t nx, ny, nz, nxy;
    const int32_t* table;
    float* data;
    float empty_value, full_value;
};

static Grid to_grid(const OracleGrid* o) {
    Grid g;
    g.sx = o->sx; g.sy = o->sy; g.sz = o->sz; g.bsx = o->bsx;
    g.nx = o->nx; g.ny = o->ny; g.nz = o->nz; g.nxy = o->nxy;
    g.table = o->table; g.data = o->data;
    g.empty_value = o->empty_value; g.full_value = o->full_value;
    return g;
}

void or_halo_fill(const OracleGrid* og, int64_t bid, int halo, int full, int bc, float* out) {
    Grid g = to_grid(og);
    Dummies d(g);
    halo_fill(g, d, bid, halo, full != 0, bc, out);
}

void or_fill_multires(const OracleGrid* fine, const OracleGrid* coarse, const uint8_t* levels,
                      int64_t bid, int halo, int full, int bc, float* out) {
    fill_multires(to_grid(fine), to_grid(coarse), levels, bid, halo, full != 0, bc, out);
}

// stencil: 0 Laplacian, 1 MeanCurvature, 2 BiLaplacian (solver.rs:44-51)
void or_kernel(int stencil, const float* halo, int bsx, float dt, int clamp01, float* out) {
    if (stencil == 0) kernel_laplacian(halo, bsx, dt, clamp01 != 0, out);
    else if (stencil == 1) kernel_meancurv(halo, bsx, dt, clamp01 != 0, out);
    else kernel_bilaplacian(halo, bsx, dt, clamp01 != 0, out);
}

uint64_t or_morton3(uint64_t x, uint64_t y, uint64_t z) { return morton3(x, y, z); }

// solver.rs:247-267 build_color_buckets + solver.rs:187-217 run: serial
// colour-ordered in-place sweep (equal to the parallel sweep, solver.rs:363-394).
// `elem` selects the storage type; for u16/bf16 `raw` holds the stored
// elements and the halo dequantizes them (Dequant::copy_row), the store
// re-quantizes (StoreBack::store_chunk).  `threads` > 1 runs each colour's
// blocks in parallel (the timed CPU baseline).
static uint64_t sweep_impl(const OracleGrid* og, void* raw, int elem, const int64_t* active,
                           int64_t n_active, int stencil, float dt, int iterations, int clamp01,
                           int threads, const OracleGrid* coarse, const uint8_t* levels,
                           uint32_t seed = 0xdeadbeefu, int lanes = 16, uint64_t stream_pos = 0) {
    Grid g = to_grid(og);
    const int bsx = g.bsx;
    const size_t N = (size_t)bsx * bsx * bsx;
    const int HALO = stencil == 2 ? 2 : 1;
    const bool FULL = stencil != 0;
    const int HSX = bsx + 2 * HALO;
    // For quantized storage keep an f32 shadow the halo reads from: the
    // reference dequantizes on every gather, which is what a f32 shadow of
    // the dequantized values reproduces as long as it is refreshed on store.
    int64_t n_slots = 0;
    for (int64_t b = 0; b < g.nx * g.ny * g.nz; ++b) n_slots = std::max<int64_t>(n_slots, g.table[b] + 1);
    std::vector<float> shadow;
    if (elem != DT_F32) {
        shadow.resize((size_t)n_slots * N);
        for (size_t i = 0; i < shadow.size(); ++i)
            shadow[i] = elem == DT_U16   ? density_to_f32(((uint16_t*)raw)[i])
                        : elem == DT_U8  ? density8_to_f32(((uint8_t*)raw)[i])
                        : elem == DT_F16 ? f16_to_f32(((uint16_t*)raw)[i])
                                         : bf16_to_f32(((uint16_t*)raw)[i]);
        g.data = shadow.data();
    } else {
        g.data = (float*)raw;
    }
    if (elem == DT_U16) g.empty_value = density_to_f32(f32_to_density(g.empty_value)), g.full_value = density_to_f32(f32_to_density(g.full_value));
    if (elem == DT_BF16) g.empty_value = bf16_to_f32(f32_to_bf16_rn(g.empty_value)), g.full_value = bf16_to_f32(f32_to_bf16_rn(g.full_value));
    if (elem == DT_U8) g.empty_value = density8_to_f32(f32_to_density8(g.empty_value)), g.full_value = density8_to_f32(f32_to_density8(g.full_value));
    if (elem == DT_F16) g.empty_value = f16_to_f32(f32_to_f16_rn(g.empty_value)), g.full_value = f16_to_f32(f32_to_f16_rn(g.full_value));
    Dummies dm(g);
    // Density8: the generator of the one sweeping thread (solver.rs:90-119),
    // advanced to the stream position; its draws follow the serial order of
    // stores, so the blocks run one after another
    LaneRng rng(seed, lanes);
    if (elem == DT_U8) {
        float u[16];
        for (uint64_t k = 0; k < stream_pos; ++k) rng.next(u);
        threads = 1;
    }
    // A block listed twice would be updated twice by concurrent threads in
    // the reference (a race); every listed block is swept once per phase.
    std::vector<std::vector<int64_t>> buckets(8);
    std::vector<int64_t> seen(active, active + n_active);
    std::sort(seen.begin(), seen.end());
    std::vector<char> taken(seen.size(), 0);
    for (int64_t k = 0; k < n_active; ++k) {
        int64_t bid = active[k];
        size_t pos = std::lower_bound(seen.begin(), seen.end(), bid) - seen.begin();
        if (taken[pos]) continue;
        taken[pos] = 1;
        int64_t bx = bid % g.nx, by = (bid / g.nx) % g.ny, bz = bid / g.nxy;
        buckets[(bx & 1) | ((by & 1) << 1) | ((bz & 1) << 2)].push_back(bid);
    }
    for (auto& b : buckets)
        std::stable_sort(b.begin(), b.end(), [&](int64_t a, int64_t c) {
            return morton3(a % g.nx, (a / g.nx) % g.ny, a / g.nxy) <
                   morton3(c % g.nx, (c / g.nx) % g.ny, c / g.nxy);
        });
    Grid gc;
    if (coarse) gc = to_grid(coarse);
    for (int it = 0; it < iterations; ++it)
        for (int color = 0; color < 8; ++color) {
            const auto& bk = buckets[color];
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(dynamic, 1)
            for (int64_t k = 0; k < (int64_t)bk.size(); ++k) {
                int64_t bid = bk[k];
                int32_t s = g.table[bid];
                if (s < 0) continue;  // dummy or absent: solver.rs:196-199
                std::vector<float> halo((size_t)HSX * HSX * HSX, 0.0f), out(N);
                if (coarse)
                    fill_multires(g, gc, levels, bid, HALO, FULL, BC_NEUMANN, halo.data());
                else
                    halo_fill(g, dm, bid, HALO, FULL, BC_NEUMANN, halo.data());
                if (stencil == 0) kernel_laplacian(halo.data(), bsx, dt, clamp01 != 0, out.data());
                else if (stencil == 1) kernel_meancurv(halo.data(), bsx, dt, clamp01 != 0, out.data());
                else kernel_bilaplacian(halo.data(), bsx, dt, clamp01 != 0, out.data());
                float* dstf = g.data + (size_t)s * N;
                float u[16];
                for (size_t i = 0; i < N; ++i) {
                    if (elem == DT_U8) {
                        if (i % (size_t)lanes == 0) {  // one draw per chunk of `lanes`
                            rng.next(u);
                            ++stream_pos;
                        }
                        uint8_t q = density8_store_sr(out[i], u[i % (size_t)lanes]);
                        ((uint8_t*)raw)[(size_t)s * N + i] = q;
                        dstf[i] = density8_to_f32(q);
                        continue;
                    }
                    if (elem == DT_F32) {
                        dstf[i] = out[i];
                    } else if (elem == DT_F16) {
                        uint16_t q = f32_to_f16_rn(out[i]);
                        ((uint16_t*)raw)[(size_t)s * N + i] = q;
                        dstf[i] = f16_to_f32(q);
                    } else if (elem == DT_U16) {
                        uint16_t q = f32_to_density(out[i]);
                        ((uint16_t*)raw)[(size_t)s * N + i] = q;
                        dstf[i] = density_to_f32(q);
                    } else {
                        uint16_t q = f32_to_bf16_rn(out[i]);
                        ((uint16_t*)raw)[(size_t)s * N + i] = q;
                        dstf[i] = bf16_to_f32(q);
                    }
                }
            }
        }
    return stream_pos;
}

void or_sweep(const OracleGrid* og, void* raw, int elem, const int64_t* active, int64_t n_active,
              int stencil, float dt, int iterations, int clamp01, int threads) {
    sweep_impl(og, raw, elem, active, n_active, stencil, dt, iterations, clamp01, threads, nullptr, nullptr);
}

// Sweeper::sweep on Density8 storage with an explicit generator (seed, SIMD
// lane count, draws already taken); returns the draws taken afterwards.
uint64_t or_sweep_stochastic(const OracleGrid* og, uint8_t* raw, const int64_t* active, int64_t n_active,
                             int stencil, float dt, int iterations, int clamp01, uint32_t seed, int lanes,
                             uint64_t stream_pos) {
    return sweep_impl(og, raw, DT_U8, active, n_active, stencil, dt, iterations, clamp01, 1, nullptr, nullptr,
                      seed, lanes, stream_pos);
}

// Element conversions, exported for the tests: binary16 both ways, the
// Density8 write-back and the lane generator's first draws.
void or_f32_to_f16(const float* x, int64_t n, uint16_t* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = f32_to_f16_rn(x[i]);
}
void or_f16_to_f32(const uint16_t* x, int64_t n, float* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = f16_to_f32(x[i]);
}
void or_density8_store_sr(const float* v, const float* u, int64_t n, uint8_t* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = density8_store_sr(v[i], u[i]);
}
void or_lane_rng(uint32_t seed, int lanes, int64_t draws, float* out) {
    LaneRng r(seed, lanes);
    for (int64_t k = 0; k < draws; ++k) r.next(out + k * lanes);
}

void or_sweep_multires(const OracleGrid* fine, float* data, const OracleGrid* coarse,
                       const uint8_t* levels, const int64_t* active, int64_t n_active, int stencil,
                       float dt, int iterations, int clamp01, int threads) {
    sweep_impl(fine, data, DT_F32, active, n_active, stencil, dt, iterations, clamp01, threads, coarse, levels);
}

int or_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// multires/sort.rs:35-57 sort_block_list_morton (stable; the reference's
// unstable sort has distinct keys for distinct blocks, so the order agrees).
void or_sort_block_list_morton(int64_t* blocks, int64_t n, int64_t nx, int64_t ny,
                               const uint8_t* levels, int n_levels) {
    const uint64_t ref_shift = (uint64_t)(n_levels - 1);
    const uint64_t mask = (1ULL << ref_shift) - 1;
    const uint64_t fine_bits = 3 * ref_shift;
    auto key = [&](int64_t bid) {
        uint64_t bx = bid % nx, by = (bid / nx) % ny, bz = bid / (nx * ny);
        uint64_t lvl = levels[bid];
        uint64_t coarse = morton3(bx >> ref_shift, by >> ref_shift, bz >> ref_shift);
        uint64_t priority = ref_shift - lvl;
        uint64_t fine = morton3(bx & mask, by & mask, bz & mask);
        return (coarse << (fine_bits + ref_shift)) | (priority << fine_bits) | fine;
    };
    std::stable_sort(blocks, blocks + n, [&](int64_t a, int64_t b) { return key(a) < key(b); });
}

// particles/sort.rs:455-490 bucket_by_block_dense (the stable counting sort the
// sparse bucket is tested against), generalised to 64-bit block ids with a
// stable sort.  Returns the number of distinct blocks.
int64_t or_bucket_indices(const uint64_t* bids, int64_t n, uint64_t* particle_blocks,
                          uint64_t* starts, uint32_t* perm) {
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return bids[a] < bids[b]; });
    int64_t nb = 0;
    for (int64_t i = 0; i < n; ++i) {
        perm[i] = idx[i];
        if (i == 0 || bids[idx[i]] != bids[idx[i - 1]]) {
            starts[nb] = (uint64_t)i;
            particle_blocks[nb++] = bids[idx[i]];
        }
    }
    starts[nb] = (uint64_t)n;
    return nb;
}

// Per-particle Morton sort: key = morton3 of the truncated cell coordinate,
// stable sort of (key, index).  The CPU reference order for the GPU radix sort.
void or_morton_sort(const float* pos, int64_t n, uint64_t* keys_out, uint32_t* perm) {
    std::vector<uint64_t> keys(n);
    for (int64_t i = 0; i < n; ++i)
        keys[i] = morton3((uint64_t)(int64_t)pos[3 * i], (uint64_t)(int64_t)pos[3 * i + 1],
                          (uint64_t)(int64_t)pos[3 * i + 2]);
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
    for (int64_t i = 0; i < n; ++i) { perm[i] = idx[i]; keys_out[i] = keys[idx[i]]; }
}

// particles/mod.rs:207-212 footprint_axis
static inline void footprint_axis(float p, float r_scan_bsx, int bsx, int64_t n, int32_t* lo, int32_t* hi) {
    float b = p / (float)bsx;
    int32_t l = (int32_t)truncf(b - r_scan_bsx);
    int32_t h = (int32_t)truncf(b + r_scan_bsx);
    *lo = std::max(l, 0);
    *hi = std::min<int32_t>(h, (int32_t)n - 1);
}

// fluid/p2g.rs:104-136 active_blocks (reach r_p + 1); writes sorted unique
// bids, returns the count (out may be NULL to query the count).
int64_t or_active_blocks(const float* pos, int64_t n, int64_t sx, int64_t sy, int64_t sz, int bsx,
                         float r_p, int64_t* out) {
    int64_t nx = (sx + bsx - 1) / bsx, ny = (sy + bsx - 1) / bsx, nz = (sz + bsx - 1) / bsx;
    std::vector<uint8_t> mark((size_t)(nx * ny * nz), 0);
    float rs = (r_p + 1.0f) / (float)bsx;
    for (int64_t i = 0; i < n; ++i) {
        int32_t x1, x2, y1, y2, z1, z2;
        footprint_axis(pos[3 * i], rs, bsx, nx, &x1, &x2);
        footprint_axis(pos[3 * i + 1], rs, bsx, ny, &y1, &y2);
        footprint_axis(pos[3 * i + 2], rs, bsx, nz, &z1, &z2);
        for (int32_t bz = z1; bz <= z2; ++bz)
            for (int32_t by = y1; by <= y2; ++by)
                for (int32_t bx = x1; bx <= x2; ++bx) mark[bx + by * nx + bz * nx * ny] = 1;
    }
    int64_t c = 0;
    for (int64_t b = 0; b < nx * ny * nz; ++b)
        if (mark[b]) { if (out) out[c] = b; ++c; }
    return c;
}

// fluid/p2g.rs:141-164 particles_to_grid with the staged splat of
// p2g.rs:169-412, serial in colour order (race-free, so equal to the parallel
// reference), particles of a block in stable bucket order.  Output channels
// are [mass_x, mass_y, mass_z, vel_x, vel_y, vel_z], each [n_active][bsx^3]
// over `active` (from or_active_blocks).  `normalize` applies
// MacGrid::normalize_velocity (mac.rs:106-132).
}  // extern "C"

template <class Acc>
static void p2g_impl(const float* pos, const float* vel, const float* mass, int64_t n, int64_t sx, int64_t sy,
                     int64_t sz, int bsx, float r_p, const int64_t* active, int64_t n_active, int normalize,
                     Acc* out, int threads) {
    const int lg = ilog2(bsx);
    const int64_t nx = (sx + bsx - 1) / bsx, ny = (sy + bsx - 1) / bsx, nz = (sz + bsx - 1) / bsx;
    const int64_t nxy = nx * ny;
    const size_t N = (size_t)bsx * bsx * bsx;
    std::vector<int64_t> slot((size_t)(nxy * nz), -1);
    for (int64_t k = 0; k < n_active; ++k) slot[active[k]] = k;
    std::fill(out, out + 6 * (size_t)n_active * N, (Acc)0);
    // bids (p2g.rs:149-157): `p as usize` saturates negatives to 0.
    std::vector<uint64_t> bids(n);
    for (int64_t i = 0; i < n; ++i) {
        uint64_t ix = pos[3 * i] > 0 ? (uint64_t)pos[3 * i] : 0, iy = pos[3 * i + 1] > 0 ? (uint64_t)pos[3 * i + 1] : 0,
                 iz = pos[3 * i + 2] > 0 ? (uint64_t)pos[3 * i + 2] : 0;
        bids[i] = (ix >> lg) + (iy >> lg) * nx + (iz >> lg) * nxy;
    }
    std::vector<uint64_t> pb(n + 1), st(n + 2);
    std::vector<uint32_t> perm(n);
    int64_t nb = n ? or_bucket_indices(bids.data(), n, pb.data(), st.data(), perm.data()) : 0;
    const int m = (int)ceilf(r_p);
    const float inv_r2 = 1.0f / (r_p * r_p);
    const int W = bsx + 2 * m;  // staging extent
    for (int a = 0; a < 3; ++a) {
        const float ofx = a == 0 ? 1.0f : 0.5f, ofy = a == 1 ? 1.0f : 0.5f, ofz = a == 2 ? 1.0f : 0.5f;
        Acc* mass_out = out + (size_t)a * n_active * N;
        Acc* mom_out = out + (size_t)(3 + a) * n_active * N;
        for (int color = 0; color < 8; ++color) {
            // Blocks of one colour commit to disjoint regions (p2g.rs:186-216):
            // the parallel loop is race-free, as in the reference.
            std::vector<int64_t> col;
            for (int64_t bi = 0; bi < nb; ++bi) {
                int64_t bid = (int64_t)pb[bi];
                int64_t bx = bid % nx, by = (bid / nx) % ny, bz = bid / nxy;
                if (((bx & 1) | ((by & 1) << 1) | ((bz & 1) << 2)) == color) col.push_back(bi);
            }
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
            {
            std::vector<Acc> sm((size_t)W * W * W), sv((size_t)W * W * W);
#pragma omp for schedule(dynamic, 1)
            for (int64_t ci = 0; ci < (int64_t)col.size(); ++ci) {
                const int64_t bi = col[ci];
                int64_t bid = (int64_t)pb[bi];
                int64_t bx = bid % nx, by = (bid / nx) % ny, bz = bid / nxy;
                std::fill(sm.begin(), sm.end(), (Acc)0);
                std::fill(sv.begin(), sv.end(), (Acc)0);
                const int32_t b0x = (int32_t)(bx * bsx), b0y = (int32_t)(by * bsx), b0z = (int32_t)(bz * bsx);
                const int32_t x0s = b0x - m, y0s = b0y - m, z0s = b0z - m;
                const int32_t whi = bsx + m - 1;
                for (uint64_t k = st[bi]; k < st[bi + 1]; ++k) {
                    uint32_t pi = perm[k];
                    const float* p = pos + 3 * (size_t)pi;
                    float m_p = mass[pi], u_a = vel[3 * (size_t)pi + a];
                    float scale_mass = m_p, scale_mom = m_p * u_a;
                    float px0 = p[0] - 0.5f, py0 = p[1] - 0.5f, pz0 = p[2] - 0.5f;
                    int32_t ix1 = std::min(std::max((int32_t)ceilf((p[0] - r_p) - ofx), b0x - m), b0x + whi);
                    int32_t ix2 = std::min(std::max((int32_t)floorf((p[0] + r_p) - ofx), b0x - m), b0x + whi);
                    int32_t iy1 = std::min(std::max((int32_t)ceilf((p[1] - r_p) - ofy), b0y - m), b0y + whi);
                    int32_t iy2 = std::min(std::max((int32_t)floorf((p[1] + r_p) - ofy), b0y - m), b0y + whi);
                    int32_t iz1 = std::min(std::max((int32_t)ceilf((p[2] - r_p) - ofz), b0z - m), b0z + whi);
                    int32_t iz2 = std::min(std::max((int32_t)floorf((p[2] + r_p) - ofz), b0z - m), b0z + whi);
                    for (int32_t iz = iz1; iz <= iz2; ++iz) {
                        float dz = (float)iz - pz0;
                        float dz2 = dz * dz;
                        for (int32_t iy = iy1; iy <= iy2; ++iy) {
                            float dy = (float)iy - py0;
                            float dyz = dz2 + dy * dy;
                            size_t row = ((size_t)(iz - z0s) * W + (size_t)(iy - y0s)) * W;
                            for (int32_t ix = ix1; ix <= ix2; ++ix) {
                                float dx = (float)ix - px0;
                                float dist_sq = dx * dx + dyz;
                                float d_a = a == 0 ? dx : (a == 1 ? dy : dz);
                                float df2 = (dist_sq + d_a) + 0.25f;
                                float w = fmaxf(1.0f - df2 * inv_r2, 0.0f);
                                w = (w * w) * w;
                                sm[row + (ix - x0s)] += (Acc)(w * scale_mass);
                                sv[row + (ix - x0s)] += (Acc)(w * scale_mom);
                            }
                        }
                    }
                }
                // 27-region commit (p2g.rs:339-411)
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            auto rr = [&](int d, int& lo, int& hi) {
                                if (d == -1) { lo = 0; hi = m; }
                                else if (d == 0) { lo = m; hi = m + bsx; }
                                else { lo = m + bsx; hi = 2 * m + bsx; }
                            };
                            int xlo, xhi, ylo, yhi, zlo, zhi;
                            rr(dx, xlo, xhi); rr(dy, ylo, yhi); rr(dz, zlo, zhi);
                            int32_t gx0 = b0x + xlo - m, gy0 = b0y + ylo - m, gz0 = b0z + zlo - m;
                            if (gx0 < 0 || gy0 < 0 || gz0 < 0) continue;
                            if (gx0 + (xhi - xlo) > sx || gy0 + (yhi - ylo) > sy || gz0 + (zhi - zlo) > sz) continue;
                            int64_t nbx = std::min<int64_t>(std::max<int64_t>(bx + dx, 0), nx - 1);
                            int64_t nby = std::min<int64_t>(std::max<int64_t>(by + dy, 0), ny - 1);
                            int64_t nbz = std::min<int64_t>(std::max<int64_t>(bz + dz, 0), nz - 1);
                            int64_t s = slot[nbx + nby * nx + nbz * nxy];
                            if (s < 0) continue;
                            int lx0 = gx0 & (bsx - 1), ly0 = gy0 & (bsx - 1), lz0 = gz0 & (bsx - 1);
                            for (int szz = zlo; szz < zhi; ++szz)
                                for (int syy = ylo; syy < yhi; ++syy)
                                    for (int sxx = xlo; sxx < xhi; ++sxx) {
                                        size_t si = ((size_t)szz * W + syy) * W + sxx;
                                        size_t di = (size_t)(lx0 + (sxx - xlo)) | ((size_t)(ly0 + (syy - ylo)) << lg) |
                                                    ((size_t)(lz0 + (szz - zlo)) << (2 * lg));
                                        mass_out[(size_t)s * N + di] += sm[si];
                                        mom_out[(size_t)s * N + di] += sv[si];
                                    }
                        }
            }
            }
        }
        if (normalize) {
            for (size_t i = 0; i < (size_t)n_active * N; ++i) {
                Acc mm = mass_out[i];
                mom_out[i] = mm > (Acc)0 ? mom_out[i] / mm : (Acc)0;
            }
        }
    }
}

extern "C" {

void or_p2g(const float* pos, const float* vel, const float* mass, int64_t n, int64_t sx, int64_t sy,
            int64_t sz, int bsx, float r_p, const int64_t* active, int64_t n_active, int normalize,
            float* out, int threads) {
    p2g_impl<float>(pos, vel, mass, n, sx, sy, sz, bsx, r_p, active, n_active, normalize, out, threads);
}

// The same f32 per-particle terms as or_p2g, accumulated in FP64 (no
// normalisation): the correctly rounded reference sums.
void or_p2g_terms_f64(const float* pos, const float* vel, const float* mass, int64_t n, int64_t sx, int64_t sy,
                      int64_t sz, int bsx, float r_p, const int64_t* active, int64_t n_active, double* out,
                      int threads) {
    p2g_impl<double>(pos, vel, mass, n, sx, sy, sz, bsx, r_p, active, n_active, 0, out, threads);
}

// The exact Eq. 6 splat (the naive reference of p2g.rs:443-536) accumulated
// in FP64: the error yardstick for the FP32 splats.  Also returns, per face,
// the sum of |w*m| and |w*m*u| (the normalisers for relative error).
void or_p2g_f64(const float* pos, const float* vel, const float* mass, int64_t n, int64_t sx, int64_t sy,
                int64_t sz, int bsx, float r_p, const int64_t* active, int64_t n_active, double* out,
                double* abs_out) {
    const int lg = ilog2(bsx);
    const int64_t nx = (sx + bsx - 1) / bsx, ny = (sy + bsx - 1) / bsx;
    const size_t N = (size_t)bsx * bsx * bsx;
    std::vector<int64_t> slot((size_t)(nx * ny * ((sz + bsx - 1) / bsx)), -1);
    for (int64_t k = 0; k < n_active; ++k) slot[active[k]] = k;
    std::fill(out, out + 6 * (size_t)n_active * N, 0.0);
    std::fill(abs_out, abs_out + 6 * (size_t)n_active * N, 0.0);
    const float inv_r2 = 1.0f / (r_p * r_p);
    for (int64_t pi = 0; pi < n; ++pi) {
        const float* p = pos + 3 * pi;
        for (int a = 0; a < 3; ++a) {
            const float ofx = a == 0 ? 1.0f : 0.5f, ofy = a == 1 ? 1.0f : 0.5f, ofz = a == 2 ? 1.0f : 0.5f;
            int32_t ix1 = std::max((int32_t)ceilf((p[0] - r_p) - ofx), 0), ix2 = std::min((int32_t)floorf((p[0] + r_p) - ofx), (int32_t)sx - 1);
            int32_t iy1 = std::max((int32_t)ceilf((p[1] - r_p) - ofy), 0), iy2 = std::min((int32_t)floorf((p[1] + r_p) - ofy), (int32_t)sy - 1);
            int32_t iz1 = std::max((int32_t)ceilf((p[2] - r_p) - ofz), 0), iz2 = std::min((int32_t)floorf((p[2] + r_p) - ofz), (int32_t)sz - 1);
            for (int32_t k = iz1; k <= iz2; ++k)
                for (int32_t j = iy1; j <= iy2; ++j)
                    for (int32_t i = ix1; i <= ix2; ++i) {
                        double fx = i + 0.5 + (a == 0 ? 0.5 : 0.0), fy = j + 0.5 + (a == 1 ? 0.5 : 0.0),
                               fz = k + 0.5 + (a == 2 ? 0.5 : 0.0);
                        double dx = fx - p[0], dy = fy - p[1], dz = fz - p[2];
                        double d2 = dx * dx + dy * dy + dz * dz;
                        double w = 1.0 - d2 * (double)inv_r2;
                        if (w <= 0.0) continue;
                        w = w * w * w;
                        int64_t bid = (i >> lg) + (int64_t)(j >> lg) * nx + (int64_t)(k >> lg) * nx * ny;
                        int64_t s = slot[bid];
                        if (s < 0) continue;
                        size_t vid = (size_t)(i & (bsx - 1)) | ((size_t)(j & (bsx - 1)) << lg) | ((size_t)(k & (bsx - 1)) << (2 * lg));
                        double wm = w * mass[pi], wmu = w * mass[pi] * vel[3 * pi + a];
                        out[(size_t)a * n_active * N + s * N + vid] += wm;
                        out[(size_t)(3 + a) * n_active * N + s * N + vid] += wmu;
                        abs_out[(size_t)a * n_active * N + s * N + vid] += fabs(wm);
                        abs_out[(size_t)(3 + a) * n_active * N + s * N + vid] += fabs(wmu);
                    }
        }
    }
}

// math/gather.rs:54-158 gather_map (dmax = 1) + sample.rs:203-211
// trilinear_value over a grid view; used by or_mac_sample.
static float sample_linear(const Grid& g, const Dummies& dm, float x, float y, float z, int bc) {
    const int bsx = g.bsx, lg = ilog2(bsx), mask = bsx - 1;
    float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    int32_t ix0 = (int32_t)fx, iy0 = (int32_t)fy, iz0 = (int32_t)fz;
    float c[8];
    bool fast = false;
    if (ix0 >= 0 && iy0 >= 0 && iz0 >= 0 && (ix0 + 1) < g.sx && (iy0 + 1) < g.sy && (iz0 + 1) < g.sz) {
        int vx0 = ix0 & mask, vy0 = iy0 & mask, vz0 = iz0 & mask;
        if (vx0 + 1 < bsx && vy0 + 1 < bsx && vz0 + 1 < bsx) {
            int64_t bid = (ix0 >> lg) + (int64_t)(iy0 >> lg) * g.nx + (int64_t)(iz0 >> lg) * g.nxy;
            const float* p = block_data_ptr(g, dm, bid);
            int s = 0;
            for (int k = 0; k < 2; ++k)
                for (int j = 0; j < 2; ++j)
                    for (int i = 0; i < 2; ++i)
                        c[s++] = p[(vx0 + i) | ((vy0 + j) << lg) | ((vz0 + k) << (2 * lg))];
            fast = true;
        }
    }
    if (!fast) {
        int64_t bx0 = std::min<int64_t>(std::max<int64_t>(ix0 >> lg, 0), g.nx - 1);
        int64_t by0 = std::min<int64_t>(std::max<int64_t>(iy0 >> lg, 0), g.ny - 1);
        int64_t bz0 = std::min<int64_t>(std::max<int64_t>(iz0 >> lg, 0), g.nz - 1);
        const float* slots[8];
        for (int sz_ = 0; sz_ < 2; ++sz_)
            for (int sy_ = 0; sy_ < 2; ++sy_)
                for (int sx_ = 0; sx_ < 2; ++sx_) {
                    int64_t bxx = std::min<int64_t>(bx0 + sx_, g.nx - 1), byy = std::min<int64_t>(by0 + sy_, g.ny - 1),
                            bzz = std::min<int64_t>(bz0 + sz_, g.nz - 1);
                    slots[sx_ | (sy_ << 1) | (sz_ << 2)] = block_data_ptr(g, dm, bxx + byy * g.nx + bzz * g.nxy);
                }
        int s = 0;
        for (int k = 0; k < 2; ++k) {
            int32_t rz; bool okz = resolve_axis(iz0 + k, (int32_t)g.sz - 1, bc, &rz);
            for (int j = 0; j < 2; ++j) {
                int32_t ry; bool oky = resolve_axis(iy0 + j, (int32_t)g.sy - 1, bc, &ry);
                for (int i = 0; i < 2; ++i) {
                    int32_t rx; bool okx = resolve_axis(ix0 + i, (int32_t)g.sx - 1, bc, &rx);
                    if (okx && oky && okz) {
                        // slot offsets mod 2 (see gather_window)
                        int sl = (int)((((rx >> lg) - bx0) & 1) | ((((ry >> lg) - by0) & 1) << 1) | ((((rz >> lg) - bz0) & 1) << 2));
                        c[s] = slots[sl][(rx & mask) | ((ry & mask) << lg) | ((rz & mask) << (2 * lg))];
                    } else {
                        c[s] = g.empty_value;
                    }
                    ++s;
                }
            }
        }
    }
    float u = x - fx, v = y - fy, w = z - fz;
    auto lerp = [](float a, float b, float t) { return fmaf(b - a, t, a); };
    float c00 = lerp(c[0], c[1], u), c10 = lerp(c[2], c[3], u), c01 = lerp(c[4], c[5], u), c11 = lerp(c[6], c[7], u);
    float c0 = lerp(c00, c10, v), c1 = lerp(c01, c11, v);
    return lerp(c0, c1, w);
}

// math/gather.rs:54-158 gather_map for a window of span = dmax + 1 (2 or 4)
// anchored at (ix0, iy0, iz0): the one-block fast path, else 2x2x2 block
// slots from the clamped anchor block and per-axis boundary resolution.
static void gather_window(const Grid& g, const Dummies& dm, int32_t ix0, int32_t iy0, int32_t iz0, int bc, int span,
                          float* out) {
    const int bsx = g.bsx, lg = ilog2(bsx), mask = bsx - 1, dmax = span - 1;
    if (ix0 >= 0 && iy0 >= 0 && iz0 >= 0 && (int64_t)ix0 + dmax < (int64_t)g.sx && (int64_t)iy0 + dmax < (int64_t)g.sy &&
        (int64_t)iz0 + dmax < (int64_t)g.sz) {
        int vx0 = ix0 & mask, vy0 = iy0 & mask, vz0 = iz0 & mask;
        if (vx0 + dmax < bsx && vy0 + dmax < bsx && vz0 + dmax < bsx) {
            int64_t bid = (ix0 >> lg) + (int64_t)(iy0 >> lg) * g.nx + (int64_t)(iz0 >> lg) * g.nxy;
            const float* p = block_data_ptr(g, dm, bid);
            int s = 0;
            for (int k = 0; k < span; ++k)
                for (int j = 0; j < span; ++j)
                    for (int i = 0; i < span; ++i) out[s++] = p[(vx0 + i) | ((vy0 + j) << lg) | ((vz0 + k) << (2 * lg))];
            return;
        }
    }
    int64_t bx0 = std::min<int64_t>(std::max<int64_t>(ix0 >> lg, 0), g.nx - 1);
    int64_t by0 = std::min<int64_t>(std::max<int64_t>(iy0 >> lg, 0), g.ny - 1);
    int64_t bz0 = std::min<int64_t>(std::max<int64_t>(iz0 >> lg, 0), g.nz - 1);
    const float* slots[8];
    for (int sz_ = 0; sz_ < 2; ++sz_)
        for (int sy_ = 0; sy_ < 2; ++sy_)
            for (int sx_ = 0; sx_ < 2; ++sx_) {
                int64_t bxx = std::min<int64_t>(bx0 + sx_, g.nx - 1), byy = std::min<int64_t>(by0 + sy_, g.ny - 1),
                        bzz = std::min<int64_t>(bz0 + sz_, g.nz - 1);
                slots[sx_ | (sy_ << 1) | (sz_ << 2)] = block_data_ptr(g, dm, bxx + byy * g.nx + bzz * g.nxy);
            }
    int s = 0;
    for (int k = 0; k < span; ++k) {
        int32_t rz; bool okz = resolve_axis(iz0 + k, (int32_t)g.sz - 1, bc, &rz);
        for (int j = 0; j < span; ++j) {
            int32_t ry; bool oky = resolve_axis(iy0 + j, (int32_t)g.sy - 1, bc, &ry);
            for (int i = 0; i < span; ++i) {
                int32_t rx; bool okx = resolve_axis(ix0 + i, (int32_t)g.sx - 1, bc, &rx);
                if (okx && oky && okz) {
                    // A Neumann window far outside the domain can reflect to
                    // a block before the anchor block, where the crate's slot
                    // index leaves the 2x2x2 slots (undefined there); the
                    // offsets are taken mod 2, as on the device.
                    int sl = (int)((((rx >> lg) - bx0) & 1) | ((((ry >> lg) - by0) & 1) << 1) | ((((rz >> lg) - bz0) & 1) << 2));
                    out[s] = slots[sl][(rx & mask) | ((ry & mask) << lg) | ((rz & mask) << (2 * lg))];
                } else {
                    out[s] = g.empty_value;
                }
                ++s;
            }
        }
    }
}

// math/bspline.rs:4-32 uniform cubic B-spline weights and their first and
// second derivatives (f32, left to right, no contraction).
static void cubic_w(float t, float w[4]) {
    const float m = 1.0f - t, s6 = 1.0f / 6.0f, t3 = 2.0f / 3.0f;
    w[0] = ((s6 * m) * m) * m;
    w[1] = t3 - ((0.5f * t) * t) * (2.0f - t);
    w[2] = t3 - ((0.5f * m) * m) * (1.0f + t);
    w[3] = ((s6 * t) * t) * t;
}
static void cubic_dw(float t, float w[4]) {
    const float m = 1.0f - t;
    w[0] = ((-m) * m) / 2.0f;
    w[1] = (0.5f * t) * t - (2.0f - t) * t;
    w[2] = m * (t + 1.0f) - (0.5f * m) * m;
    w[3] = (t * t) / 2.0f;
}
static void cubic_d2w(float t, float w[4]) {
    w[0] = 1.0f - t;
    w[1] = 3.0f * t - 2.0f;
    w[2] = 1.0f - 3.0f * t;
    w[3] = t;
}
// (f * w).reduce_sum() of a row of 4 (ordered lane sum)
static inline float row_dot(const float* f, const float w[4]) {
    return ((f[0] * w[0] + f[1] * w[1]) + f[2] * w[2]) + f[3] * w[3];
}

// sample.rs:493-649 Sample for SparseGrid, cubic B-spline (cell-centred
// regardless of alignment; window base floor(x - 0.5) - 1, t = frac) and the
// trilinear gradient (sample.rs:215-237).  mode 0: cubic value -> out[n];
// 1: cubic gradient -> out[n][3]; 2: Hessian (fxx, fyy, fzz, fxy, fxz, fyz) ->
// out[n][6]; 3: trilinear gradient at the given alignment -> out[n][3].
void or_sample_ext(const OracleGrid* og, const float* pos, int64_t n, int mode, int align, int bc, float* out) {
    Grid g = to_grid(og);
    Dummies dm(g);
    for (int64_t i = 0; i < n; ++i) {
        float x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        if (mode == 3) {
            if (align == 1) { x = x - 0.5f; y = y - 0.5f; z = z - 0.5f; }
            const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
            float c[8];
            gather_window(g, dm, (int32_t)fx, (int32_t)fy, (int32_t)fz, bc, 2, c);
            const float u = x - fx, v = y - fy, w = z - fz;
            const float f01234567 = ((((((c[7] - c[6]) - c[5]) + c[4]) - c[3]) + c[2]) + c[1]) - c[0];
            const float f01234567u = f01234567 * u;
            const float f01234567uf6420 = (((f01234567u + c[6]) - c[4]) - c[2]) + c[0];
            const float f5410 = ((c[5] - c[4]) - c[1]) + c[0];
            const float f3210 = ((c[3] - c[2]) - c[1]) + c[0];
            out[3 * i] = fmaf(f01234567 * v + f5410, w, ((f3210 * v + c[1]) - c[0]));
            out[3 * i + 1] = fmaf(f01234567uf6420, w, ((f3210 * u + c[2]) - c[0]));
            out[3 * i + 2] = fmaf(f01234567uf6420, v, ((f5410 * u + c[4]) - c[0]));
            continue;
        }
        x = x - 0.5f; y = y - 0.5f; z = z - 0.5f;
        const float xf = floorf(x), yf = floorf(y), zf = floorf(z);
        const float tx = x - xf, ty = y - yf, tz = z - zf;
        float win[64];
        gather_window(g, dm, (int32_t)xf - 1, (int32_t)yf - 1, (int32_t)zf - 1, bc, 4, win);
        float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4], ddx[4], ddy[4], ddz[4];
        cubic_w(tx, wx); cubic_w(ty, wy); cubic_w(tz, wz);
        cubic_dw(tx, dx); cubic_dw(ty, dy); cubic_dw(tz, dz);
        cubic_d2w(tx, ddx); cubic_d2w(ty, ddy); cubic_d2w(tz, ddz);
        float val = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
        float fxx = 0.0f, fyy = 0.0f, fzz = 0.0f, fxy = 0.0f, fxz = 0.0f, fyz = 0.0f;
        for (int k = 0; k < 4; ++k)
            for (int j = 0; j < 4; ++j) {
                const float* f = win + 16 * k + 4 * j;
                const float sx = row_dot(f, wx);
                if (mode == 0) {
                    val = fmaf(sx, wy[j] * wz[k], val);
                } else if (mode == 1) {
                    const float sxp = row_dot(f, dx);
                    const float wyz = wy[j] * wz[k];
                    val = fmaf(sx, wyz, val);
                    gx = fmaf(sxp, wyz, gx);
                    gy = fmaf(sx, dy[j] * wz[k], gy);
                    gz = fmaf(sx, wy[j] * dz[k], gz);
                } else {
                    const float sxp = row_dot(f, dx), sxpp = row_dot(f, ddx);
                    const float wyz = wy[j] * wz[k], wpyz = dy[j] * wz[k], wypz = wy[j] * dz[k];
                    const float wppyz = ddy[j] * wz[k], wyppz = wy[j] * ddz[k], wpyzp = dy[j] * dz[k];
                    fxx = fmaf(sxpp, wyz, fxx);
                    fyy = fmaf(sx, wppyz, fyy);
                    fzz = fmaf(sx, wyppz, fzz);
                    fxy = fmaf(sxp, wpyz, fxy);
                    fxz = fmaf(sxp, wypz, fxz);
                    fyz = fmaf(sx, wpyzp, fyz);
                }
            }
        if (mode == 0) out[i] = val;
        else if (mode == 1) { out[3 * i] = gx; out[3 * i + 1] = gy; out[3 * i + 2] = gz; }
        else {
            float* h = out + 6 * i;
            h[0] = fxx; h[1] = fyy; h[2] = fzz; h[3] = fxy; h[4] = fxz; h[5] = fyz;
        }
    }
}

// Scalar trilinear Sampler::sample::<Linear> (sample.rs:494-512) with the
// given alignment (0 Corner, 1 CellCentered).
void or_sample_linear(const OracleGrid* og, const float* pos, int64_t n, int align, int bc, float* out) {
    Grid g = to_grid(og);
    Dummies dm(g);
    for (int64_t i = 0; i < n; ++i) {
        float x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        if (align == 1) { x = x - 0.5f; y = y - 0.5f; z = z - 0.5f; }
        out[i] = sample_linear(g, dm, x, y, z, bc);
    }
}

// fluid/g2p.rs:15-32 MacSampler::sample::<Linear>: per face component a, a
// cell-centred sample at p - 1/2 e_a.  vgrids[a] views velocity[a].
void or_mac_sample(const OracleGrid* vx, const OracleGrid* vy, const OracleGrid* vz, const float* pos,
                   int64_t n, int bc, float* out) {
    const OracleGrid* v[3] = {vx, vy, vz};
    for (int a = 0; a < 3; ++a) {
        Grid g = to_grid(v[a]);
        Dummies dm(g);
#pragma omp parallel for schedule(static) if (n > 100000)
        for (int64_t i = 0; i < n; ++i) {
            float px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
            if (a == 0) px = px - 0.5f;
            if (a == 1) py = py - 0.5f;
            if (a == 2) pz = pz - 0.5f;
            out[3 * i + a] = sample_linear(g, dm, px - 0.5f, py - 0.5f, pz - 0.5f, bc);
        }
    }
}

// fluid/g2p.rs:42-45 g2p_blend (component-wise Vec3 arithmetic).
void or_g2p_blend(const float* u_old, const float* u, const float* u_tilde, int64_t n, float alpha, float* out) {
    for (int64_t i = 0; i < 3 * n; ++i) {
        float delta = u[i] - u_tilde[i];
        out[i] = (u_old[i] + delta) * alpha + u[i] * (1.0f - alpha);
    }
}

// fluid/mac.rs:137-171 divergence over `active` (get_voxel semantics: absent
// blocks read the empty value 0; the leftmost faces read 0).
void or_divergence(const OracleGrid* ux, const OracleGrid* uy, const OracleGrid* uz, const int64_t* active,
                   int64_t n_active, float* out) {
    Grid g[3] = {to_grid(ux), to_grid(uy), to_grid(uz)};
    Dummies dm(g[0]);
    const int bsx = g[0].bsx, lg = ilog2(bsx), mask = bsx - 1;
    const size_t N = (size_t)bsx * bsx * bsx;
    auto get = [&](int a, int64_t x, int64_t y, int64_t z) -> float {
        int64_t bid = (x >> lg) + (y >> lg) * g[a].nx + (z >> lg) * g[a].nxy;
        int32_t s = g[a].table[bid];
        if (s == -2) return g[a].full_value;
        if (s < 0) return g[a].empty_value;
        return g[a].data[(size_t)s * N + ((x & mask) | ((y & mask) << lg) | ((z & mask) << (2 * lg)))];
    };
    for (int64_t k = 0; k < n_active; ++k) {
        int64_t bid = active[k];
        int64_t bx = bid % g[0].nx, by = (bid / g[0].nx) % g[0].ny, bz = bid / g[0].nxy;
        int64_t gx0 = bx * bsx, gy0 = by * bsx, gz0 = bz * bsx;
        int64_t gx1 = std::min<int64_t>(gx0 + bsx, g[0].sx), gy1 = std::min<int64_t>(gy0 + bsx, g[0].sy),
                gz1 = std::min<int64_t>(gz0 + bsx, g[0].sz);
        float* dp = out + (size_t)k * N;
        size_t vid = 0;
        for (int64_t z = gz0; z < gz1; ++z)
            for (int64_t y = gy0; y < gy1; ++y)
                for (int64_t x = gx0; x < gx1; ++x) {
                    float ux1 = get(0, x, y, z), ux0 = x == 0 ? 0.0f : get(0, x - 1, y, z);
                    float vy1 = get(1, x, y, z), vy0 = y == 0 ? 0.0f : get(1, x, y - 1, z);
                    float wz1 = get(2, x, y, z), wz0 = z == 0 ? 0.0f : get(2, x, y, z - 1);
                    dp[vid++] = ((ux1 - ux0) + (vy1 - vy0)) + (wz1 - wz0);
                }
    }
}

// multires/downsample.rs:13-59 downsample_channel_avg: coarse block `k` (block
// size bsx/2) is the 2^3 mean of fine block `k`.
void or_downsample_avg(const float* fine, int64_t n_blocks, int bsx, float* coarse) {
    const int lg = ilog2(bsx), bsc = bsx / 2;
    const size_t N = (size_t)bsx * bsx * bsx, NC = (size_t)bsc * bsc * bsc;
    for (int64_t b = 0; b < n_blocks; ++b) {
        const float* sp = fine + b * N;
        float* dp = coarse + b * NC;
        size_t vid = 0;
        for (int cz = 0; cz < bsc; ++cz)
            for (int cy = 0; cy < bsc; ++cy)
                for (int cx = 0; cx < bsc; ++cx) {
                    float sum = 0.0f;
                    for (int dz = 0; dz < 2; ++dz)
                        for (int dy = 0; dy < 2; ++dy)
                            for (int dx = 0; dx < 2; ++dx)
                                sum += sp[(size_t)(2 * cx + dx) | ((size_t)(2 * cy + dy) << lg) | ((size_t)(2 * cz + dz) << (2 * lg))];
                    dp[vid++] = sum / 8.0f;
                }
    }
}

// ===========================================================================
// FP64 Poisson oracle (no reference implementation: parity unpinned).
//
// Problem: the unknowns are the cells of the active blocks (block size bs on
// an nx*ny*nz block grid); every other cell is zero (Dirichlet).  Level 0:
//   (A_0 x)_c = 6 x_c - sum of the x of its active face neighbours
// (docs/roadmap.md:618-627: matvec `y = D x - sum nb`, relaxation
// `y = w (b + sum nb) D^-1 + (1-w) x`).  Level l+1 has cells twice as wide.
// While bs_l >= 4 the block grid is kept and the block size halves ("same
// grid" levels); from bs_l == 2 on, the block grid halves and the block size
// stays 2.  A coarse cell is active when any of its 8 children is, so every
// level covers the same cells as level 0 (while coarse cells are no wider
// than a level-0 block).  At level l the operator is the 7-point stencil
// rediscretised on cells of width 2^l, in the units of the level-0 equation:
//   (A_l x)_c = s_l ((6 - g_l m_c) x_c - sum of active neighbours),
//   s_l = 0.25^l,
// where m_c counts the missing face neighbours of c and g_l places the zero
// Dirichlet value where level 0 has it, half a level-0 cell outside the
// boundary face: linear extrapolation from the cell centre, at distance
// d = (1/2 + 2^(-l-1)) cells of level l from that point, gives the ghost
// value g_l x_c with g_l = 1 - 1/d (g_0 = 0).  Prolongation P is cell-centred
// trilinear (per axis 3/4 from the parent cell and 1/4 from its neighbour on
// the child's side; inactive coarse cells count as zero) and restriction is
// R = P^T / 8, so the V-cycle with nu1 = nu2 is a symmetric preconditioner.
// Coarsening stops at <= kPoissonDirect cells, which are solved directly
// (dense Cholesky, FP64; inactive cells have identity rows).
// V-cycle: nu1 weighted-Jacobi sweeps, residual, restriction, recursion,
// prolongation-correction, nu2 sweeps.
// ===========================================================================
static const int64_t kPoissonDirect = 1024;
static double g_corr = 1.0;  // coarse-correction scale of the V-cycle

struct PLevel {
    int bs, lg;
    int64_t nx, ny, nz;
    std::vector<int64_t> bids;  // sorted active block ids
    std::vector<int64_t> nbr;   // [n][6] slot of the -x,+x,-y,+y,-z,+z neighbour block or -1
    std::vector<int64_t> parent;  // [n] slot of the parent block at level l+1
    double scale;
    double ghost = 0.0;           // g_l
    std::vector<uint8_t> mask;    // per cell: active (empty = all active)
    int64_t n() const { return (int64_t)bids.size(); }
    int64_t cells() const { return n() * bs * bs * bs; }
};

static void build_nbr(PLevel& L) {
    std::vector<int64_t> slot((size_t)(L.nx * L.ny * L.nz), -1);
    for (int64_t k = 0; k < L.n(); ++k) slot[L.bids[k]] = k;
    L.nbr.assign((size_t)L.n() * 6, -1);
    for (int64_t k = 0; k < L.n(); ++k) {
        int64_t b = L.bids[k], bx = b % L.nx, by = (b / L.nx) % L.ny, bz = b / (L.nx * L.ny);
        const int64_t d[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
        for (int f = 0; f < 6; ++f) {
            int64_t X = bx + d[f][0], Y = by + d[f][1], Z = bz + d[f][2];
            if (X < 0 || Y < 0 || Z < 0 || X >= L.nx || Y >= L.ny || Z >= L.nz) continue;
            L.nbr[k * 6 + f] = slot[X + Y * L.nx + Z * L.nx * L.ny];
        }
    }
}

// value of cell (cx,cy,cz) relative to block k, where one coordinate may be -1 or bs
static inline double cell_at(const PLevel& L, const double* x, int64_t k, int cx, int cy, int cz) {
    int64_t kk = k;
    if (cx < 0) { kk = L.nbr[k * 6 + 0]; cx += L.bs; }
    else if (cx >= L.bs) { kk = L.nbr[k * 6 + 1]; cx -= L.bs; }
    else if (cy < 0) { kk = L.nbr[k * 6 + 2]; cy += L.bs; }
    else if (cy >= L.bs) { kk = L.nbr[k * 6 + 3]; cy -= L.bs; }
    else if (cz < 0) { kk = L.nbr[k * 6 + 4]; cz += L.bs; }
    else if (cz >= L.bs) { kk = L.nbr[k * 6 + 5]; cz -= L.bs; }
    if (kk < 0) return 0.0;
    size_t N = (size_t)L.bs * L.bs * L.bs;
    return x[kk * N + ((size_t)cx | ((size_t)cy << L.lg) | ((size_t)cz << (2 * L.lg)))];
}

static inline double nbsum(const PLevel& L, const double* x, int64_t k, int cx, int cy, int cz) {
    double s = cell_at(L, x, k, cx - 1, cy, cz);
    s += cell_at(L, x, k, cx + 1, cy, cz);
    s += cell_at(L, x, k, cx, cy - 1, cz);
    s += cell_at(L, x, k, cx, cy + 1, cz);
    s += cell_at(L, x, k, cx, cy, cz - 1);
    s += cell_at(L, x, k, cx, cy, cz + 1);
    return s;
}

// 1 when the cell at (cx,cy,cz) relative to block k (one coordinate may be -1
// or bs) is an active cell
static inline int present(const PLevel& L, int64_t k, int cx, int cy, int cz) {
    int64_t kk = k;
    if (cx < 0) { kk = L.nbr[k * 6 + 0]; cx += L.bs; }
    else if (cx >= L.bs) { kk = L.nbr[k * 6 + 1]; cx -= L.bs; }
    else if (cy < 0) { kk = L.nbr[k * 6 + 2]; cy += L.bs; }
    else if (cy >= L.bs) { kk = L.nbr[k * 6 + 3]; cy -= L.bs; }
    else if (cz < 0) { kk = L.nbr[k * 6 + 4]; cz += L.bs; }
    else if (cz >= L.bs) { kk = L.nbr[k * 6 + 5]; cz -= L.bs; }
    if (kk < 0) return 0;
    if (L.mask.empty()) return 1;
    const size_t N = (size_t)L.bs * L.bs * L.bs;
    return L.mask[kk * N + ((size_t)cx | ((size_t)cy << L.lg) | ((size_t)cz << (2 * L.lg)))];
}

// 6 - g_l m_c (unscaled diagonal)
static inline double diag_of(const PLevel& L, int64_t k, int cx, int cy, int cz) {
    const int miss = 6 - present(L, k, cx - 1, cy, cz) - present(L, k, cx + 1, cy, cz) - present(L, k, cx, cy - 1, cz) -
                     present(L, k, cx, cy + 1, cz) - present(L, k, cx, cy, cz - 1) - present(L, k, cx, cy, cz + 1);
    return 6.0 - L.ghost * miss;
}

static void p_matvec(const PLevel& L, const double* x, double* y) {
    const size_t N = (size_t)L.bs * L.bs * L.bs;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < L.n(); ++k)
        for (int cz = 0; cz < L.bs; ++cz)
            for (int cy = 0; cy < L.bs; ++cy)
                for (int cx = 0; cx < L.bs; ++cx) {
                    size_t i = k * N + ((size_t)cx | ((size_t)cy << L.lg) | ((size_t)cz << (2 * L.lg)));
                    if (!L.mask.empty() && !L.mask[i]) { y[i] = 0.0; continue; }
                    y[i] = L.scale * (diag_of(L, k, cx, cy, cz) * x[i] - nbsum(L, x, k, cx, cy, cz));
                }
}

static void p_jacobi(const PLevel& L, double* x, const double* b, double omega, int sweeps, std::vector<double>& tmp) {
    const size_t N = (size_t)L.bs * L.bs * L.bs, tot = N * L.n();
    tmp.resize(tot);
    for (int s = 0; s < sweeps; ++s) {
#pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < L.n(); ++k)
            for (int cz = 0; cz < L.bs; ++cz)
                for (int cy = 0; cy < L.bs; ++cy)
                    for (int cx = 0; cx < L.bs; ++cx) {
                        size_t i = k * N + ((size_t)cx | ((size_t)cy << L.lg) | ((size_t)cz << (2 * L.lg)));
                        if (!L.mask.empty() && !L.mask[i]) { tmp[i] = 0.0; continue; }
                        double sn = nbsum(L, x, k, cx, cy, cz);
                        tmp[i] = omega * (b[i] + L.scale * sn) / (diag_of(L, k, cx, cy, cz) * L.scale) + (1.0 - omega) * x[i];
                    }
        std::copy(tmp.begin(), tmp.end(), x);
    }
}

// global cell (gx,gy,gz) -> index into the level's array, or -1
static inline int64_t cell_index(const PLevel& L, const std::vector<int64_t>& slot, int64_t gx, int64_t gy, int64_t gz) {
    int64_t bx = gx >> L.lg, by = gy >> L.lg, bz = gz >> L.lg;
    if (bx >= L.nx || by >= L.ny || bz >= L.nz) return -1;
    int64_t s = slot[bx + by * L.nx + bz * L.nx * L.ny];
    if (s < 0) return -1;
    int m = L.bs - 1;
    return s * L.bs * L.bs * L.bs + ((gx & m) | ((gy & m) << L.lg) | ((gz & m) << (2 * L.lg)));
}

struct PHier {
    std::vector<PLevel> lv;
    std::vector<std::vector<int64_t>> slot;  // per level: dense bid -> slot
    std::vector<double> chol;
    int64_t nc = 0;
};

static void build_hier(PHier& H, const int64_t* active, int64_t n_active, int64_t nx, int64_t ny, int64_t nz, int bs,
                       int max_levels) {
    H.lv.clear();
    H.slot.clear();
    PLevel L0;
    L0.bs = bs; L0.lg = ilog2(bs); L0.nx = nx; L0.ny = ny; L0.nz = nz; L0.scale = 1.0;
    L0.bids.assign(active, active + n_active);
    std::sort(L0.bids.begin(), L0.bids.end());
    L0.bids.erase(std::unique(L0.bids.begin(), L0.bids.end()), L0.bids.end());
    H.lv.push_back(L0);
    while ((int)H.lv.size() < max_levels && H.lv.back().cells() > kPoissonDirect) {
        const PLevel& F = H.lv.back();
        PLevel C;
        C.scale = F.scale * 0.25;
        if (F.bs >= 4) {
            C.bs = F.bs / 2; C.nx = F.nx; C.ny = F.ny; C.nz = F.nz;
            C.bids = F.bids;
        } else {
            C.bs = F.bs; C.nx = (F.nx + 1) / 2; C.ny = (F.ny + 1) / 2; C.nz = (F.nz + 1) / 2;
            for (int64_t b : F.bids) {
                int64_t bx = b % F.nx, by = (b / F.nx) % F.ny, bz = b / (F.nx * F.ny);
                C.bids.push_back((bx >> 1) + (by >> 1) * C.nx + (bz >> 1) * C.nx * C.ny);
            }
            std::sort(C.bids.begin(), C.bids.end());
            C.bids.erase(std::unique(C.bids.begin(), C.bids.end()), C.bids.end());
        }
        C.lg = ilog2(C.bs);
        const double d = 0.5 + std::ldexp(1.0, -(int)H.lv.size() - 1);
        C.ghost = 1.0 - 1.0 / d;
        H.lv.push_back(C);
    }
    for (auto& L : H.lv) {
        build_nbr(L);
        std::vector<int64_t> sl((size_t)(L.nx * L.ny * L.nz), -1);
        for (int64_t k = 0; k < L.n(); ++k) sl[L.bids[k]] = k;
        H.slot.push_back(sl);
    }
    // cell masks: a coarse cell is active when any of its 8 children is
    for (size_t l = 1; l < H.lv.size(); ++l) {
        PLevel& C = H.lv[l];
        const PLevel& F = H.lv[l - 1];
        const size_t N = (size_t)C.bs * C.bs * C.bs;
        C.mask.assign(N * C.n(), 0);
        for (int64_t k = 0; k < C.n(); ++k) {
            const int64_t b = C.bids[k], bx = b % C.nx, by = (b / C.nx) % C.ny, bz = b / (C.nx * C.ny);
            for (size_t v = 0; v < N; ++v) {
                const int cx = v & (C.bs - 1), cy = (v >> C.lg) & (C.bs - 1), cz = (int)(v >> (2 * C.lg));
                const int64_t q[3] = {bx * C.bs + cx, by * C.bs + cy, bz * C.bs + cz};
                uint8_t a = 0;
                for (int c = 0; c < 8; ++c) {
                    const int64_t fi = cell_index(F, H.slot[l - 1], 2 * q[0] + (c & 1), 2 * q[1] + ((c >> 1) & 1), 2 * q[2] + (c >> 2));
                    if (fi >= 0 && (F.mask.empty() || F.mask[fi])) a = 1;
                }
                C.mask[k * N + v] = a;
            }
        }
    }
    const PLevel& C = H.lv.back();
    const int64_t n = C.cells();
    H.nc = n;
    H.chol.clear();
    if (n > 4 * kPoissonDirect) return;  // max_levels cut the hierarchy short: iterate instead
    std::vector<double> A((size_t)n * n, 0.0), e(n, 0.0), col(n);
    for (int64_t j = 0; j < n; ++j) {
        e[j] = 1.0;
        p_matvec(C, e.data(), col.data());
        for (int64_t i = 0; i < n; ++i) A[(size_t)i * n + j] = col[i];
        if (!C.mask.empty() && !C.mask[j]) A[(size_t)j * n + j] = 1.0;  // inactive cell: identity row
        e[j] = 0.0;
    }
    for (int64_t j = 0; j < n; ++j) {
        double d = A[(size_t)j * n + j];
        for (int64_t k = 0; k < j; ++k) d -= A[(size_t)j * n + k] * A[(size_t)j * n + k];
        d = std::sqrt(d);
        A[(size_t)j * n + j] = d;
        for (int64_t i = j + 1; i < n; ++i) {
            double s2 = A[(size_t)i * n + j];
            for (int64_t k = 0; k < j; ++k) s2 -= A[(size_t)i * n + k] * A[(size_t)j * n + k];
            A[(size_t)i * n + j] = s2 / d;
        }
    }
    H.chol.swap(A);
}

static void coarse_solve(const PHier& H, double* x, const double* b) {
    const int64_t n = H.nc;
    const PLevel& C = H.lv.back();
    if (H.chol.empty()) {
        std::vector<double> tmp;
        std::fill(x, x + n, 0.0);
        p_jacobi(C, x, b, 2.0 / 3.0, 400, tmp);
        return;
    }
    const double* L = H.chol.data();
    std::vector<double> y(n);
    for (int64_t i = 0; i < n; ++i) {
        double s = b[i];
        for (int64_t k = 0; k < i; ++k) s -= L[(size_t)i * n + k] * y[k];
        y[i] = s / L[(size_t)i * n + i];
    }
    for (int64_t i = n - 1; i >= 0; --i) {
        double s = y[i];
        for (int64_t k = i + 1; k < n; ++k) s -= L[(size_t)k * n + i] * x[k];
        x[i] = s / L[(size_t)i * n + i];
    }
}

static void vcycle(const PHier& H, int l, double* x, const double* b, int nu1, int nu2, double omega) {
    if (l == (int)H.lv.size() - 1) { coarse_solve(H, x, b); return; }
    const PLevel& F = H.lv[l];
    const PLevel& C = H.lv[l + 1];
    const size_t N = (size_t)F.bs * F.bs * F.bs;
    const size_t tot = F.cells(), totc = C.cells();
    std::vector<double> tmp, r(tot), bc(totc, 0.0), xc(totc, 0.0);
    p_jacobi(F, x, b, omega, nu1, tmp);
    p_matvec(F, x, r.data());
    for (size_t i = 0; i < tot; ++i) r[i] = b[i] - r[i];
    // restriction R = P^T / 8: each fine cell adds w / 8 of its residual to
    // each of the (up to 8) coarse cells its prolongation reads
    for (int64_t k = 0; k < F.n(); ++k) {
        int64_t bid = F.bids[k], bx = bid % F.nx, by = (bid / F.nx) % F.ny, bz = bid / (F.nx * F.ny);
        for (int cz = 0; cz < F.bs; ++cz)
            for (int cy = 0; cy < F.bs; ++cy)
                for (int cx = 0; cx < F.bs; ++cx) {
                    const int64_t g[3] = {bx * F.bs + cx, by * F.bs + cy, bz * F.bs + cz};
                    const double rf = r[k * N + ((size_t)cx | ((size_t)cy << F.lg) | ((size_t)cz << (2 * F.lg)))];
                    for (int c = 0; c < 8; ++c) {
                        int64_t q[3];
                        double w = 1.0;
                        for (int a = 0; a < 3; ++a) {
                            const bool far = (c >> a) & 1;
                            q[a] = (g[a] >> 1) + (far ? ((g[a] & 1) ? 1 : -1) : 0);
                            w *= far ? 0.25 : 0.75;
                        }
                        if (q[0] < 0 || q[1] < 0 || q[2] < 0) continue;
                        const int64_t ci = cell_index(C, H.slot[l + 1], q[0], q[1], q[2]);
                        if (ci >= 0 && (C.mask.empty() || C.mask[ci])) bc[ci] += (w * 0.125) * rf;
                    }
                }
    }
    vcycle(H, l + 1, xc.data(), bc.data(), nu1, nu2, omega);
    for (int64_t k = 0; k < F.n(); ++k) {  // prolongation: trilinear
        int64_t bid = F.bids[k], bx = bid % F.nx, by = (bid / F.nx) % F.ny, bz = bid / (F.nx * F.ny);
        for (int cz = 0; cz < F.bs; ++cz)
            for (int cy = 0; cy < F.bs; ++cy)
                for (int cx = 0; cx < F.bs; ++cx) {
                    const int64_t g[3] = {bx * F.bs + cx, by * F.bs + cy, bz * F.bs + cz};
                    double v = 0.0;
                    for (int c = 0; c < 8; ++c) {
                        int64_t q[3];
                        double w = 1.0;
                        for (int a = 0; a < 3; ++a) {
                            const bool far = (c >> a) & 1;
                            q[a] = (g[a] >> 1) + (far ? ((g[a] & 1) ? 1 : -1) : 0);
                            w *= far ? 0.25 : 0.75;
                        }
                        if (q[0] < 0 || q[1] < 0 || q[2] < 0) continue;
                        const int64_t ci = cell_index(C, H.slot[l + 1], q[0], q[1], q[2]);
                        if (ci >= 0 && (C.mask.empty() || C.mask[ci])) v += w * xc[ci];
                    }
                    x[k * N + ((size_t)cx | ((size_t)cy << F.lg) | ((size_t)cz << (2 * F.lg)))] += g_corr * v;
                }
    }
    p_jacobi(F, x, b, omega, nu2, tmp);
}

static double dot(const double* a, const double* b, size_t n) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) s += a[i] * b[i];
    return s;
}

static PLevel single_level(const int64_t* active, int64_t n_active, int64_t nx, int64_t ny, int64_t nz, int bs, double scale) {
    PLevel L;
    L.bs = bs; L.lg = ilog2(bs); L.nx = nx; L.ny = ny; L.nz = nz; L.scale = scale;
    L.bids.assign(active, active + n_active);  // caller order = slot order
    build_nbr(L);
    return L;
}

}  // extern "C" (reopened below)
extern "C" {

void or_poisson_matvec(const int64_t* active, int64_t n_active, int64_t nx, int64_t ny, int64_t nz, int bs,
                       double scale, const double* x, double* y) {
    PLevel L = single_level(active, n_active, nx, ny, nz, bs, scale);
    p_matvec(L, x, y);
}

void or_poisson_jacobi(const int64_t* active, int64_t n_active, int64_t nx, int64_t ny, int64_t nz, int bs,
                       double scale, double omega, int sweeps, double* x, const double* b) {
    PLevel L = single_level(active, n_active, nx, ny, nz, bs, scale);
    std::vector<double> tmp;
    p_jacobi(L, x, b, omega, sweeps, tmp);
}

void or_poisson_set_correction(double c) { g_corr = c; }

// Number of levels and cells per level of the hierarchy (for tests).
int or_poisson_levels(const int64_t* active, int64_t n_active, int64_t nx, int64_t ny, int64_t nz, int bs, int max_levels,
                      int64_t* cells_out) {
    PHier H;
    build_hier(H, active, n_active, nx, ny, nz, bs, max_levels);
    for (size_t l = 0; l < H.lv.size(); ++l) cells_out[l] = H.lv[l].cells();
    return (int)H.lv.size();
}

// mode 0: plain V-cycles; mode 1: V-cycle-preconditioned CG.  The unknowns
// are ordered by ascending block id (x, b are [n_active][bs^3]).  Iterates
// until ||b - A x|| <= tol ||b|| or max_iter; writes the relative residual
// history, returns the iteration count.
int or_poisson_solve(const int64_t* active, int64_t n_active, int64_t nx, int64_t ny, int64_t nz, int bs,
                     int max_levels, int nu1, int nu2, double omega, int mode, double tol, int max_iter,
                     double* x, const double* b, double* hist) {
    PHier H;
    build_hier(H, active, n_active, nx, ny, nz, bs, max_levels);
    const PLevel& F = H.lv[0];
    const size_t tot = F.cells();
    std::vector<double> r(tot), z(tot), p(tot), q(tot);
    const double bn = std::sqrt(dot(b, b, tot));
    if (bn == 0.0) { std::fill(x, x + tot, 0.0); return 0; }
    p_matvec(F, x, r.data());
    for (size_t i = 0; i < tot; ++i) r[i] = b[i] - r[i];
    double rn = std::sqrt(dot(r.data(), r.data(), tot));
    int it = 0;
    if (mode == 0) {
        while (rn > tol * bn && it < max_iter) {
            vcycle(H, 0, x, b, nu1, nu2, omega);
            p_matvec(F, x, r.data());
            for (size_t i = 0; i < tot; ++i) r[i] = b[i] - r[i];
            rn = std::sqrt(dot(r.data(), r.data(), tot));
            if (hist) hist[it] = rn / bn;
            ++it;
        }
        return it;
    }
    std::fill(z.begin(), z.end(), 0.0);
    vcycle(H, 0, z.data(), r.data(), nu1, nu2, omega);
    p = z;
    double rz = dot(r.data(), z.data(), tot);
    while (rn > tol * bn && it < max_iter) {
        p_matvec(F, p.data(), q.data());
        double alpha = rz / dot(p.data(), q.data(), tot);
        for (size_t i = 0; i < tot; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
        rn = std::sqrt(dot(r.data(), r.data(), tot));
        if (hist) hist[it] = rn / bn;
        ++it;
        if (rn <= tol * bn) break;
        std::fill(z.begin(), z.end(), 0.0);
        vcycle(H, 0, z.data(), r.data(), nu1, nu2, omega);
        double rz2 = dot(r.data(), z.data(), tot);
        double beta = rz2 / rz;
        rz = rz2;
        for (size_t i = 0; i < tot; ++i) p[i] = z[i] + beta * p[i];
    }
    return it;
}

}  // extern "C"

// ===========================================================================
// Surface reconstruction from particles (particles/{sort,splat,finalize}.rs).
// ===========================================================================
extern "C" {

// particles/sort.rs:31-144 place: instance i of the base cloud has origin
// 0.2 smax + 0.6 smax bs (b_i - bbox) and scale smin * factor * bs (bs =
// 1 / span_max); each base point j is placed at origin + scale (b_j - bbox),
// kept when inside the domain bounds and its truncated cell inside the grid.
// Positions come out instance-major; bids are their centre blocks.  Writes
// at most cap particles; returns the number placed.
int64_t or_place(const float* base, int64_t n_base, const float* bbox_min, float span_max, int64_t sx, int64_t sy,
                 int64_t sz, int bsx, float factor, int64_t n_instances, const float* dom_min, const float* dom_max,
                 float* pos_out, int64_t* bids_out, int64_t cap) {
    const int64_t nx = (sx + bsx - 1) / bsx, ny = (sy + bsx - 1) / bsx;
    const int lg = ilog2(bsx);
    const float base_scale = 1.0f / span_max;
    const float smin = (float)std::min(sx, std::min(sy, sz)), smax = (float)std::max(sx, std::max(sy, sz));
    const float scale = smin * factor;
    const float inst_scale = scale * base_scale;
    const int64_t dims[3] = {sx, sy, sz};
    int64_t c = 0;
    for (int64_t i = 0; i < n_instances; ++i) {
        const float* bi = base + 3 * i;
        float origin[3];
        for (int a = 0; a < 3; ++a) origin[a] = 0.2f * smax + ((0.6f * smax) * base_scale) * (bi[a] - bbox_min[a]);
        for (int64_t j = 0; j < n_base; ++j) {
            const float* bj = base + 3 * j;
            float p[3];
            bool in = true;
            for (int a = 0; a < 3; ++a) {
                p[a] = origin[a] + inst_scale * (bj[a] - bbox_min[a]);
                if (!(p[a] >= dom_min[a] && p[a] <= dom_max[a])) in = false;
            }
            if (!in) continue;
            int32_t ip[3];
            for (int a = 0; a < 3; ++a) {
                ip[a] = (int32_t)p[a];
                if (ip[a] < 0 || ip[a] >= dims[a]) in = false;
            }
            if (!in) continue;
            if (c < cap) {
                for (int a = 0; a < 3; ++a) pos_out[3 * c + a] = p[a];
                bids_out[c] = (int64_t)(ip[0] >> lg) + (int64_t)(ip[1] >> lg) * nx + (int64_t)(ip[2] >> lg) * nx * ny;
            }
            ++c;
        }
    }
    return c;
}

// particles/active.rs:15-47 footprint union with r_scan = r_particle +
// nb_dist: sorted unique bids; returns the count (out may be NULL).
int64_t or_surface_active(const float* pos, int64_t n, int64_t sx, int64_t sy, int64_t sz, int bsx, float r_scan,
                          int64_t* out) {
    int64_t nx = (sx + bsx - 1) / bsx, ny = (sy + bsx - 1) / bsx, nz = (sz + bsx - 1) / bsx;
    std::vector<uint8_t> mark((size_t)(nx * ny * nz), 0);
    const float rs = r_scan / (float)bsx;
    for (int64_t i = 0; i < n; ++i) {
        int32_t x1, x2, y1, y2, z1, z2;
        footprint_axis(pos[3 * i], rs, bsx, nx, &x1, &x2);
        footprint_axis(pos[3 * i + 1], rs, bsx, ny, &y1, &y2);
        footprint_axis(pos[3 * i + 2], rs, bsx, nz, &z1, &z2);
        for (int32_t bz = z1; bz <= z2; ++bz)
            for (int32_t by = y1; by <= y2; ++by)
                for (int32_t bx = x1; bx <= x2; ++bx) mark[bx + by * nx + bz * nx * ny] = 1;
    }
    int64_t c = 0;
    for (int64_t b = 0; b < nx * ny * nz; ++b)
        if (mark[b]) { if (out) out[c] = b; ++c; }
    return c;
}

// particles/splat.rs:92-319 splat into active blocks filled with the full
// value: per particle, over its footprint voxels [ceil(p - r - 1/2),
// floor(p + r - 1/2)] (r = r_scan, clipped to its block's staging window),
// dist_sq = dx dx + (dz dz + dy dy) with d = voxel - (p - 1/2); where dist_sq
// <= r^2 the voxel takes min(old, q), q = dist_sq / r^2 (f32 storage) or
// round(dist_sq / r^2 * qmax) (Density: qmax 65535, channel.rs:392-417;
// Density8: qmax 255, channel.rs:425-447).  Voxels
// outside the domain or in blocks outside `active` are skipped (the
// reference's commit skips them).  The reference stages per block and
// commits by colour; min is order-independent, so a direct scatter-min gives
// the same grid.  out is [n_active][bsx^3] f32 (the stored integers as
// floats when qmax != 0; qmax 0 is f32 storage).
void or_density_splat(const float* pos, int64_t n, int64_t sx, int64_t sy, int64_t sz, int bsx, float r_particle,
                      float nb_dist, int qmax, const int64_t* active, int64_t n_active, float* out) {
    const int64_t nx = (sx + bsx - 1) / bsx, ny = (sy + bsx - 1) / bsx, nz = (sz + bsx - 1) / bsx;
    const int lg = ilog2(bsx), msk = bsx - 1;
    const int64_t N = (int64_t)bsx * bsx * bsx;
    std::vector<int64_t> slot((size_t)(nx * ny * nz), -1);
    for (int64_t k = 0; k < n_active; ++k) slot[active[k]] = k;
    const float r_scan = r_particle + nb_dist;
    const float dmax = r_scan * r_scan, inv = 1.0f / dmax;
    const int m = (int)ceilf(r_scan);
    std::vector<uint32_t> q((size_t)(n_active * N), qmax ? (uint32_t)qmax : 0x3f800000u);  // full: MAX or 1.0f
    for (int64_t i = 0; i < n; ++i) {
        const float* p = pos + 3 * i;
        int32_t b0[3];
        for (int a = 0; a < 3; ++a) b0[a] = ((int32_t)p[a] >> lg) << lg;
        int32_t lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(std::max((int32_t)ceilf((p[a] - r_scan) - 0.5f), b0[a] - m), b0[a] + bsx + m - 1);
            hi[a] = std::min(std::max((int32_t)floorf((p[a] + r_scan) - 0.5f), b0[a] - m), b0[a] + bsx + m - 1);
        }
        const float px0 = p[0] - 0.5f, py0 = p[1] - 0.5f, pz0 = p[2] - 0.5f;
        for (int32_t iz = lo[2]; iz <= hi[2]; ++iz) {
            const float dz = (float)iz - pz0, dz2 = dz * dz;
            for (int32_t iy = lo[1]; iy <= hi[1]; ++iy) {
                const float dy = (float)iy - py0, dyz = dz2 + dy * dy;
                for (int32_t ix = lo[0]; ix <= hi[0]; ++ix) {
                    const float dx = (float)ix - px0;
                    const float d2 = dx * dx + dyz;
                    if (!(d2 <= dmax)) continue;
                    if (ix < 0 || iy < 0 || iz < 0 || ix >= sx || iy >= sy || iz >= sz) continue;
                    const int64_t s = slot[(ix >> lg) + (int64_t)(iy >> lg) * nx + (int64_t)(iz >> lg) * nx * ny];
                    if (s < 0) continue;
                    const float t = d2 * inv;
                    uint32_t v;
                    if (qmax) v = (uint32_t)(int32_t)roundf(t * (float)qmax) & (uint32_t)qmax;
                    else memcpy(&v, &t, 4);
                    uint32_t& o = q[(size_t)(s * N + ((ix & msk) | ((iy & msk) << lg) | ((iz & msk) << (2 * lg))))];
                    if (v < o) o = v;
                }
            }
        }
    }
    for (size_t k = 0; k < q.size(); ++k) {
        if (qmax) out[k] = (float)q[k];
        else memcpy(&out[k], &q[k], 4);
    }
}

// particles/finalize.rs:35-71 in place on [n][bsx^3] values (the stored
// integers as floats when qmax != 0): ratio (dequantised, q / qmax),
// touched = ratio < 0.999, f = 1 - clamp((sqrt(ratio r^2) - r_p + r_p) /
// (2 r_p + nb), 0, 1), 0 when untouched; stored back (round(f * qmax)).
void or_density_finalize(float* vals, int64_t n, int qmax, float r_particle, float nb_dist) {
    const float r_scan = r_particle + nb_dist, dmax = r_scan * r_scan;
    const float denom = 2.0f * r_particle + nb_dist;
    for (int64_t k = 0; k < n; ++k) {
        const float ratio = qmax ? (float)(uint32_t)vals[k] * (1.0f / (float)qmax) : vals[k];
        const bool touched = ratio < 0.999f;
        const float dist = sqrtf(ratio * dmax) - r_particle;
        float t = (dist + r_particle) / denom;
        t = std::min(std::max(t, 0.0f), 1.0f);
        const float f = touched ? 1.0f - t : 0.0f;
        if (qmax) {
            const float r = roundf(f * (float)qmax);
            vals[k] = (float)((uint32_t)(int32_t)r & (uint32_t)qmax);
        } else {
            vals[k] = f;
        }
    }
}

}  // extern "C"

// ===========================================================================
// Refinement map (multires/refinement.rs).
// ===========================================================================
extern "C" {

// refinement.rs:63-107 regularize_refinement_map: passes ll = 1 .. n_levels-2;
// a block at level >= ll whose minimum neighbour level (26-neighbourhood, in
// range; starting from n_levels - 1) is ll - 1 moves to level ll.
void or_regularize_refinement_map(uint8_t* map, int64_t nx, int64_t ny, int64_t nz, int n_levels) {
    if (n_levels <= 2) return;
    const int64_t n = nx * ny * nz;
    std::vector<uint8_t> prev(map, map + n);
    for (int ll = 1; ll <= n_levels - 2; ++ll) {
        for (int64_t bid = 0; bid < n; ++bid) {
            const uint8_t level = prev[bid];
            uint8_t out = level;
            if (level >= ll) {
                const int64_t bx = bid % nx, by = (bid / nx) % ny, bz = bid / (nx * ny);
                uint8_t level2 = (uint8_t)(n_levels - 1);
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            if (!dx && !dy && !dz) continue;
                            const int64_t X = bx + dx, Y = by + dy, Z = bz + dz;
                            if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
                            level2 = std::min(level2, prev[X + Y * nx + Z * nx * ny]);
                        }
                if (level2 == ll - 1) out = (uint8_t)ll;
            }
            map[bid] = out;
        }
        std::copy(map, map + n, prev.begin());
    }
}

// refinement.rs:124-208 compute_block_topology (levelMg == 0): per block the
// user flags plus DOM_BORDER (1 << 1) on the block grid's faces, FINE_COARSE
// (1 << 3) when a neighbour is coarser, COARSE_FINE (1 << 2) when one is
// finer; the FINE_COARSE blocks of each level in bid order; the number of
// EXISTS (1 << 12) blocks.  fc_out is [n_levels][n] (each row holds the list
// of its level, fc_count[l] entries).
uint64_t or_block_topology(const uint8_t* map, int64_t nx, int64_t ny, int64_t nz, int n_levels, const uint16_t* user,
                           uint16_t* flags_out, int64_t* fc_out, int64_t* fc_count) {
    const int64_t n = nx * ny * nz;
    for (int l = 0; l < n_levels; ++l) fc_count[l] = 0;
    uint64_t n_act = 0;
    for (int64_t bid = 0; bid < n; ++bid) {
        const uint8_t level = map[bid];
        uint16_t f = user ? user[bid] : 0;
        const int64_t bx = bid % nx, by = (bid / nx) % ny, bz = bid / (nx * ny);
        if (bx == 0 || bx == nx - 1 || by == 0 || by == ny - 1 || bz == 0 || bz == nz - 1) f |= 1u << 1;
        uint8_t lmax = 0, lmin = (uint8_t)(n_levels - 1);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (!dx && !dy && !dz) continue;
                    const int64_t X = bx + dx, Y = by + dy, Z = bz + dz;
                    if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
                    const uint8_t l2 = map[X + Y * nx + Z * nx * ny];
                    lmax = std::max(lmax, l2);
                    lmin = std::min(lmin, l2);
                }
        if (lmax > level) f |= 1u << 3;
        if (lmin < level) f |= 1u << 2;
        if (f & (1u << 3)) fc_out[(int64_t)level * n + fc_count[level]++] = bid;
        if (f & (1u << 12)) ++n_act;
        flags_out[bid] = f;
    }
    return n_act;
}

}  // extern "C"
