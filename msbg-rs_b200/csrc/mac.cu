// mac.cu -- MAC grid channels, normalize_velocity, divergence (fluid/mac.rs),
// trilinear sampling and G2P (fluid/g2p.rs, math/gather.rs, math/sample.rs),
// the FLIP/PIC blend and the 2^3 downsample (multires/downsample.rs).
//
// Built with --fmad=false: every sample is the reference's f32 arithmetic
// (three-level fmaf lerp of gather_map's corners), bit-identical to the CPU
// restatement.
#include <algorithm>

#include "mac.cuh"

msbg_mac::~msbg_mac() {
    for (auto* c : ch) delete c;
}

namespace msbg {

void mac_ensure(msbg_mac* m, const uint64_t* bids, size_t n, int32_t* slots) {
    for (int c = 0; c < 6; ++c) grid_ensure(m->ch[c], bids, n, c == 0 ? slots : nullptr);
}

struct SampleGrid {
    const float* payload;  // f32 grids (the G2P path); null otherwise
    const void* raw;       // the payload in the grid's storage type
    const int32_t* dense;  // bid -> code, or null (use the hash)
    DevHash hash;
    int64_t nx, ny, nz;
    int32_t sx, sy, sz;
    int lg;
    float empty, full;
};

// any_dtype: the Sampler of any InterpElem (sample.rs:45-70 Dequant) reads
// every storage type; the MAC velocity paths need f32.
static SampleGrid sample_grid(msbg_grid* g, bool any_dtype = false) {
    MSBG_REQUIRE(any_dtype || g->dtype == MSBG_F32, "sampling needs an f32 grid");
    SampleGrid s;
    s.payload = g->dtype == MSBG_F32 ? g->payload.as<float>() : nullptr;
    s.raw = g->payload.p;
    s.hash = device_hash(g);
    s.dense = device_dense(g);
    s.nx = (int64_t)g->nx; s.ny = (int64_t)g->ny; s.nz = (int64_t)g->nz;
    s.sx = (int32_t)g->sx; s.sy = (int32_t)g->sy; s.sz = (int32_t)g->sz;
    s.lg = g->lg;
    s.empty = quantize_roundtrip(g->dtype, g->empty_value);
    s.full = quantize_roundtrip(g->dtype, g->full_value);
    return s;
}

template <class E = ElemF32>
__device__ __forceinline__ float code_value(const SampleGrid& g, int32_t code, int vid) {
    if (code >= 0) {
        if constexpr (std::is_same<E, ElemF32>::value) return g.payload[((size_t)code << (3 * g.lg)) + vid];
        else return E::load(static_cast<const typename E::T*>(g.raw)[((size_t)code << (3 * g.lg)) + vid]);
    }
    return code == kCodeFull ? g.full : g.empty;
}

__device__ __forceinline__ int32_t block_code(const SampleGrid& g, uint64_t bid) {
    return g.dense ? __ldg(g.dense + bid) : hash_find(g.hash, bid);
}

__device__ __forceinline__ float lerpf(float a, float b, float t) { return fmaf(b - a, t, a); }

// gather_map (math/gather.rs:54-158, dmax = 1) + trilinear_value (sample.rs:203-211)
// at a position already in the grid's node frame.
template <class E = ElemF32>
__device__ float sample_linear_dev(const SampleGrid& g, float x, float y, float z, int bc) {
    const int bsx = 1 << g.lg, mask = bsx - 1, lg = g.lg;
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const int32_t ix0 = (int32_t)fx, iy0 = (int32_t)fy, iz0 = (int32_t)fz;
    float c[8];
    bool fast = false;
    if (ix0 >= 0 && iy0 >= 0 && iz0 >= 0 && ix0 + 1 < g.sx && iy0 + 1 < g.sy && iz0 + 1 < g.sz) {
        const int vx0 = ix0 & mask, vy0 = iy0 & mask, vz0 = iz0 & mask;
        if (vx0 + 1 < bsx && vy0 + 1 < bsx && vz0 + 1 < bsx) {
            const uint64_t bid = (uint64_t)(ix0 >> lg) + (uint64_t)(iy0 >> lg) * g.nx + (uint64_t)(iz0 >> lg) * g.nx * g.ny;
            const int32_t code = block_code(g, bid);
            int s = 0;
            for (int k = 0; k < 2; ++k)
                for (int j = 0; j < 2; ++j)
                    for (int i = 0; i < 2; ++i)
                        c[s++] = code_value<E>(g, code, (vx0 + i) | ((vy0 + j) << lg) | ((vz0 + k) << (2 * lg)));
            fast = true;
        }
    }
    if (!fast) {
        const int64_t bx0 = min(max((int64_t)(ix0 >> lg), (int64_t)0), g.nx - 1);
        const int64_t by0 = min(max((int64_t)(iy0 >> lg), (int64_t)0), g.ny - 1);
        const int64_t bz0 = min(max((int64_t)(iz0 >> lg), (int64_t)0), g.nz - 1);
        int32_t codes[8];
        for (int s = 0; s < 8; ++s) {
            const int64_t bxx = min(bx0 + (s & 1), g.nx - 1), byy = min(by0 + ((s >> 1) & 1), g.ny - 1),
                          bzz = min(bz0 + (s >> 2), g.nz - 1);
            codes[s] = block_code(g, (uint64_t)bxx + (uint64_t)byy * g.nx + (uint64_t)bzz * g.nx * g.ny);
        }
        int s = 0;
        for (int k = 0; k < 2; ++k) {
            int32_t rz;
            const bool okz = resolve_axis(iz0 + k, g.sz - 1, bc, &rz);
            for (int j = 0; j < 2; ++j) {
                int32_t ry;
                const bool oky = resolve_axis(iy0 + j, g.sy - 1, bc, &ry);
                for (int i = 0; i < 2; ++i) {
                    int32_t rx;
                    const bool okx = resolve_axis(ix0 + i, g.sx - 1, bc, &rx);
                    if (okx && oky && okz) {
                        const int sl = (int)((((rx >> lg) - bx0) & 1) | ((((ry >> lg) - by0) & 1) << 1) |
                                             ((((rz >> lg) - bz0) & 1) << 2));
                        c[s] = code_value<E>(g, codes[sl], (rx & mask) | ((ry & mask) << lg) | ((rz & mask) << (2 * lg)));
                    } else {
                        c[s] = g.empty;
                    }
                    ++s;
                }
            }
        }
    }
    const float u = x - fx, v = y - fy, w = z - fz;
    const float c00 = lerpf(c[0], c[1], u), c10 = lerpf(c[2], c[3], u), c01 = lerpf(c[4], c[5], u),
                c11 = lerpf(c[6], c[7], u);
    const float c0 = lerpf(c00, c10, v), c1 = lerpf(c01, c11, v);
    return lerpf(c0, c1, w);
}

template <class E>
__global__ void sample_linear_kernel(SampleGrid g, const float* pos, size_t n, int align, int bc, float* out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        if (align == 1) { x = x - 0.5f; y = y - 0.5f; z = z - 0.5f; }
        out[i] = sample_linear_dev<E>(g, x, y, z, bc);
    }
}

// gather_map (math/gather.rs:54-158) for a window of SPAN = dmax + 1 (2 or
// 4) anchored at (ix0, iy0, iz0): the one-block fast path, else the 2x2x2
// block slots from the clamped anchor block and per-axis boundary resolution.
// A Neumann window far outside the domain can reflect to a block before the
// anchor block, where the crate's slot index leaves the 2x2x2 slots
// (undefined there); slot offsets are taken mod 2.
template <int SPAN, class E = ElemF32>
__device__ void gather_window_dev(const SampleGrid& g, int32_t ix0, int32_t iy0, int32_t iz0, int bc, float* out) {
    constexpr int DMAX = SPAN - 1;
    const int bsx = 1 << g.lg, mask = bsx - 1, lg = g.lg;
    if (ix0 >= 0 && iy0 >= 0 && iz0 >= 0 && ix0 + DMAX < g.sx && iy0 + DMAX < g.sy && iz0 + DMAX < g.sz) {
        const int vx0 = ix0 & mask, vy0 = iy0 & mask, vz0 = iz0 & mask;
        if (vx0 + DMAX < bsx && vy0 + DMAX < bsx && vz0 + DMAX < bsx) {
            const uint64_t bid = (uint64_t)(ix0 >> lg) + (uint64_t)(iy0 >> lg) * g.nx + (uint64_t)(iz0 >> lg) * g.nx * g.ny;
            const int32_t code = block_code(g, bid);
            int s = 0;
#pragma unroll
            for (int k = 0; k < SPAN; ++k)
#pragma unroll
                for (int j = 0; j < SPAN; ++j)
#pragma unroll
                    for (int i = 0; i < SPAN; ++i)
                        out[s++] = code_value<E>(g, code, (vx0 + i) | ((vy0 + j) << lg) | ((vz0 + k) << (2 * lg)));
            return;
        }
    }
    const int64_t bx0 = min(max((int64_t)(ix0 >> lg), (int64_t)0), g.nx - 1);
    const int64_t by0 = min(max((int64_t)(iy0 >> lg), (int64_t)0), g.ny - 1);
    const int64_t bz0 = min(max((int64_t)(iz0 >> lg), (int64_t)0), g.nz - 1);
    int32_t codes[8];
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const int64_t bxx = min(bx0 + (s & 1), g.nx - 1), byy = min(by0 + ((s >> 1) & 1), g.ny - 1),
                      bzz = min(bz0 + (s >> 2), g.nz - 1);
        codes[s] = block_code(g, (uint64_t)bxx + (uint64_t)byy * g.nx + (uint64_t)bzz * g.nx * g.ny);
    }
    int s = 0;
#pragma unroll
    for (int k = 0; k < SPAN; ++k) {
        int32_t rz;
        const bool okz = resolve_axis(iz0 + k, g.sz - 1, bc, &rz);
#pragma unroll
        for (int j = 0; j < SPAN; ++j) {
            int32_t ry;
            const bool oky = resolve_axis(iy0 + j, g.sy - 1, bc, &ry);
#pragma unroll
            for (int i = 0; i < SPAN; ++i) {
                int32_t rx;
                const bool okx = resolve_axis(ix0 + i, g.sx - 1, bc, &rx);
                if (okx && oky && okz) {
                    const int sl = (int)((((rx >> lg) - bx0) & 1) | ((((ry >> lg) - by0) & 1) << 1) |
                                         ((((rz >> lg) - bz0) & 1) << 2));
                    out[s] = code_value<E>(g, codes[sl], (rx & mask) | ((ry & mask) << lg) | ((rz & mask) << (2 * lg)));
                } else {
                    out[s] = g.empty;
                }
                ++s;
            }
        }
    }
}

// math/bspline.rs:4-32 uniform cubic B-spline weights, first and second
// derivative weights (f32, left to right; built without contraction).
__device__ __forceinline__ void cubic_w_dev(float t, float w[4]) {
    const float m = 1.0f - t, s6 = 1.0f / 6.0f, t3 = 2.0f / 3.0f;
    w[0] = ((s6 * m) * m) * m;
    w[1] = t3 - ((0.5f * t) * t) * (2.0f - t);
    w[2] = t3 - ((0.5f * m) * m) * (1.0f + t);
    w[3] = ((s6 * t) * t) * t;
}
__device__ __forceinline__ void cubic_dw_dev(float t, float w[4]) {
    const float m = 1.0f - t;
    w[0] = ((-m) * m) / 2.0f;
    w[1] = (0.5f * t) * t - (2.0f - t) * t;
    w[2] = m * (t + 1.0f) - (0.5f * m) * m;
    w[3] = (t * t) / 2.0f;
}
__device__ __forceinline__ void cubic_d2w_dev(float t, float w[4]) {
    w[0] = 1.0f - t;
    w[1] = 3.0f * t - 2.0f;
    w[2] = 1.0f - 3.0f * t;
    w[3] = t;
}
// (f * w).reduce_sum() of one window row: lanes added in order
__device__ __forceinline__ float row_dot_dev(const float* f, const float w[4]) {
    return ((f[0] * w[0] + f[1] * w[1]) + f[2] * w[2]) + f[3] * w[3];
}

// Sample for SparseGrid (math/sample.rs:493-649).  mode 0: cubic B-spline
// value -> out[n]; 1: cubic gradient -> out[n][3]; 2: cubic Hessian (fxx,
// fyy, fzz, fxy, fxz, fyz) -> out[n][6]; 3: trilinear gradient
// (trilinear_value_grad, sample.rs:215-237) at `align` -> out[n][3].  The
// cubic basis is cell-centred whatever the alignment: window base
// floor(p - 0.5) - 1, t = frac(p - 0.5).  One thread per position.
template <class E>
__global__ void sample_ext_kernel(SampleGrid g, const float* __restrict__ pos, size_t n, int mode, int align, int bc,
                                  float* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        if (mode == 3) {
            if (align == 1) { x = x - 0.5f; y = y - 0.5f; z = z - 0.5f; }
            const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
            float c[8];
            gather_window_dev<2, E>(g, (int32_t)fx, (int32_t)fy, (int32_t)fz, bc, c);
            const float u = x - fx, v = y - fy, w = z - fz;
            const float f01234567 = ((((((c[7] - c[6]) - c[5]) + c[4]) - c[3]) + c[2]) + c[1]) - c[0];
            const float f01234567u = f01234567 * u;
            const float f01234567uf6420 = (((f01234567u + c[6]) - c[4]) - c[2]) + c[0];
            const float f5410 = ((c[5] - c[4]) - c[1]) + c[0];
            const float f3210 = ((c[3] - c[2]) - c[1]) + c[0];
            out[3 * i] = fmaf(f01234567 * v + f5410, w, (f3210 * v + c[1]) - c[0]);
            out[3 * i + 1] = fmaf(f01234567uf6420, w, (f3210 * u + c[2]) - c[0]);
            out[3 * i + 2] = fmaf(f01234567uf6420, v, (f5410 * u + c[4]) - c[0]);
            continue;
        }
        x = x - 0.5f; y = y - 0.5f; z = z - 0.5f;
        const float xf = floorf(x), yf = floorf(y), zf = floorf(z);
        const float tx = x - xf, ty = y - yf, tz = z - zf;
        float win[64];
        gather_window_dev<4, E>(g, (int32_t)xf - 1, (int32_t)yf - 1, (int32_t)zf - 1, bc, win);
        float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4], ddx[4], ddy[4], ddz[4];
        cubic_w_dev(tx, wx); cubic_w_dev(ty, wy); cubic_w_dev(tz, wz);
        cubic_dw_dev(tx, dx); cubic_dw_dev(ty, dy); cubic_dw_dev(tz, dz);
        cubic_d2w_dev(tx, ddx); cubic_d2w_dev(ty, ddy); cubic_d2w_dev(tz, ddz);
        float val = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
        float fxx = 0.0f, fyy = 0.0f, fzz = 0.0f, fxy = 0.0f, fxz = 0.0f, fyz = 0.0f;
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float* f = win + 16 * k + 4 * j;
                const float sx = row_dot_dev(f, wx);
                if (mode == 0) {
                    val = fmaf(sx, wy[j] * wz[k], val);
                } else if (mode == 1) {
                    const float sxp = row_dot_dev(f, dx);
                    const float wyz = wy[j] * wz[k];
                    val = fmaf(sx, wyz, val);
                    gx = fmaf(sxp, wyz, gx);
                    gy = fmaf(sx, dy[j] * wz[k], gy);
                    gz = fmaf(sx, wy[j] * dz[k], gz);
                } else {
                    const float sxp = row_dot_dev(f, dx), sxpp = row_dot_dev(f, ddx);
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
        else if (mode == 1) {
            out[3 * i] = gx;
            out[3 * i + 1] = gy;
            out[3 * i + 2] = gz;
        } else {
            float* h = out + 6 * i;
            h[0] = fxx; h[1] = fyy; h[2] = fzz; h[3] = fxy; h[4] = fxz; h[5] = fyz;
        }
    }
}

// Block code lookups of the G2P interior path through the hash (grids too
// large for a dense table) out of line, so the kernel's lookup sites stay
// small.
__device__ __noinline__ int32_t block_code_hashed(const DevHash h, uint64_t bid) { return hash_find(h, bid); }

// One component's sample when its 2x2x2 corners lie inside the domain
// (gather_map's interior case, no boundary condition applies).  CornerBase:
// the sample's corner (0, 0, 0), its block's code c0 and the axes along
// which the +1 corners cross into the next block.
struct CornerBase {
    int32_t jx0, jy0, jz0;  // corner (0, 0, 0), 0 where not ok
    int32_t c0, vid0;
    float u, v, w;  // x - floor(x), ...
    bool ok, crx, cry, crz;
};

__device__ __forceinline__ CornerBase corner_base(const SampleGrid& g, float x, float y, float z) {
    CornerBase b;
    const int mask = (1 << g.lg) - 1, lg = g.lg;
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    b.u = x - fx;
    b.v = y - fy;
    b.w = z - fz;
    const int32_t ix0 = (int32_t)fx, iy0 = (int32_t)fy, iz0 = (int32_t)fz;
    b.ok = ix0 >= 0 && iy0 >= 0 && iz0 >= 0 && ix0 + 1 < g.sx && iy0 + 1 < g.sy && iz0 + 1 < g.sz;
    b.jx0 = b.ok ? ix0 : 0;
    b.jy0 = b.ok ? iy0 : 0;
    b.jz0 = b.ok ? iz0 : 0;
    const int lx = b.jx0 & mask, ly = b.jy0 & mask, lz = b.jz0 & mask;
    b.crx = lx == mask;
    b.cry = ly == mask;
    b.crz = lz == mask;
    b.vid0 = lx | (ly << lg) | (lz << (2 * lg));
    // a dense table has at most 2^24 entries, so its index arithmetic is 32-bit
    if (g.dense) {
        const uint32_t bid0 = (uint32_t)(b.jx0 >> lg) + (uint32_t)(b.jy0 >> lg) * (uint32_t)g.nx +
                              (uint32_t)(b.jz0 >> lg) * (uint32_t)(g.nx * g.ny);
        b.c0 = b.ok ? __ldg(g.dense + bid0) : kCodeEmpty;
    } else {
        const uint64_t bid0 = (uint64_t)(b.jx0 >> lg) + (uint64_t)(b.jy0 >> lg) * (uint64_t)g.nx +
                              (uint64_t)(b.jz0 >> lg) * (uint64_t)g.nx * g.ny;
        b.c0 = b.ok ? block_code_hashed(g.hash, bid0) : kCodeEmpty;
    }
    return b;
}

// The eight corner values when no corner crosses a block: c0's block at
// constant offsets from corner (0, 0, 0) (corner s = (i, j, k) at
// vid0 + i + j bsx + k bsx^2).
__device__ __forceinline__ void corners_one_block(const SampleGrid& g, const CornerBase& b, float c[8]) {
    const int bs = 1 << g.lg;
    if (b.c0 >= 0) {
        const float* p = g.payload + ((size_t)b.c0 << (3 * g.lg)) + b.vid0;
#pragma unroll
        for (int s = 0; s < 8; ++s) c[s] = __ldg(p + ((s & 1) ? 1 : 0) + ((s & 2) ? bs : 0) + ((s & 4) ? bs * bs : 0));
    } else {
        const float v = b.c0 == kCodeFull ? g.full : g.empty;
#pragma unroll
        for (int s = 0; s < 8; ++s) c[s] = v;
    }
}

// The eight corner values in general: corner s = (i, j, k) at local index
// vid0 + i dv[0] + j dv[1] + k dv[2] (a step that wraps to the next block's
// first cell where the corner crosses) in the block across the axes it
// crosses (looked up only for the crossings a sample has).
__device__ __forceinline__ void corners_general(const SampleGrid& g, const CornerBase& b, float c[8]) {
    const int bsx = 1 << g.lg, mask = bsx - 1, lg = g.lg;
    const int32_t dv0 = b.crx ? -mask : 1, dv1 = b.cry ? -(mask << lg) : bsx, dv2 = b.crz ? -(mask << (2 * lg)) : bsx << lg;
    // the codes of the blocks across the crossed axes (x, y, xy, z, xz, yz, xyz)
    int32_t cc[8];
    cc[0] = b.c0;
    if (g.dense) {
        const uint32_t sy = (uint32_t)g.nx, sz = (uint32_t)(g.nx * g.ny);
        const uint32_t bid0 = (uint32_t)(b.jx0 >> lg) + (uint32_t)(b.jy0 >> lg) * sy + (uint32_t)(b.jz0 >> lg) * sz;
#pragma unroll
        for (int s = 1; s < 8; ++s) {
            const bool need = b.ok && (!(s & 1) || b.crx) && (!(s & 2) || b.cry) && (!(s & 4) || b.crz);
            cc[s] = need ? __ldg(g.dense + (bid0 + (uint32_t)(s & 1) + ((s & 2) ? sy : 0u) + ((s & 4) ? sz : 0u))) : b.c0;
        }
    } else {
        const uint64_t sy = (uint64_t)g.nx, sz = (uint64_t)g.nx * g.ny;
        const uint64_t bid0 = (uint64_t)(b.jx0 >> lg) + (uint64_t)(b.jy0 >> lg) * sy + (uint64_t)(b.jz0 >> lg) * sz;
#pragma unroll
        for (int s = 1; s < 8; ++s) {
            const bool need = b.ok && (!(s & 1) || b.crx) && (!(s & 2) || b.cry) && (!(s & 4) || b.crz);
            cc[s] = need ? block_code_hashed(g.hash, bid0 + (uint64_t)(s & 1) + ((s & 2) ? sy : 0) + ((s & 4) ? sz : 0))
                         : b.c0;
        }
    }
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const int x = (s & 1) && b.crx ? 1 : 0, y = (s & 2) && b.cry ? 2 : 0, z = (s & 4) && b.crz ? 4 : 0;
        const int32_t code = cc[x | y | z];
        const int32_t vid = b.vid0 + ((s & 1) ? dv0 : 0) + ((s & 2) ? dv1 : 0) + ((s & 4) ? dv2 : 0);
        c[s] = code >= 0 ? __ldg(g.payload + ((size_t)code << (3 * g.lg)) + vid) : (code == kCodeFull ? g.full : g.empty);
    }
}

// The same three-level lerp as sample_linear_dev.
__device__ __forceinline__ float lerp_corners(const float c[8], const CornerBase& b) {
    const float c00 = lerpf(c[0], c[1], b.u), c10 = lerpf(c[2], c[3], b.u), c01 = lerpf(c[4], c[5], b.u),
                c11 = lerpf(c[6], c[7], b.u);
    const float c0 = lerpf(c00, c10, b.v), c1 = lerpf(c01, c11, b.v);
    return lerpf(c0, c1, b.w);
}

// The general gather (boundary conditions) out of line: rare, and large.
__device__ __noinline__ float sample_linear_boundary(const SampleGrid g, float x, float y, float z, int bc) {
    return sample_linear_dev(g, x, y, z, bc);
}

// MacSampler::sample::<Linear> (fluid/g2p.rs:26-32): component a is a
// cell-centred sample of velocity[a] at p - 1/2 e_a.  One thread per
// particle; the block lookups, then the 24 corner loads, are issued
// together; only samples whose corners leave the domain take the general
// gather (boundary conditions), after the interior samples are stored.
// (One thread per particle and component measured slower: 1.34 against
// 0.95 ms at 25.4 M particles.)
//
// BLEND 1 writes g2p_blend (fluid/g2p.rs:42-45) of the sample instead:
// (u_old + (u - u_tilde)) alpha + u (1 - alpha), with u_tilde the caller's
// array, or the sample itself where u_tilde is null (no grid change between
// the two samples); the same operations as g2p_blend_kernel, so the result
// equals the sample-then-blend pair bit for bit without the round trip of
// the samples through memory.
struct BlendArgs {
    const float* u_old;
    const float* u_tilde;
    float alpha;
};

template <int BLEND>
__global__ void __launch_bounds__(256, 4) g2p_kernel(SampleGrid gx, SampleGrid gy, SampleGrid gz,
                                                  const float* __restrict__ pos, size_t n, int bc, BlendArgs bl,
                                                  float* __restrict__ out) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    const float cx = px - 0.5f, cy = py - 0.5f, cz = pz - 0.5f;
    const float x0 = (px - 0.5f) - 0.5f, y1 = (py - 0.5f) - 0.5f, z2 = (pz - 0.5f) - 0.5f;
    auto emit = [&](int c, float u) {
        if (BLEND) {
            const float ut = bl.u_tilde ? bl.u_tilde[3 * i + c] : u;
            const float delta = u - ut;
            out[3 * i + c] = (bl.u_old[3 * i + c] + delta) * bl.alpha + u * (1.0f - bl.alpha);
        } else {
            out[3 * i + c] = u;
        }
    };
    const CornerBase b0 = corner_base(gx, x0, cy, cz), b1 = corner_base(gy, cx, y1, cz), b2 = corner_base(gz, cx, cy, z2);
    // a component whose samples in the whole warp are interior and cross no
    // block takes the one-block path (most of them, for Morton-sorted
    // particles); the 24 corner loads are issued before any lerp
    const unsigned am = __activemask();
    float c0[8], c1[8], c2[8];
    if (__all_sync(am, b0.ok && !(b0.crx || b0.cry || b0.crz))) corners_one_block(gx, b0, c0);
    else corners_general(gx, b0, c0);
    if (__all_sync(am, b1.ok && !(b1.crx || b1.cry || b1.crz))) corners_one_block(gy, b1, c1);
    else corners_general(gy, b1, c1);
    if (__all_sync(am, b2.ok && !(b2.crx || b2.cry || b2.crz))) corners_one_block(gz, b2, c2);
    else corners_general(gz, b2, c2);
    const bool ok0 = b0.ok, ok1 = b1.ok, ok2 = b2.ok;
    if (ok0) emit(0, lerp_corners(c0, b0));
    if (ok1) emit(1, lerp_corners(c1, b1));
    if (ok2) emit(2, lerp_corners(c2, b2));
    // the general gathers last, with little live across their calls
    if (!ok0) emit(0, sample_linear_boundary(gx, x0, cy, cz, bc));
    if (!ok1) emit(1, sample_linear_boundary(gy, cx, y1, cz, bc));
    if (!ok2) emit(2, sample_linear_boundary(gz, cx, cy, z2, bc));
}

// g2p_blend (fluid/g2p.rs:42-45), component-wise.
__global__ void g2p_blend_kernel(const float* u_old, const float* u, const float* ut, size_t n3, float alpha, float* out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
        const float delta = u[i] - ut[i];
        out[i] = (u_old[i] + delta) * alpha + u[i] * (1.0f - alpha);
    }
}

// MacGrid::normalize_velocity (mac.rs:106-132) over the given slots.
__global__ void normalize_kernel(float* vel, const float* mass, const int32_t* slots, size_t n, size_t be) {
    for (size_t k = blockIdx.x; k < n; k += gridDim.x) {
        const int32_t s = slots[k];
        if (s < 0) continue;
        float* v = vel + (size_t)s * be;
        const float* m = mass + (size_t)s * be;
        for (size_t i = threadIdx.x; i < be; i += blockDim.x) {
            const float mm = m[i];
            v[i] = mm > 0.0f ? v[i] / mm : 0.0f;
        }
    }
}

// MacGrid::divergence (mac.rs:137-171).  nb[k][0..3] = codes of the block
// itself and its -x, -y, -z neighbours in each channel (same block set).
struct DivArgs {
    const float* u[3];
    float* dst;
    int64_t nx, ny;
    int32_t sx, sy, sz;
    int lg;
    float empty, full;
};

__global__ void divergence_kernel(DivArgs a, const uint64_t* bids, const int32_t* codes, const int32_t* dst_slots, size_t n) {
    const int bsx = 1 << a.lg, mask = bsx - 1;
    const size_t be = (size_t)bsx * bsx * bsx;
    for (size_t k = blockIdx.x; k < n; k += gridDim.x) {
        const int32_t ds = dst_slots[k];
        if (ds < 0) continue;
        const uint64_t bid = bids[k];
        const int64_t bx = (int64_t)(bid % a.nx), by = (int64_t)((bid / a.nx) % a.ny), bz = (int64_t)(bid / (a.nx * a.ny));
        const int32_t gx0 = (int32_t)(bx * bsx), gy0 = (int32_t)(by * bsx), gz0 = (int32_t)(bz * bsx);
        const int32_t gx1 = min(gx0 + bsx, a.sx), gy1 = min(gy0 + bsx, a.sy), gz1 = min(gz0 + bsx, a.sz);
        const int32_t lx = gx1 - gx0, ly = gy1 - gy0, lz = gz1 - gz0;
        const int32_t* c = codes + k * 4;
        for (int i = threadIdx.x; i < lx * ly * lz; i += blockDim.x) {
            const int x = i % lx, y = (i / lx) % ly, z = i / (lx * ly);
            const int vid = x | (y << a.lg) | (z << (2 * a.lg));
            auto val = [&](int ch, int32_t code, int v) -> float {
                if (code >= 0) return a.u[ch][(size_t)code * be + v];
                return code == kCodeFull ? a.full : a.empty;
            };
            const float ux1 = val(0, c[0], vid);
            const float ux0 = (gx0 + x == 0) ? 0.0f
                              : x > 0 ? val(0, c[0], vid - 1) : val(0, c[1], (mask) | (y << a.lg) | (z << (2 * a.lg)));
            const float vy1 = val(1, c[0], vid);
            const float vy0 = (gy0 + y == 0) ? 0.0f
                              : y > 0 ? val(1, c[0], vid - bsx) : val(1, c[2], x | (mask << a.lg) | (z << (2 * a.lg)));
            const float wz1 = val(2, c[0], vid);
            const float wz0 = (gz0 + z == 0) ? 0.0f
                              : z > 0 ? val(2, c[0], vid - bsx * bsx) : val(2, c[3], x | (y << a.lg) | (mask << (2 * a.lg)));
            // The reference writes a compact running index over the in-domain
            // cells of the block (mac.rs:151-168).
            a.dst[(size_t)ds * be + i] = ((ux1 - ux0) + (vy1 - vy0)) + (wz1 - wz0);
        }
    }
}

// downsample_channel_avg (downsample.rs:13-59): coarse cell = mean of its 8
// children, summed z-major as the reference.
__global__ void downsample_kernel(const float* src, const int32_t* src_slots, float* dst, const int32_t* dst_slots, size_t n,
                                  int lg) {
    const int bsx = 1 << lg, bsc = bsx >> 1, clg = lg - 1;
    const size_t be = (size_t)bsx * bsx * bsx, bc = (size_t)bsc * bsc * bsc;
    for (size_t k = blockIdx.x; k < n; k += gridDim.x) {
        const float* sp = src + (size_t)src_slots[k] * be;
        float* dp = dst + (size_t)dst_slots[k] * bc;
        for (int i = threadIdx.x; i < (int)bc; i += blockDim.x) {
            const int cx = i & (bsc - 1), cy = (i >> clg) & (bsc - 1), cz = i >> (2 * clg);
            float sum = 0.0f;
            for (int dz = 0; dz < 2; ++dz)
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx)
                        sum += sp[(2 * cx + dx) | ((2 * cy + dy) << lg) | ((2 * cz + dz) << (2 * lg))];
            dp[i] = sum / 8.0f;
        }
    }
}

static unsigned grid_for(size_t n) { return (unsigned)std::min<size_t>(std::max<size_t>(div_up(n, 256), 1), 8192); }

// d_u_old non-null: the blended velocities (g2p_kernel<1>) instead of the samples.
void g2p_device(msbg_mac* m, const float* d_pos, size_t n, int bc, float* d_out, const float* d_u_old = nullptr,
                const float* d_u_tilde = nullptr, float alpha = 0.0f) {
    MSBG_REQUIRE(bc >= 0 && bc <= 2, "bad boundary condition");
    if (!n) return;
    SampleGrid gx = sample_grid(m->ch[0]), gy = sample_grid(m->ch[1]), gz = sample_grid(m->ch[2]);
    const BlendArgs bl{d_u_old, d_u_tilde, alpha};
    begin_launch(m->ctx);
    if (d_u_old) g2p_kernel<1><<<(unsigned)div_up(n, 256), 256, 0, m->ctx->stream>>>(gx, gy, gz, d_pos, n, bc, bl, d_out);
    else g2p_kernel<0><<<(unsigned)div_up(n, 256), 256, 0, m->ctx->stream>>>(gx, gy, gz, d_pos, n, bc, bl, d_out);
    after_launch(m->ctx, "g2p_kernel");
}

}  // namespace msbg

using namespace msbg;

extern "C" {

int msbg_mac_create(msbg_ctx* ctx, uint64_t sx, uint64_t sy, uint64_t sz, int bsx, msbg_mac** out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && out, "null argument");
    auto* m = new msbg_mac;
    m->ctx = ctx;
    for (int c = 0; c < 6; ++c) {
        int st = msbg_grid_create(ctx, sx, sy, sz, bsx, MSBG_F32, 0.0f, 0.0f, &m->ch[c]);
        if (st != MSBG_OK) {
            std::string msg = msbg_last_error();
            delete m;
            MSBG_THROW(st, msg);
        }
    }
    *out = m;
    MSBG_API_END
}

int msbg_mac_destroy(msbg_mac* m) {
    MSBG_API_BEGIN
    if (!m) return MSBG_OK;
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    delete m;
    MSBG_API_END
}

int msbg_mac_channel(msbg_mac* m, int which, msbg_grid** out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && out, "null argument");
    MSBG_REQUIRE(which >= 0 && which < 6, "channel index must be 0..5");
    *out = m->ch[which];
    MSBG_API_END
}

int msbg_mac_zero_blocks(msbg_mac* m, const uint64_t* bids, size_t n) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && (bids || !n), "null argument");
    set_device(m->ctx);
    std::vector<int32_t> slots(n);
    mac_ensure(m, bids, n, slots.data());
    if (n) {
        ScratchLayout L;
        size_t o = L.add<int32_t>(n);
        char* base = scratch(m->ctx, L);
        int32_t* d = ScratchLayout::at<int32_t>(base, o);
        CUDA_CHECK(cudaMemcpyAsync(d, slots.data(), n * 4, cudaMemcpyHostToDevice, m->ctx->stream));
        for (int c = 0; c < 6; ++c) grid_fill_slots(m->ch[c], d, n, 0.0f);
        sync(m->ctx);
    }
    MSBG_API_END
}

int msbg_mac_active_blocks(const msbg_mac* m, uint64_t* out, size_t cap, size_t* n_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && n_out, "null argument");
    for (size_t k = 0; k < m->active.size() && k < cap; ++k) out[k] = m->active[k];
    *n_out = m->active.size();
    MSBG_API_END
}

int msbg_mac_normalize_velocity(msbg_mac* m, const uint64_t* bids, size_t n) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && (bids || !n), "null argument");
    if (!n) return MSBG_OK;
    set_device(m->ctx);
    std::vector<int32_t> slots(n);
    for (size_t k = 0; k < n; ++k) {
        int32_t c = bids[k] < m->ch[0]->n_blocks ? grid_code(m->ch[0], bids[k]) : kCodeEmpty;
        slots[k] = c >= 0 ? c : -1;
    }
    ScratchLayout L;
    size_t o = L.add<int32_t>(n);
    char* base = scratch(m->ctx, L);
    int32_t* d = ScratchLayout::at<int32_t>(base, o);
    CUDA_CHECK(cudaMemcpyAsync(d, slots.data(), n * 4, cudaMemcpyHostToDevice, m->ctx->stream));
    for (int a = 0; a < 3; ++a) {
        begin_launch(m->ctx);
        normalize_kernel<<<(unsigned)std::min<size_t>(n, 65535), 256, 0, m->ctx->stream>>>(
            m->ch[a]->payload.as<float>(), m->ch[3 + a]->payload.as<float>(), d, n, m->ch[a]->block_elems);
        after_launch(m->ctx, "normalize_kernel");
    }
    sync(m->ctx);
    MSBG_API_END
}

int msbg_mac_divergence(msbg_mac* m, msbg_grid* dst, const uint64_t* active, size_t n) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && dst && (active || !n), "null argument");
    msbg_grid* u = m->ch[0];
    MSBG_REQUIRE(dst->dtype == MSBG_F32 && dst->bsx == u->bsx && dst->sx == u->sx && dst->sy == u->sy && dst->sz == u->sz,
                 "divergence target must be an f32 grid with the MAC grid's dims");
    if (!n) return MSBG_OK;
    set_device(m->ctx);
    std::vector<int32_t> dslots(n);
    grid_ensure(dst, active, n, dslots.data());
    std::vector<int32_t> codes(4 * n);
    for (size_t k = 0; k < n; ++k) {
        int64_t bx, by, bz;
        block_coords(u, active[k], &bx, &by, &bz);
        codes[4 * k + 0] = grid_code(u, active[k]);
        codes[4 * k + 1] = bx > 0 ? grid_code(u, active[k] - 1) : kCodeEmpty;
        codes[4 * k + 2] = by > 0 ? grid_code(u, active[k] - u->nx) : kCodeEmpty;
        codes[4 * k + 3] = bz > 0 ? grid_code(u, active[k] - u->nxy) : kCodeEmpty;
    }
    ScratchLayout L;
    size_t ob = L.add<uint64_t>(n), oc = L.add<int32_t>(4 * n), od = L.add<int32_t>(n);
    char* base = scratch(m->ctx, L);
    uint64_t* db = ScratchLayout::at<uint64_t>(base, ob);
    int32_t* dc = ScratchLayout::at<int32_t>(base, oc);
    int32_t* dd = ScratchLayout::at<int32_t>(base, od);
    CUDA_CHECK(cudaMemcpyAsync(db, active, n * 8, cudaMemcpyHostToDevice, m->ctx->stream));
    CUDA_CHECK(cudaMemcpyAsync(dc, codes.data(), 16 * n, cudaMemcpyHostToDevice, m->ctx->stream));
    CUDA_CHECK(cudaMemcpyAsync(dd, dslots.data(), 4 * n, cudaMemcpyHostToDevice, m->ctx->stream));
    DivArgs a;
    for (int c = 0; c < 3; ++c) a.u[c] = m->ch[c]->payload.as<float>();
    a.dst = dst->payload.as<float>();
    a.nx = (int64_t)u->nx; a.ny = (int64_t)u->ny;
    a.sx = (int32_t)u->sx; a.sy = (int32_t)u->sy; a.sz = (int32_t)u->sz;
    a.lg = u->lg;
    a.empty = u->empty_value;
    a.full = u->full_value;
    begin_launch(m->ctx);
    divergence_kernel<<<(unsigned)std::min<size_t>(n, 65535), 256, 0, m->ctx->stream>>>(a, db, dc, dd, n);
    after_launch(m->ctx, "divergence_kernel");
    sync(m->ctx);
    MSBG_API_END
}

int msbg_g2p_device(msbg_mac* m, const float* d_pos, size_t n, int bc, float* d_vel_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && ((d_pos && d_vel_out) || !n), "null argument");
    set_device(m->ctx);
    g2p_device(m, d_pos, n, bc, d_vel_out);
    MSBG_API_END
}

int msbg_g2p(msbg_mac* m, const float* pos, size_t n, int bc, float* vel_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && ((pos && vel_out) || !n), "null argument");
    if (!n) return MSBG_OK;
    set_device(m->ctx);
    DevBuf io;
    io.reserve(2 * ((n * 12 + 255) & ~size_t(255)));
    float* dp = io.as<float>();
    float* dv = (float*)((char*)io.p + ((n * 12 + 255) & ~size_t(255)));
    CUDA_CHECK(cudaMemcpyAsync(dp, pos, n * 12, cudaMemcpyHostToDevice, m->ctx->stream));
    g2p_device(m, dp, n, bc, dv);
    CUDA_CHECK(cudaMemcpyAsync(vel_out, dv, n * 12, cudaMemcpyDeviceToHost, m->ctx->stream));
    sync(m->ctx);
    MSBG_API_END
}

int msbg_g2p_flip_device(msbg_mac* m, const float* d_pos, size_t n, int bc, const float* d_u_old, const float* d_u_tilde,
                         float alpha, float* d_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && ((d_pos && d_u_old && d_out) || !n), "null argument");
    MSBG_REQUIRE(d_out != d_pos && d_out != d_u_old && d_out != d_u_tilde, "the output cannot alias an input");
    set_device(m->ctx);
    g2p_device(m, d_pos, n, bc, d_out, d_u_old, d_u_tilde, alpha);
    MSBG_API_END
}

int msbg_g2p_blend_device(msbg_ctx* ctx, const float* d_u_old, const float* d_u, const float* d_u_tilde, size_t n,
                          float alpha, float* d_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && ((d_u_old && d_u && d_u_tilde && d_out) || !n), "null argument");
    if (!n) return MSBG_OK;
    set_device(ctx);
    begin_launch(ctx);
    g2p_blend_kernel<<<grid_for(3 * n), 256, 0, ctx->stream>>>(d_u_old, d_u, d_u_tilde, 3 * n, alpha, d_out);
    after_launch(ctx, "g2p_blend_kernel");
    MSBG_API_END
}

int msbg_sample_linear(msbg_grid* g, const float* pos, size_t n, int align, int bc, float* out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && ((pos && out) || !n), "null argument");
    MSBG_REQUIRE(align == 0 || align == 1, "align must be 0 (Corner) or 1 (CellCentered)");
    MSBG_REQUIRE(bc >= 0 && bc <= 2, "bad boundary condition");
    if (!n) return MSBG_OK;
    set_device(g->ctx);
    SampleGrid s = sample_grid(g, true);
    ScratchLayout L;
    size_t op = L.add<float>(3 * n), oo = L.add<float>(n);
    char* base = scratch(g->ctx, L);
    float* dp = ScratchLayout::at<float>(base, op);
    float* dout = ScratchLayout::at<float>(base, oo);
    CUDA_CHECK(cudaMemcpyAsync(dp, pos, 12 * n, cudaMemcpyHostToDevice, g->ctx->stream));
    begin_launch(g->ctx);
    switch (g->dtype) {
        case MSBG_F32: sample_linear_kernel<ElemF32><<<grid_for(n), 256, 0, g->ctx->stream>>>(s, dp, n, align, bc, dout); break;
        case MSBG_U16: sample_linear_kernel<ElemU16><<<grid_for(n), 256, 0, g->ctx->stream>>>(s, dp, n, align, bc, dout); break;
        case MSBG_BF16: sample_linear_kernel<ElemBF16><<<grid_for(n), 256, 0, g->ctx->stream>>>(s, dp, n, align, bc, dout); break;
        case MSBG_U8: sample_linear_kernel<ElemU8><<<grid_for(n), 256, 0, g->ctx->stream>>>(s, dp, n, align, bc, dout); break;
        default: sample_linear_kernel<ElemF16><<<grid_for(n), 256, 0, g->ctx->stream>>>(s, dp, n, align, bc, dout); break;
    }
    after_launch(g->ctx, "sample_linear_kernel");
    CUDA_CHECK(cudaMemcpyAsync(out, dout, 4 * n, cudaMemcpyDeviceToHost, g->ctx->stream));
    sync(g->ctx);
    MSBG_API_END
}

static int sample_width(int mode) { return mode == 0 ? 1 : mode == 2 ? 6 : 3; }

int msbg_sample_ext_device(msbg_grid* g, const float* d_pos, size_t n, int mode, int align, int bc, float* d_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && ((d_pos && d_out) || !n), "null argument");
    MSBG_REQUIRE(mode >= 0 && mode <= 3, "mode must be 0 (cubic value), 1 (cubic gradient), 2 (Hessian) or 3 (trilinear gradient)");
    MSBG_REQUIRE(align == 0 || align == 1, "align must be 0 (Corner) or 1 (CellCentered)");
    MSBG_REQUIRE(bc >= 0 && bc <= 2, "bad boundary condition");
    MSBG_REQUIRE(g->bsx >= 4, "cubic sampling needs blocks of at least 4^3 cells");
    if (!n) return MSBG_OK;
    set_device(g->ctx);
    SampleGrid s = sample_grid(g, true);
    begin_launch(g->ctx);
    switch (g->dtype) {
        case MSBG_F32: sample_ext_kernel<ElemF32><<<grid_for(n), 128, 0, g->ctx->stream>>>(s, d_pos, n, mode, align, bc, d_out); break;
        case MSBG_U16: sample_ext_kernel<ElemU16><<<grid_for(n), 128, 0, g->ctx->stream>>>(s, d_pos, n, mode, align, bc, d_out); break;
        case MSBG_BF16: sample_ext_kernel<ElemBF16><<<grid_for(n), 128, 0, g->ctx->stream>>>(s, d_pos, n, mode, align, bc, d_out); break;
        case MSBG_U8: sample_ext_kernel<ElemU8><<<grid_for(n), 128, 0, g->ctx->stream>>>(s, d_pos, n, mode, align, bc, d_out); break;
        default: sample_ext_kernel<ElemF16><<<grid_for(n), 128, 0, g->ctx->stream>>>(s, d_pos, n, mode, align, bc, d_out); break;
    }
    after_launch(g->ctx, "sample_ext_kernel");
    MSBG_API_END
}

int msbg_sample_ext(msbg_grid* g, const float* pos, size_t n, int mode, int align, int bc, float* out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && ((pos && out) || !n), "null argument");
    MSBG_REQUIRE(mode >= 0 && mode <= 3, "mode must be 0 (cubic value), 1 (cubic gradient), 2 (Hessian) or 3 (trilinear gradient)");
    if (!n) return MSBG_OK;
    set_device(g->ctx);
    const int w = sample_width(mode);
    ScratchLayout L;
    size_t op = L.add<float>(3 * n), oo = L.add<float>((size_t)w * n);
    char* base = scratch(g->ctx, L);
    float* dp = ScratchLayout::at<float>(base, op);
    float* dout = ScratchLayout::at<float>(base, oo);
    CUDA_CHECK(cudaMemcpyAsync(dp, pos, 12 * n, cudaMemcpyHostToDevice, g->ctx->stream));
    const int st = msbg_sample_ext_device(g, dp, n, mode, align, bc, dout);
    if (st != MSBG_OK) MSBG_THROW(st, msbg_last_error());
    CUDA_CHECK(cudaMemcpyAsync(out, dout, 4 * (size_t)w * n, cudaMemcpyDeviceToHost, g->ctx->stream));
    sync(g->ctx);
    MSBG_API_END
}

int msbg_downsample_avg(msbg_grid* dst, msbg_grid* src) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(dst && src, "null argument");
    MSBG_REQUIRE(dst->dtype == MSBG_F32 && src->dtype == MSBG_F32, "downsample needs f32 levels");
    MSBG_REQUIRE(src->bsx >= 2 && dst->bsx * 2 == src->bsx && dst->nx == src->nx && dst->ny == src->ny && dst->nz == src->nz,
                 "dst must have half the block size of src on the same block grid");
    MSBG_REQUIRE(dst->ctx == src->ctx, "levels on different contexts");
    set_device(src->ctx);
    const size_t n = src->n_slots();
    if (!n) return MSBG_OK;
    std::vector<uint64_t> bids(src->slot_bid);
    std::vector<int32_t> sslots(n), dslots(n);
    for (size_t k = 0; k < n; ++k) sslots[k] = (int32_t)k;
    grid_ensure(dst, bids.data(), n, dslots.data());
    ScratchLayout L;
    size_t os = L.add<int32_t>(n), od = L.add<int32_t>(n);
    char* base = scratch(src->ctx, L);
    int32_t* ds = ScratchLayout::at<int32_t>(base, os);
    int32_t* dd = ScratchLayout::at<int32_t>(base, od);
    CUDA_CHECK(cudaMemcpyAsync(ds, sslots.data(), 4 * n, cudaMemcpyHostToDevice, src->ctx->stream));
    CUDA_CHECK(cudaMemcpyAsync(dd, dslots.data(), 4 * n, cudaMemcpyHostToDevice, src->ctx->stream));
    begin_launch(src->ctx);
    downsample_kernel<<<(unsigned)std::min<size_t>(n, 65535), 256, 0, src->ctx->stream>>>(
        src->payload.as<float>(), ds, dst->payload.as<float>(), dd, n, src->lg);
    after_launch(src->ctx, "downsample_kernel");
    sync(src->ctx);
    MSBG_API_END
}

}  // extern "C"
