// sweep.cu -- the fused halo-gather + stencil colour phase of the 8-colour
// in-place block smoother (solver.rs:141-267, multires/halo.rs:31-358,
// math/{laplacian,meancurv,bilaplacian}.rs).
//
// One CTA updates one block of the current colour: it stages the block and
// the part of its halo the stencil reads into shared memory (resolving the
// Neumann boundary and dequantising on the way), synchronises, then every
// thread walks one z-column of the block computing the stencil from shared
// memory and writes the result straight back into the block (in place, as
// StoreBack does).  Blocks of one colour never share a halo, so the CTAs of a
// phase are independent; the 8 phases of an iteration are consecutive kernels
// on one stream (block Gauss-Seidel across colours, Jacobi inside a block on
// the staged snapshot, exactly the reference's schedule).
//
// Arithmetic is the reference's operation by operation: this file is built
// with --fmad=false so `a*b+c` is never contracted, and fmaf() appears exactly
// where the reference calls mul_add.  Results are bit-identical to the CPU
// restatement in oracle/.
#include <algorithm>
#include <cstring>
#include <type_traits>

#include "sweep.cuh"

namespace msbg {

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// laplacian.rs:41-64 (7 taps)
__device__ __forceinline__ float stencil_laplacian(const float* h, int i, int dy, int dz, float dt, int clamp01) {
    float c = h[i], lx = h[i - 1], rx = h[i + 1], dyu = h[i - dy], dyd = h[i + dy], dzb = h[i - dz], dzf = h[i + dz];
    float nb = lx + rx;
    nb = nb + dyu;
    nb = nb + dyd;
    nb = nb + dzb;
    nb = nb + dzf;
    float lap = fmaf(c, -6.0f, nb);
    float fx = (rx - lx) * 0.5f, fy = (dyd - dyu) * 0.5f, fz = (dzf - dzb) * 0.5f;
    float g = sqrtf(fmaf(fx, fx, fmaf(fy, fy, fz * fz)));
    float nv = fmaf(dt * lap, g, c);
    return clamp01 ? clampf(nv, 0.0f, 1.0f) : nv;
}

// meancurv.rs:50-101 (19 taps)
__device__ __forceinline__ float stencil_meancurv(const float* h, int i, int dy, int dz, float dt, int clamp01) {
    float f0 = h[i], f1 = h[i - 1], f2 = h[i + 1], f3 = h[i - dy], f4 = h[i + dy], f5 = h[i - dz], f6 = h[i + dz];
    float fx = (f2 - f1) * 0.5f, fy = (f4 - f3) * 0.5f, fz = (f6 - f5) * 0.5f;
    float fxx = (f1 + f2) - 2.0f * f0, fyy = (f3 + f4) - 2.0f * f0, fzz = (f5 + f6) - 2.0f * f0;
    float d1 = h[i + 1 + dy], d2 = h[i + 1 - dy], d3 = h[i - 1 + dy], d4 = h[i - 1 - dy];
    float d5 = h[i + 1 + dz], d6 = h[i + 1 - dz], d7 = h[i - 1 + dz], d8 = h[i - 1 - dz];
    float d9 = h[i + dy + dz], d10 = h[i + dy - dz], d11 = h[i - dy + dz], d12 = h[i - dy - dz];
    float fyx = (((d1 - d2) - d3) + d4) * 0.25f;
    float fzx = (((d5 - d6) - d7) + d8) * 0.25f;
    float fzy = (((d9 - d10) - d11) + d12) * 0.25f;
    float cross = (fx * (fy * fyx) + fx * (fz * fzx)) + fy * (fz * fzy);
    float hnum = fmaf(fy * fy + fz * fz, fxx, fmaf(fx * fx + fz * fz, fyy, fmaf(fx * fx + fy * fy, fzz, -2.0f * cross)));
    float grad = fmaf(fx, fx, fmaf(fy, fy, fz * fz));
    float hc = grad > 1e-7f ? hnum / grad : 0.0f;
    float d = clampf(dt * hc, -0.1f, 0.1f);
    float nv = f0 + d;
    return clamp01 ? clampf(nv, 0.0f, 1.0f) : nv;
}

// bilaplacian.rs:45-92 (25 taps)
// bilaplacian.rs:40-90 on the 25 values: the centre f0, the face
// neighbours f1..f6 (x-, x+, y-, y+, z-, z+), the distance-2 neighbours g1..g6
// in the same order, and the 12 edge diagonals in the reference's order
// (x+y+, x+y-, x-y+, x-y-, x+z+, x+z-, x-z+, x-z-, y+z+, y+z-, y-z+, y-z-).
__device__ __forceinline__ float bilaplacian_values(float f0, float f1, float f2, float f3, float f4, float f5, float f6,
                                                    float g1, float g2, float g3, float g4, float g5, float g6,
                                                    const float (&e)[12], float dt, int clamp01) {
    float s1 = f1 + f2;
    s1 = s1 + f3; s1 = s1 + f4; s1 = s1 + f5; s1 = s1 + f6;
    float s2 = g1 + g2;
    s2 = s2 + g3; s2 = s2 + g4; s2 = s2 + g5; s2 = s2 + g6;
    float sd = e[0] + e[1];
#pragma unroll
    for (int k = 2; k < 12; ++k) sd = sd + e[k];
    float hv = ((42.0f * f0 - 12.0f * s1) + s2) + 2.0f * sd;
    float fx = (f2 - f1) * 0.5f, fy = (f4 - f3) * 0.5f, fz = (f6 - f5) * 0.5f;
    float g = sqrtf(fmaf(fx, fx, fmaf(fy, fy, fz * fz)));
    float upd = (dt * hv) * g;
    float d = clampf(-upd, -0.1f, 0.1f);
    float nv = f0 + d;
    return clamp01 ? clampf(nv, 0.0f, 1.0f) : nv;
}

__device__ __forceinline__ float stencil_bilaplacian(const float* h, int i, int dy, int dz, float dt, int clamp01) {
    const float e[12] = {h[i + 1 + dy], h[i + 1 - dy], h[i - 1 + dy], h[i - 1 - dy], h[i + 1 + dz], h[i + 1 - dz],
                         h[i - 1 + dz], h[i - 1 - dz], h[i + dy + dz], h[i + dy - dz], h[i - dy + dz], h[i - dy - dz]};
    return bilaplacian_values(h[i], h[i - 1], h[i + 1], h[i - dy], h[i + dy], h[i - dz], h[i + dz], h[i - 2], h[i + 2],
                              h[i - 2 * dy], h[i + 2 * dy], h[i - 2 * dz], h[i + 2 * dz], e, dt, clamp01);
}

struct SweepArgs {
    void* payload;              // fine payload (grid dtype)
    float* xface;               // [slots][2 XD][bsx^2] stored x-planes of every block ([z][y]), or null:
                                // x = 0 .. XD-1, then x = bsx-1 .. bsx-XD (XD = 2 for the 25-tap
                                // stencil's two-cell halo, else 1)
    const float* coarse;        // coarse payload (f32) for multiresolution halos
    const int32_t* nbr;         // [n][27]
    const int32_t* bxyz;        // [n][4]: block coords + flags (bit h-1: interior for halo h; bit 4 + k: neighbour k at the domain edge)
    int32_t sx, sy, sz;
    float empty, full, dt;
    int clamp01;
    // Density8 stores: lane seeds of the generator, the stream position of
    // this launch's plan index 0, log2 of the lane count and the generator
    // step over one z-plane of a block (16807^(bsx^2 / lanes))
    uint32_t sr_seed[16];
    uint64_t sr_base;
    uint32_t sr_zstep;
    int sr_lg;
};

template <int BSX> struct Lg { static constexpr int v = BSX == 4 ? 2 : BSX == 8 ? 3 : BSX == 16 ? 4 : 5; };

// Vector load of 4 consecutive stored elements as floats.
template <class E> struct Quad;
template <> struct Quad<ElemF32> {
    __device__ static float4 load(const float* p) { return *reinterpret_cast<const float4*>(p); }
};
template <> struct Quad<ElemU16> {
    __device__ static float4 load(const uint16_t* p) {
        const uint2 u = *reinterpret_cast<const uint2*>(p);
        return make_float4(ElemU16::load((uint16_t)(u.x & 0xffff)), ElemU16::load((uint16_t)(u.x >> 16)),
                           ElemU16::load((uint16_t)(u.y & 0xffff)), ElemU16::load((uint16_t)(u.y >> 16)));
    }
};
template <> struct Quad<ElemU8> {
    __device__ static float4 load(const uint8_t* p) {
        const uint32_t u = *reinterpret_cast<const uint32_t*>(p);
        return make_float4(ElemU8::load((uint8_t)(u & 0xff)), ElemU8::load((uint8_t)((u >> 8) & 0xff)),
                           ElemU8::load((uint8_t)((u >> 16) & 0xff)), ElemU8::load((uint8_t)(u >> 24)));
    }
};
template <> struct Quad<ElemF16> {
    __device__ static float4 load(const uint16_t* p) {
        const uint2 u = *reinterpret_cast<const uint2*>(p);
        return make_float4(ElemF16::load((uint16_t)(u.x & 0xffff)), ElemF16::load((uint16_t)(u.x >> 16)),
                           ElemF16::load((uint16_t)(u.y & 0xffff)), ElemF16::load((uint16_t)(u.y >> 16)));
    }
};
template <> struct Quad<ElemBF16> {
    __device__ static float4 load(const uint16_t* p) {
        const uint2 u = *reinterpret_cast<const uint2*>(p);
        return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u), __uint_as_float(u.y << 16),
                           __uint_as_float(u.y & 0xffff0000u));
    }
};

// Shared-memory layout of the staged halo block: rows of RS floats with the
// block's x = 0 at column 4 (16-byte aligned), HSX rows per plane.
template <int BSX> struct Stage { static constexpr int RS = BSX + 8; };

// Which staged cells a stencil reads: depth of a halo coordinate is 0 inside
// the block, 1 or 2 outside.
template <int ST> __device__ __forceinline__ bool row_needed(int dy, int dz) {
    if (ST == MSBG_LAPLACIAN) return dy == 0 || dz == 0;
    if (ST == MSBG_MEAN_CURVATURE) return true;
    return dy == 0 || dz == 0 || (dy == 1 && dz == 1);
}
template <int ST> __device__ __forceinline__ bool xhalo_needed(int dx, int dy, int dz) {
    if (ST == MSBG_LAPLACIAN) return dy == 0 && dz == 0;
    if (ST == MSBG_MEAN_CURVATURE) return (dy == 0 && dz == 0) || (dy + dz == 1);
    return (dy == 0 && dz == 0) || (dx == 1 && dy + dz == 1 && (dy == 1 || dz == 1));
}

// The stencil over one staged block: thread (x, y) walks its z-column, reads
// the staged values from shared memory, writes the result in place (and the
// block's new x-planes to the side buffer).
template <class E, int BSX, int ST>
__device__ __forceinline__ void sweep_compute(const SweepArgs& a, const float* __restrict__ h, int slot, int pi, int tid) {
    constexpr int HALO = ST == MSBG_BILAPLACIAN ? 2 : 1;
    constexpr int HSX = BSX + 2 * HALO;
    constexpr int RS = Stage<BSX>::RS;
    constexpr int PL = HSX * RS;
    constexpr int X0 = 4 - HALO;
    constexpr int N = BSX * BSX * BSX;
    typename E::T* payload = (typename E::T*)a.payload;
    if (tid < BSX * BSX) {
        // 16^3 blocks: each warp takes rows y and y + 2 of the plane, whose
        // shared-memory rows (pitch RS = 24 floats) fall on disjoint banks
        const int x = tid % BSX;
        const int y = BSX == 16 ? (((tid >> 6) << 2) | ((tid >> 5) & 1) | (((tid >> 4) & 1) << 1)) : tid / BSX;
        typename E::T* out = payload + (size_t)slot * N + x + y * BSX;
        // this block's new x-planes go to the side buffer as well
        constexpr int XD = ST == MSBG_BILAPLACIAN ? 2 : 1;
        float* xo = nullptr;
        if (a.xface && (x < XD || x >= BSX - XD))
            xo = a.xface + ((size_t)slot * 2 * XD + (x < XD ? x : XD + (BSX - 1 - x))) * (BSX * BSX) + y;
        const int i0 = (HALO * HSX + (y + HALO)) * RS + X0 + x + HALO;  // z = 0
        const float dt = a.dt;
        const int clamp01 = a.clamp01;
        // generator state of this thread's element at z = 0: the chunk of
        // element x + y*BSX + z*BSX^2 is that index >> sr_lg, its lane x's
        // low bits; each z step advances the chunk by BSX^2 >> sr_lg
        uint32_t st = 0, zs = 0;
        if constexpr (std::is_same<E, ElemU8>::value) {
            const uint64_t q0 = (uint64_t)((x + y * BSX) >> a.sr_lg);
            st = a.sr_seed[x & ((1 << a.sr_lg) - 1)] * sr_pow(a.sr_base + (uint64_t)pi * (uint64_t)(N >> a.sr_lg) + q0 + 1);
            zs = a.sr_zstep;
        }
        if (ST == MSBG_LAPLACIAN) {
            // taps along z slide through registers: 5 shared loads per output
            float zb = h[i0 - PL], c = h[i0], zf = h[i0 + PL];
#pragma unroll 4
            for (int z = 0; z < BSX; ++z) {
                const int i = i0 + z * PL;
                const float lx = h[i - 1], rx = h[i + 1], dyu = h[i - RS], dyd = h[i + RS];
                float nbs = lx + rx;
                nbs = nbs + dyu;
                nbs = nbs + dyd;
                nbs = nbs + zb;
                nbs = nbs + zf;
                const float lap = fmaf(c, -6.0f, nbs);
                const float fx = (rx - lx) * 0.5f, fy = (dyd - dyu) * 0.5f, fz = (zf - zb) * 0.5f;
                const float g = sqrtf(fmaf(fx, fx, fmaf(fy, fy, fz * fz)));
                const float nv = fmaf(dt * lap, g, c);
                const typename E::T sv = StoreBack<E>::store(clamp01 ? clampf(nv, 0.0f, 1.0f) : nv, st);
                st *= zs;
                out[z * BSX * BSX] = sv;
                if (xo) xo[z * BSX] = E::load(sv);
                zb = c;
                c = zf;
                if (z + 1 < BSX) zf = h[i + 2 * PL];
            }
        } else if (ST == MSBG_MEAN_CURVATURE) {
            // plane z-1: cross (c, x-, x+, y-, y+); plane z: 3x3; plane z+1: cross
            float pc = h[i0 - PL], pxm = h[i0 - PL - 1], pxp = h[i0 - PL + 1], pym = h[i0 - PL - RS], pyp = h[i0 - PL + RS];
            float c = h[i0], cxm = h[i0 - 1], cxp = h[i0 + 1], cym = h[i0 - RS], cyp = h[i0 + RS];
            float nc = h[i0 + PL], nxm = h[i0 + PL - 1], nxp = h[i0 + PL + 1], nym = h[i0 + PL - RS], nyp = h[i0 + PL + RS];
#pragma unroll 2
            for (int z = 0; z < BSX; ++z) {
                const int i = i0 + z * PL;
                const float xpyp = h[i + 1 + RS], xpym = h[i + 1 - RS], xmyp = h[i - 1 + RS], xmym = h[i - 1 - RS];
                // meancurv.rs:50-101 with f1..f6 = x-, x+, y-, y+, z-, z+
                const float f0 = c, f1 = cxm, f2 = cxp, f3 = cym, f4 = cyp, f5 = pc, f6 = nc;
                const float fx = (f2 - f1) * 0.5f, fy = (f4 - f3) * 0.5f, fz = (f6 - f5) * 0.5f;
                const float fxx = (f1 + f2) - 2.0f * f0, fyy = (f3 + f4) - 2.0f * f0, fzz = (f5 + f6) - 2.0f * f0;
                const float d1 = xpyp, d2 = xpym, d3 = xmyp, d4 = xmym;
                const float d5 = nxp, d6 = pxp, d7 = nxm, d8 = pxm;
                const float d9 = nyp, d10 = pyp, d11 = nym, d12 = pym;
                const float fyx = (((d1 - d2) - d3) + d4) * 0.25f;
                const float fzx = (((d5 - d6) - d7) + d8) * 0.25f;
                const float fzy = (((d9 - d10) - d11) + d12) * 0.25f;
                const float cross = (fx * (fy * fyx) + fx * (fz * fzx)) + fy * (fz * fzy);
                const float hnum = fmaf(fy * fy + fz * fz, fxx, fmaf(fx * fx + fz * fz, fyy, fmaf(fx * fx + fy * fy, fzz, -2.0f * cross)));
                const float grad = fmaf(fx, fx, fmaf(fy, fy, fz * fz));
                const float hc = grad > 1e-7f ? hnum / grad : 0.0f;
                const float d = clampf(dt * hc, -0.1f, 0.1f);
                const float nv = f0 + d;
                const typename E::T sv = StoreBack<E>::store(clamp01 ? clampf(nv, 0.0f, 1.0f) : nv, st);
                st *= zs;
                out[z * BSX * BSX] = sv;
                if (xo) xo[z * BSX] = E::load(sv);
                pc = c; pxm = cxm; pxp = cxp; pym = cym; pyp = cyp;
                c = nc; cxm = nxm; cxp = nxp; cym = nym; cyp = nyp;
                if (z + 1 < BSX) {
                    const int j = i + 2 * PL;
                    nc = h[j]; nxm = h[j - 1]; nxp = h[j + 1]; nym = h[j - RS]; nyp = h[j + RS];
                }
            }
        } else {
#pragma unroll 4
            for (int z = 0; z < BSX; ++z) {
                const int i = i0 + z * PL;
                const typename E::T sv = StoreBack<E>::store(stencil_bilaplacian(h, i, RS, PL, dt, clamp01), st);
                st *= zs;
                out[z * BSX * BSX] = sv;
                if (xo) xo[z * BSX] = E::load(sv);
            }
        }
    }
}

// General staging (blocks at the domain edge): resolve every staged
// coordinate with the Neumann rule (solver.rs:205-209).  ok/dd/ll are shared
// scratch arrays [3][HSX].
template <int BSX> struct Compact;

// CG: the block's neighbours may be updated by other CTAs of the same launch
// (sweep_wave_kernel), so their values are read through L2 (L1 is not
// coherent across SMs).
template <class E, int BSX, int ST, bool COMPACT = false, bool CG = false>
__device__ void stage_general(const SweepArgs& a, float* __restrict__ h, const int32_t* nb, int pi, int8_t* ok, int8_t* dd,
                              int8_t* ll) {
    constexpr int HALO = ST == MSBG_BILAPLACIAN ? 2 : 1;
    constexpr int HSX = BSX + 2 * HALO;
    constexpr int RS = Stage<BSX>::RS;
    constexpr int X0 = 4 - HALO;
    constexpr int LG = Lg<BSX>::v;
    constexpr int N = BSX * BSX * BSX;
    const typename E::T* payload = (const typename E::T*)a.payload;
    const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarp = nthr >> 5;
    // General path (blocks at the domain edge): resolve every staged
    // coordinate with the Neumann rule (solver.rs:205-209).
    for (int i = tid; i < 3 * HSX; i += nthr) {
        int ax = i / HSX, hh = i % HSX;
        int32_t smax = ax == 0 ? a.sx : ax == 1 ? a.sy : a.sz;
        int32_t b0 = a.bxyz[(size_t)pi * 4 + ax];
        int32_t g = b0 * BSX + hh - HALO, r;
        bool o = resolve_axis(g, smax - 1, MSBG_NEUMANN, &r);
        ok[ax * HSX + hh] = o;
        dd[ax * HSX + hh] = (int8_t)((r >> LG) - b0 + 1);
        ll[ax * HSX + hh] = (int8_t)(r & (BSX - 1));
    }
    __syncthreads();
    for (int r = warp; r < HSX * HSX; r += nwarp) {
        const int hz = r / HSX, hy = r % HSX;
        const bool midy = hy >= HALO && hy < HALO + BSX, midz = hz >= HALO && hz < HALO + BSX;
        for (int hx = lane; hx < HSX; hx += 32) {
            const bool midx = hx >= HALO && hx < HALO + BSX;
            const int nout = (!midx) + (!midy) + (!midz);
            bool need;
            if (ST == MSBG_LAPLACIAN) {
                need = nout <= 1;
            } else if (ST == MSBG_MEAN_CURVATURE) {
                need = nout <= 2;
            } else {
                const bool d1x = hx == HALO - 1 || hx == HALO + BSX, d1y = hy == HALO - 1 || hy == HALO + BSX,
                           d1z = hz == HALO - 1 || hz == HALO + BSX;
                need = nout <= 1 || (nout == 2 && (midx || d1x) && (midy || d1y) && (midz || d1z));
            }
            if (!need) continue;
            float v = a.empty;
            if (ok[hx] && ok[HSX + hy] && ok[2 * HSX + hz]) {
                const int c = nb[dd[hx] + 3 * dd[HSX + hy] + 9 * dd[2 * HSX + hz]];
                const int lx = ll[hx], ly = ll[HSX + hy], lz = ll[2 * HSX + hz];
                if (c >= 0) {
                    const typename E::T* src = payload + (size_t)c * N + (lx | (ly << LG) | (lz << (2 * LG)));
                    v = E::load(CG ? __ldcg(src) : *src);
                } else if (c == kCodeFull) {
                    v = a.full;
                } else if (c <= kCodeCoarse0) {
                    constexpr int CLG = LG - 1;
                    const int cs = kCodeCoarse0 - c;
                    v = a.coarse[(size_t)cs * (N / 8) + ((lx >> 1) | ((ly >> 1) << CLG) | ((lz >> 1) << (2 * CLG)))];
                }
            }
            if (COMPACT) h[Compact<BSX>::index(hx, hy, hz)] = v;
            else h[(hz * HSX + hy) * RS + X0 + hx] = v;
        }
    }
}

template <class E, int BSX, int ST>
__global__ void __launch_bounds__(BSX * BSX < 32 ? 32 : BSX * BSX, BSX == 16 && ST == MSBG_BILAPLACIAN ? 4 : 1)
sweep_phase_kernel(SweepArgs a, const int32_t* __restrict__ order, int n) {
    constexpr int HALO = ST == MSBG_BILAPLACIAN ? 2 : 1;
    constexpr int HSX = BSX + 2 * HALO;
    constexpr int RS = Stage<BSX>::RS;
    constexpr int X0 = 4 - HALO;  // column of halo x = 0
    constexpr int LG = Lg<BSX>::v;
    constexpr int N = BSX * BSX * BSX;
    constexpr int QR = BSX / 4;  // float4 quads per row
    extern __shared__ float4 h4[];
    float* h = reinterpret_cast<float*>(h4);
    __shared__ int32_t nb[27];
    __shared__ int32_t flags;
    __shared__ int8_t ok[3][HSX], dd[3][HSX], ll[3][HSX];
    typename E::T* payload = (typename E::T*)a.payload;
    const int tid = threadIdx.x, nthr = blockDim.x;

    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const int pi = order[t];
        __syncthreads();  // the previous block's compute is done with h
        if (tid < 27) nb[tid] = a.nbr[(size_t)pi * 27 + tid];
        if (tid == 32 || (nthr <= 32 && tid == 31)) flags = a.bxyz[(size_t)pi * 4 + 3];
        __syncthreads();
        const bool interior = (flags >> (HALO - 1)) & 1;
        if (interior) {
            // Fast path: the block and its needed halo lie inside the domain,
            // so every staged cell comes from one of the 27 neighbour slots
            // without boundary resolution.  Centre and face rows move as
            // 16-byte quads; all loads of a category are issued before its
            // shared-memory stores.
            constexpr int NT = BSX * BSX < 32 ? 32 : BSX * BSX;
            constexpr int NC4 = N / 4;
            constexpr int KC = (NC4 + NT - 1) / NT;
            const int c13 = nb[13];
            float4 vq[KC];
#pragma unroll
            for (int k = 0; k < KC; ++k) {
                const int it = tid + k * NT;
                if (it < NC4) vq[k] = Quad<E>::load(payload + (size_t)c13 * N + 4 * it);
            }
#pragma unroll
            for (int k = 0; k < KC; ++k) {
                const int it = tid + k * NT;
                if (it < NC4) {
                    const int q = it % QR, r = it / QR, y = r % BSX, z = r / BSX;
                    h4[(((z + HALO) * HSX + y + HALO) * RS + 4 + 4 * q) >> 2] = vq[k];
                }
            }
            // face rows: y and z planes at depth 1..HALO on both sides, and
            // (19/25 taps) the four x-edge rows at depth 1
            constexpr int NFACE = 4 * HALO * BSX * QR;
            constexpr int NEDGE = ST == MSBG_LAPLACIAN ? 0 : 4 * QR;
            constexpr int KF = (NFACE + NEDGE + NT - 1) / NT;
            float4 vf[KF];
            int df[KF];
#pragma unroll
            for (int k = 0; k < KF; ++k) {
                const int it = tid + k * NT;
                df[k] = -1;
                if (it < NFACE) {
                    const int q = it % QR, rr = it / QR;
                    const int row = rr % BSX, pd = rr / BSX;        // pd: plane descriptor
                    const int axis = pd / (2 * HALO), sd = pd % (2 * HALO);
                    const int side = sd < HALO ? -1 : 1, d = sd < HALO ? sd + 1 : sd - HALO + 1;
                    const int l = side < 0 ? BSX - d : d - 1;        // source coordinate
                    const int hh = side < 0 ? HALO - d : HALO + BSX - 1 + d;
                    int c, src, dst;
                    if (axis == 0) {  // y plane: rows over z
                        c = nb[13 + 3 * side];
                        src = (l << LG) + (row << (2 * LG));
                        dst = ((row + HALO) * HSX + hh) * RS + 4;
                    } else {          // z plane: rows over y
                        c = nb[13 + 9 * side];
                        src = (row << LG) + (l << (2 * LG));
                        dst = (hh * HSX + row + HALO) * RS + 4;
                    }
                    df[k] = dst + 4 * q;
                    if (c >= 0) {
                        vf[k] = Quad<E>::load(payload + (size_t)c * N + src + 4 * q);
                    } else if (c <= kCodeCoarse0) {
                        constexpr int CLG = LG > 0 ? LG - 1 : 0;
                        const int lx = 4 * q, ly = axis == 0 ? l : row, lz = axis == 0 ? row : l;
                        const float* cp = a.coarse + (size_t)(kCodeCoarse0 - c) * (N / 8) + ((ly >> 1) << CLG) + ((lz >> 1) << (2 * CLG));
                        vf[k] = make_float4(cp[lx >> 1], cp[(lx + 1) >> 1], cp[(lx + 2) >> 1], cp[(lx + 3) >> 1]);
                    } else {
                        const float f = c == kCodeFull ? a.full : a.empty;
                        vf[k] = make_float4(f, f, f, f);
                    }
                } else if (it < NFACE + NEDGE) {
                    const int e = it - NFACE, q = e % QR, corner = e / QR;
                    const int sy = (corner & 1) ? 1 : -1, sz = (corner & 2) ? 1 : -1;
                    const int ly = sy < 0 ? BSX - 1 : 0, lz = sz < 0 ? BSX - 1 : 0;
                    const int hy = sy < 0 ? HALO - 1 : HALO + BSX, hz = sz < 0 ? HALO - 1 : HALO + BSX;
                    const int c = nb[13 + 3 * sy + 9 * sz];
                    df[k] = (hz * HSX + hy) * RS + 4 + 4 * q;
                    if (c >= 0) {
                        vf[k] = Quad<E>::load(payload + (size_t)c * N + (ly << LG) + (lz << (2 * LG)) + 4 * q);
                    } else if (c <= kCodeCoarse0) {
                        constexpr int CLG = LG > 0 ? LG - 1 : 0;
                        const int lx = 4 * q;
                        const float* cp = a.coarse + (size_t)(kCodeCoarse0 - c) * (N / 8) + ((ly >> 1) << CLG) + ((lz >> 1) << (2 * CLG));
                        vf[k] = make_float4(cp[lx >> 1], cp[(lx + 1) >> 1], cp[(lx + 2) >> 1], cp[(lx + 3) >> 1]);
                    } else {
                        const float f = c == kCodeFull ? a.full : a.empty;
                        vf[k] = make_float4(f, f, f, f);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < KF; ++k)
                if (df[k] >= 0) h4[df[k] >> 2] = vf[k];
            // x-halo cells: the x planes at depth 1..HALO (rows over y, z) and
            // (19/25 taps) the y- and z-edges at x depth 1
            constexpr int NXF = 2 * HALO * BSX * BSX;
            constexpr int NXE = ST == MSBG_LAPLACIAN ? 0 : 8 * BSX;
            constexpr int KX = (NXF + NXE + NT - 1) / NT;
            float vx[KX];
            int dx[KX];
#pragma unroll
            for (int k = 0; k < KX; ++k) {
                const int it = tid + k * NT;
                dx[k] = -1;
                int c = kCodeEmpty, lx = 0, ly = 0, lz = 0;
                if (it < NXF) {
                    const int y = it % BSX, z = (it / BSX) % BSX, sd = it / (BSX * BSX);
                    const int side = sd < HALO ? -1 : 1, d = sd < HALO ? sd + 1 : sd - HALO + 1;
                    lx = side < 0 ? BSX - d : d - 1;
                    ly = y;
                    lz = z;
                    const int hx = side < 0 ? HALO - d : HALO + BSX - 1 + d;
                    c = nb[13 + side];
                    dx[k] = ((z + HALO) * HSX + y + HALO) * RS + X0 + hx;
                } else if (it < NXF + NXE) {
                    const int e = it - NXF, j = e % BSX, kind = e / BSX;  // kind 0..3: y-edges, 4..7: z-edges
                    const int sx = (kind & 1) ? 1 : -1, so = (kind & 2) ? 1 : -1;
                    lx = sx < 0 ? BSX - 1 : 0;
                    const int hx = sx < 0 ? HALO - 1 : HALO + BSX;
                    const int ho = so < 0 ? HALO - 1 : HALO + BSX, lo = so < 0 ? BSX - 1 : 0;
                    if (kind < 4) {  // edge along y at (x side, z side)
                        ly = j;
                        lz = lo;
                        c = nb[13 + sx + 9 * so];
                        dx[k] = (ho * HSX + j + HALO) * RS + X0 + hx;
                    } else {         // edge along z at (x side, y side)
                        ly = lo;
                        lz = j;
                        c = nb[13 + sx + 3 * so];
                        dx[k] = ((j + HALO) * HSX + ho) * RS + X0 + hx;
                    }
                }
                if (dx[k] >= 0) {
                    constexpr int XD = ST == MSBG_BILAPLACIAN ? 2 : 1;
                    if (c >= 0 && a.xface && (lx < XD || lx >= BSX - XD)) {
                        // x-plane cells from the side buffer: 16 contiguous
                        // floats per (z) row instead of one sector per cell
                        const int pl = lx < XD ? lx : XD + (BSX - 1 - lx);
                        vx[k] = a.xface[((size_t)c * 2 * XD + pl) * (BSX * BSX) + lz * BSX + ly];
                    } else if (c >= 0) {
                        vx[k] = E::load(payload[(size_t)c * N + lx + (ly << LG) + (lz << (2 * LG))]);
                    } else if (c <= kCodeCoarse0) {
                        constexpr int CLG = LG > 0 ? LG - 1 : 0;
                        vx[k] = a.coarse[(size_t)(kCodeCoarse0 - c) * (N / 8) + ((lx >> 1) | ((ly >> 1) << CLG) | ((lz >> 1) << (2 * CLG)))];
                    } else {
                        vx[k] = c == kCodeFull ? a.full : a.empty;
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < KX; ++k)
                if (dx[k] >= 0) h[dx[k]] = vx[k];
        } else {
            stage_general<E, BSX, ST>(a, h, nb, pi, &ok[0][0], &dd[0][0], &ll[0][0]);
        }
        __syncthreads();
        sweep_compute<E, BSX, ST>(a, h, nb[13], pi, tid);
    }
}

// ---- pipelined f32 sweep ------------------------------------------------------
// Persistent CTAs, two staging buffers: while a CTA computes one block, the
// cp.async copies of the next block it owns (interior blocks: centre, face
// rows, x-planes from the side buffer) are in flight into the other buffer,
// so staging latency overlaps the stencil instead of preceding it.  Blocks at
// the domain edge are staged synchronously by stage_general.  f32 grids only
// (cp.async copies bytes; the other storage types need dequantising).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int K> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(K) : "memory"); }

// Issues the staging of an interior block (flag bit HALO-1 set) into h.
template <int BSX, int ST>
__device__ __forceinline__ void issue_interior_f32(const SweepArgs& a, float* __restrict__ h, const int32_t* nb) {
    constexpr int HALO = ST == MSBG_BILAPLACIAN ? 2 : 1;
    constexpr int HSX = BSX + 2 * HALO;
    constexpr int RS = Stage<BSX>::RS;
    constexpr int X0 = 4 - HALO;
    constexpr int LG = Lg<BSX>::v;
    constexpr int N = BSX * BSX * BSX;
    constexpr int QR = BSX / 4;
    constexpr int NT = BSX * BSX < 32 ? 32 : BSX * BSX;
    const float* payload = (const float*)a.payload;
    const int tid = threadIdx.x;
    const int c13 = nb[13];
    for (int it = tid; it < N / 4; it += NT) {
        const int q = it % QR, r = it / QR, y = r % BSX, z = r / BSX;
        cp_async16(h + ((z + HALO) * HSX + y + HALO) * RS + 4 + 4 * q, payload + (size_t)c13 * N + 4 * it);
    }
    constexpr int NFACE = 4 * HALO * BSX * QR;
    constexpr int NEDGE = ST == MSBG_LAPLACIAN ? 0 : 4 * QR;
    for (int it = tid; it < NFACE + NEDGE; it += NT) {
        int c, dst, lyq, lzq, srcoff;
        if (it < NFACE) {
            const int q = it % QR, rr = it / QR;
            const int row = rr % BSX, pd = rr / BSX;
            const int axis = pd / (2 * HALO), sd = pd % (2 * HALO);
            const int side = sd < HALO ? -1 : 1, d = sd < HALO ? sd + 1 : sd - HALO + 1;
            const int l = side < 0 ? BSX - d : d - 1;
            const int hh = side < 0 ? HALO - d : HALO + BSX - 1 + d;
            if (axis == 0) {
                c = nb[13 + 3 * side];
                srcoff = (l << LG) + (row << (2 * LG)) + 4 * q;
                dst = ((row + HALO) * HSX + hh) * RS + 4 + 4 * q;
                lyq = l;
                lzq = row;
            } else {
                c = nb[13 + 9 * side];
                srcoff = (row << LG) + (l << (2 * LG)) + 4 * q;
                dst = (hh * HSX + row + HALO) * RS + 4 + 4 * q;
                lyq = row;
                lzq = l;
            }
        } else {
            const int e = it - NFACE, q = e % QR, corner = e / QR;
            const int sy = (corner & 1) ? 1 : -1, sz = (corner & 2) ? 1 : -1;
            lyq = sy < 0 ? BSX - 1 : 0;
            lzq = sz < 0 ? BSX - 1 : 0;
            const int hy = sy < 0 ? HALO - 1 : HALO + BSX, hz = sz < 0 ? HALO - 1 : HALO + BSX;
            c = nb[13 + 3 * sy + 9 * sz];
            dst = (hz * HSX + hy) * RS + 4 + 4 * q;
            srcoff = (lyq << LG) + (lzq << (2 * LG)) + 4 * q;
        }
        if (c >= 0) {
            cp_async16(h + dst, payload + (size_t)c * N + srcoff);
        } else if (c <= kCodeCoarse0) {
            constexpr int CLG = LG > 0 ? LG - 1 : 0;
            const int lx = srcoff & (BSX - 1);
            const float* cp = a.coarse + (size_t)(kCodeCoarse0 - c) * (N / 8) + ((lyq >> 1) << CLG) + ((lzq >> 1) << (2 * CLG));
            *reinterpret_cast<float4*>(h + dst) = make_float4(cp[lx >> 1], cp[(lx + 1) >> 1], cp[(lx + 2) >> 1], cp[(lx + 3) >> 1]);
        } else {
            const float f = c == kCodeFull ? a.full : a.empty;
            *reinterpret_cast<float4*>(h + dst) = make_float4(f, f, f, f);
        }
    }
    constexpr int NXF = 2 * HALO * BSX * BSX;
    constexpr int NXE = ST == MSBG_LAPLACIAN ? 0 : 8 * BSX;
    for (int it = tid; it < NXF + NXE; it += NT) {
        int c, lx, ly, lz, dst;
        if (it < NXF) {
            const int y = it % BSX, z = (it / BSX) % BSX, sd = it / (BSX * BSX);
            const int side = sd < HALO ? -1 : 1, d = sd < HALO ? sd + 1 : sd - HALO + 1;
            lx = side < 0 ? BSX - d : d - 1;
            ly = y;
            lz = z;
            const int hx = side < 0 ? HALO - d : HALO + BSX - 1 + d;
            c = nb[13 + side];
            dst = ((z + HALO) * HSX + y + HALO) * RS + X0 + hx;
        } else {
            const int e = it - NXF, j = e % BSX, kind = e / BSX;
            const int sx = (kind & 1) ? 1 : -1, so = (kind & 2) ? 1 : -1;
            lx = sx < 0 ? BSX - 1 : 0;
            const int hx = sx < 0 ? HALO - 1 : HALO + BSX;
            const int ho = so < 0 ? HALO - 1 : HALO + BSX, lo = so < 0 ? BSX - 1 : 0;
            if (kind < 4) {
                ly = j;
                lz = lo;
                c = nb[13 + sx + 9 * so];
                dst = (ho * HSX + j + HALO) * RS + X0 + hx;
            } else {
                ly = lo;
                lz = j;
                c = nb[13 + sx + 3 * so];
                dst = ((j + HALO) * HSX + ho) * RS + X0 + hx;
            }
        }
        constexpr int XD = ST == MSBG_BILAPLACIAN ? 2 : 1;
        if (c >= 0 && a.xface && (lx < XD || lx >= BSX - XD)) {
            const int pl = lx < XD ? lx : XD + (BSX - 1 - lx);
            cp_async4(h + dst, a.xface + ((size_t)c * 2 * XD + pl) * (BSX * BSX) + lz * BSX + ly);
        } else if (c >= 0) {
            cp_async4(h + dst, payload + (size_t)c * N + lx + (ly << LG) + (lz << (2 * LG)));
        } else if (c <= kCodeCoarse0) {
            constexpr int CLG = LG > 0 ? LG - 1 : 0;
            h[dst] = a.coarse[(size_t)(kCodeCoarse0 - c) * (N / 8) + ((lx >> 1) | ((ly >> 1) << CLG) | ((lz >> 1) << (2 * CLG)))];
        } else {
            h[dst] = c == kCodeFull ? a.full : a.empty;
        }
    }
}

template <int BSX, int ST>
__global__ void __launch_bounds__(BSX * BSX < 32 ? 32 : BSX * BSX)
sweep_pipe_kernel(SweepArgs a, const int32_t* __restrict__ order, int n) {
    constexpr int HALO = ST == MSBG_BILAPLACIAN ? 2 : 1;
    constexpr int HSX = BSX + 2 * HALO;
    constexpr int BUF = HSX * HSX * Stage<BSX>::RS;  // floats per staging buffer
    extern __shared__ float4 h4[];
    float* hb = reinterpret_cast<float*>(h4);
    __shared__ int32_t nbs[2][27];
    __shared__ int32_t flg[2], pis[2];
    __shared__ int8_t ok[3][HSX], dd[3][HSX], ll[3][HSX];
    const int tid = threadIdx.x, nthr = blockDim.x;
    int t = blockIdx.x;
    if (t >= n) return;
    auto meta = [&](int tt, int b) {
        const int pi = order[tt];
        if (tid < 27) nbs[b][tid] = a.nbr[(size_t)pi * 27 + tid];
        if (tid == nthr - 1) {
            flg[b] = a.bxyz[(size_t)pi * 4 + 3];
            pis[b] = pi;
        }
    };
    meta(t, 0);
    __syncthreads();
    if ((flg[0] >> (HALO - 1)) & 1) issue_interior_f32<BSX, ST>(a, hb, nbs[0]);
    cp_async_commit();
    for (int j = 0; t < n; t += gridDim.x, ++j) {
        const int b = j & 1, bn = b ^ 1;
        const int tn = t + gridDim.x;
        if (tn < n) meta(tn, bn);
        __syncthreads();  // nbs[bn] visible; every thread is done with buffer bn (the previous block)
        if (tn < n && ((flg[bn] >> (HALO - 1)) & 1)) issue_interior_f32<BSX, ST>(a, hb + bn * BUF, nbs[bn]);
        cp_async_commit();
        if ((flg[b] >> (HALO - 1)) & 1) cp_async_wait<1>();  // this block's copies have landed
        else stage_general<ElemF32, BSX, ST>(a, hb + b * BUF, nbs[b], pis[b], &ok[0][0], &dd[0][0], &ll[0][0]);
        __syncthreads();
        sweep_compute<ElemF32, BSX, ST>(a, hb + b * BUF, nbs[b][13], 0, tid);
    }
    cp_async_wait<0>();
}

// ---- compact staging layout (one-cell halos) -------------------------------
// Rows of BSX floats for the block and its y/z halo, [hz][hy][x] with hy, hz in
// 0..BSX+1 (halo coordinates) and x in 0..BSX-1; the x = -1 and x = BSX halo
// columns apart, [hz][4 + hy - 1] at a row pitch of XP floats, so that the
// BSX y-values of one z sit 16-byte aligned.  Two buffers of this size let
// 4 CTAs share an SM (the padded layout allows 3).
template <int BSX> struct Compact {
    static constexpr int H = BSX + 2;
    static constexpr int MAIN = H * H * BSX;  // floats
    static constexpr int XP = ((BSX + 2 + 3 + 3) / 4) * 4;  // x-halo row pitch: columns 3 .. BSX+4
    static constexpr int XS = H * XP;
    static constexpr int BUF = MAIN + 2 * XS;
    __device__ __forceinline__ static int index(int hx, int hy, int hz) {
        if (hx == 0) return MAIN + hz * XP + 3 + hy;
        if (hx == BSX + 1) return MAIN + XS + hz * XP + 3 + hy;
        return (hz * H + hy) * BSX + hx - 1;
    }
};

// Issues the staging of an interior block (one-cell halo) in the compact layout.
// SLAB: only the cells of halo planes hz0 .. hz1 (the z-slab of one CTA of a
// cluster that shares the block).
template <int BSX, int ST, int NT = BSX * BSX, bool CG = false, bool SLAB = false>
__device__ __forceinline__ void issue_compact(const SweepArgs& a, float* __restrict__ h, const int32_t* nb, int hz0 = 0,
                                              int hz1 = BSX + 1) {
    auto in = [&](int hz) { return !SLAB || (hz >= hz0 && hz <= hz1); };
    using CL = Compact<BSX>;
    constexpr int H = CL::H;
    constexpr int LG = Lg<BSX>::v;
    constexpr int N = BSX * BSX * BSX;
    constexpr int QR = BSX / 4;
    static_assert((N / 4) % NT == 0, "centre rows must split evenly over the threads");
    const float* payload = (const float*)a.payload;
    const int tid = threadIdx.x;
    const int c13 = nb[13];
    // centre rows
#pragma unroll
    for (int k = 0; k < N / 4 / NT; ++k) {
        const int it = tid + k * NT;
        const int q = it % QR, r = it / QR, y = r & (BSX - 1), z = r >> LG;
        if (in(z + 1)) cp_async16(h + ((z + 1) * H + y + 1) * BSX + 4 * q, payload + (size_t)c13 * N + 4 * it);
    }
    // y and z face rows (and the four x-edge rows of the 19-tap stencil)
    constexpr int NFACE = 4 * BSX * QR;
    constexpr int NEDGE = ST == MSBG_LAPLACIAN ? 0 : 4 * QR;
    for (int it = tid; it < NFACE + NEDGE; it += NT) {
        int c, dst, srcoff, ly, lz, hz;
        if (it < NFACE) {
            const int q = it % QR, rr = it / QR, row = rr % BSX, pd = rr / BSX;  // pd: y-, y+, z-, z+
            const int side = (pd & 1) ? 1 : -1, l = side < 0 ? BSX - 1 : 0, hh = side < 0 ? 0 : H - 1;
            if (pd < 2) {
                c = nb[13 + 3 * side];
                ly = l;
                lz = row;
                dst = ((row + 1) * H + hh) * BSX + 4 * q;
                hz = row + 1;
            } else {
                c = nb[13 + 9 * side];
                ly = row;
                lz = l;
                dst = (hh * H + row + 1) * BSX + 4 * q;
                hz = hh;
            }
            srcoff = (ly << LG) + (lz << (2 * LG)) + 4 * q;
        } else {
            const int e = it - NFACE, q = e % QR, corner = e / QR;
            const int sy = (corner & 1) ? 1 : -1, sz = (corner & 2) ? 1 : -1;
            ly = sy < 0 ? BSX - 1 : 0;
            lz = sz < 0 ? BSX - 1 : 0;
            c = nb[13 + 3 * sy + 9 * sz];
            dst = ((sz < 0 ? 0 : H - 1) * H + (sy < 0 ? 0 : H - 1)) * BSX + 4 * q;
            srcoff = (ly << LG) + (lz << (2 * LG)) + 4 * q;
            hz = sz < 0 ? 0 : H - 1;
        }
        if (!in(hz)) continue;
        if (c >= 0) {
            cp_async16(h + dst, payload + (size_t)c * N + srcoff);
        } else if (c <= kCodeCoarse0) {
            constexpr int CLG = LG - 1;
            const int lx = srcoff & (BSX - 1);
            const float* cp = a.coarse + (size_t)(kCodeCoarse0 - c) * (N / 8) + ((ly >> 1) << CLG) + ((lz >> 1) << (2 * CLG));
            *reinterpret_cast<float4*>(h + dst) = make_float4(cp[lx >> 1], cp[(lx + 1) >> 1], cp[(lx + 2) >> 1], cp[(lx + 3) >> 1]);
        } else {
            const float f = c == kCodeFull ? a.full : a.empty;
            *reinterpret_cast<float4*>(h + dst) = make_float4(f, f, f, f);
        }
    }
    // x-halo planes: BSX rows of BSX y-values per side, 16-byte copies from the
    // side buffer (x = BSX-1 plane of the -x neighbour, x = 0 plane of the +x one)
    constexpr int NXR = 2 * BSX * QR;
    for (int it = tid; it < NXR; it += NT) {
        const int q = it % QR, z = (it / QR) % BSX, side = it / (QR * BSX);  // side 0: x = -1, 1: x = BSX
        if (!in(z + 1)) continue;
        const int c = nb[13 + (side ? 1 : -1)];
        float* d = h + CL::MAIN + side * CL::XS + (z + 1) * CL::XP + 4 + 4 * q;
        if (c >= 0) {
            cp_async16(d, a.xface + ((size_t)c * 2 + (side ? 0 : 1)) * (BSX * BSX) + z * BSX + 4 * q);
        } else if (c <= kCodeCoarse0) {
            constexpr int CLG = LG - 1;
            const int lx = side ? 0 : BSX - 1;
            const float* cp = a.coarse + (size_t)(kCodeCoarse0 - c) * (N / 8) + ((lx >> 1) | ((z >> 1) << (2 * CLG)));
            float v[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = cp[((4 * q + j) >> 1) << CLG];
            *reinterpret_cast<float4*>(d) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
            const float f = c == kCodeFull ? a.full : a.empty;
            *reinterpret_cast<float4*>(d) = make_float4(f, f, f, f);
        }
    }
    if (ST != MSBG_LAPLACIAN) {
        // x-halo edges: along y at z = -1 / BSX (rows of the diagonal
        // neighbours' x-planes) and along z at y = -1 / BSX (strided)
        for (int it = tid; it < 4 * QR + 4 * BSX; it += NT) {
            if (it < 4 * QR) {
                const int q = it % QR, kind = it / QR;  // kind: x side (bit 0), z side (bit 1)
                const int sx = (kind & 1) ? 1 : -1, sz = (kind & 2) ? 1 : -1;
                const int c = nb[13 + sx + 9 * sz];
                const int lz = sz < 0 ? BSX - 1 : 0, hz = sz < 0 ? 0 : H - 1, side = sx < 0 ? 0 : 1;
                if (!in(hz)) continue;
                float* d = h + CL::MAIN + side * CL::XS + hz * CL::XP + 4 + 4 * q;
                if (c >= 0) {
                    cp_async16(d, a.xface + ((size_t)c * 2 + (sx < 0 ? 1 : 0)) * (BSX * BSX) + lz * BSX + 4 * q);
                } else if (c <= kCodeCoarse0) {
                    constexpr int CLG = LG - 1;
                    const int lx = sx < 0 ? BSX - 1 : 0;
                    const float* cp = a.coarse + (size_t)(kCodeCoarse0 - c) * (N / 8) + ((lx >> 1) | ((lz >> 1) << (2 * CLG)));
                    float v[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) v[j] = cp[((4 * q + j) >> 1) << CLG];
                    *reinterpret_cast<float4*>(d) = make_float4(v[0], v[1], v[2], v[3]);
                } else {
                    const float f = c == kCodeFull ? a.full : a.empty;
                    *reinterpret_cast<float4*>(d) = make_float4(f, f, f, f);
                }
            } else {
                const int e = it - 4 * QR, j = e % BSX, kind = e / BSX;  // x side (bit 0), y side (bit 1)
                const int sx = (kind & 1) ? 1 : -1, sy = (kind & 2) ? 1 : -1;
                const int c = nb[13 + sx + 3 * sy];
                const int ly = sy < 0 ? BSX - 1 : 0, hy = sy < 0 ? 0 : H - 1, side = sx < 0 ? 0 : 1;
                if (!in(j + 1)) continue;
                float* d = h + CL::MAIN + side * CL::XS + (j + 1) * CL::XP + 3 + hy;
                if (c >= 0) {
                    const float* src = a.xface + ((size_t)c * 2 + (sx < 0 ? 1 : 0)) * (BSX * BSX) + j * BSX + ly;
                    if (CG) *d = __ldcg(src);  // the 4-byte cp.async goes through L1
                    else cp_async4(d, src);
                } else if (c <= kCodeCoarse0) {
                    constexpr int CLG = LG - 1;
                    const int lx = sx < 0 ? BSX - 1 : 0;
                    *d = a.coarse[(size_t)(kCodeCoarse0 - c) * (N / 8) + ((lx >> 1) | ((ly >> 1) << CLG) | ((j >> 1) << (2 * CLG)))];
                } else {
                    *d = c == kCodeFull ? a.full : a.empty;
                }
            }
        }
    }
}

// The stencil over a block staged in the compact layout (thread (x, y) walks
// its z-column).  x-1 and x+1 come through per-thread accessors: from the
// block rows, or from the x-halo columns for x = 0 and x = BSX-1.
// ZS < BSX: only planes z0 .. z0 + ZS - 1 (the z-slab of one CTA of a
// cluster that shares the block; the slab's planes and one halo plane on
// either side are staged).
template <int BSX, int ST, bool CLAMP, int ZS = BSX>
__device__ __forceinline__ void compute_compact(const SweepArgs& a, const float* __restrict__ h, int slot, int tid,
                                                int z0_ = 0) {
    const int z0 = ZS == BSX ? 0 : z0_, z1 = z0 + ZS;
    using CL = Compact<BSX>;
    constexpr int H = CL::H;
    constexpr int RS = BSX, PL = H * BSX;
    constexpr int N = BSX * BSX * BSX;
    float* payload = (float*)a.payload;
    const int x = tid % BSX, y = tid / BSX;
    float* out = payload + (size_t)slot * N + x + y * BSX;
    float* xo = (x == 0 || x == BSX - 1) ? a.xface + ((size_t)slot * 2 + (x == 0 ? 0 : 1)) * (BSX * BSX) + y : nullptr;
    const int i0 = (1 * H + (y + 1)) * BSX + x;  // z = 0
    // left / right neighbour accessors: value at (x -+ 1, y + dy, z + dz) = p[(z + dz) * sz + dy * sy]
    const float* lp = x > 0 ? h + i0 - 1 : h + CL::MAIN + 1 * CL::XP + 3 + (y + 1);
    const float* rp = x < BSX - 1 ? h + i0 + 1 : h + CL::MAIN + CL::XS + 1 * CL::XP + 3 + (y + 1);
    const int lsz = x > 0 ? PL : CL::XP, lsy = x > 0 ? RS : 1;
    const int rsz = x < BSX - 1 ? PL : CL::XP, rsy = x < BSX - 1 ? RS : 1;
    const float dt = a.dt;
    if (ST == MSBG_LAPLACIAN) {
        float zb = h[i0 + (z0 - 1) * PL], c = h[i0 + z0 * PL], zf = h[i0 + (z0 + 1) * PL];
#pragma unroll 4
        for (int z = z0; z < z1; ++z) {
            const int i = i0 + z * PL;
            const float lx = lp[z * lsz], rx = rp[z * rsz], dyu = h[i - RS], dyd = h[i + RS];
            float nbs = lx + rx;
            nbs = nbs + dyu;
            nbs = nbs + dyd;
            nbs = nbs + zb;
            nbs = nbs + zf;
            const float lap = fmaf(c, -6.0f, nbs);
            const float fx = (rx - lx) * 0.5f, fy = (dyd - dyu) * 0.5f, fz = (zf - zb) * 0.5f;
            const float g = sqrtf(fmaf(fx, fx, fmaf(fy, fy, fz * fz)));
            float nv = fmaf(dt * lap, g, c);
            if (CLAMP) nv = clampf(nv, 0.0f, 1.0f);
            out[z * BSX * BSX] = nv;
            if (xo) xo[z * BSX] = nv;
            zb = c;
            c = zf;
            if (z + 1 < z1) zf = h[i + 2 * PL];
        }
    } else {
        // plane z-1: cross (c, x-, x+, y-, y+); plane z: 3x3; plane z+1: cross
        const int j0 = i0 + z0 * PL;
        float pc = h[j0 - PL], pxm = lp[(z0 - 1) * lsz], pxp = rp[(z0 - 1) * rsz], pym = h[j0 - PL - RS], pyp = h[j0 - PL + RS];
        float c = h[j0], cxm = lp[z0 * lsz], cxp = rp[z0 * rsz], cym = h[j0 - RS], cyp = h[j0 + RS];
        float nc = h[j0 + PL], nxm = lp[(z0 + 1) * lsz], nxp = rp[(z0 + 1) * rsz], nym = h[j0 + PL - RS], nyp = h[j0 + PL + RS];
#pragma unroll 2
        for (int z = z0; z < z1; ++z) {
            const int i = i0 + z * PL;
            const float xpyp = rp[z * rsz + rsy], xpym = rp[z * rsz - rsy], xmyp = lp[z * lsz + lsy], xmym = lp[z * lsz - lsy];
            // meancurv.rs:50-101 with f1..f6 = x-, x+, y-, y+, z-, z+
            const float f0 = c, f1 = cxm, f2 = cxp, f3 = cym, f4 = cyp, f5 = pc, f6 = nc;
            const float fx = (f2 - f1) * 0.5f, fy = (f4 - f3) * 0.5f, fz = (f6 - f5) * 0.5f;
            const float fxx = (f1 + f2) - 2.0f * f0, fyy = (f3 + f4) - 2.0f * f0, fzz = (f5 + f6) - 2.0f * f0;
            const float d1 = xpyp, d2 = xpym, d3 = xmyp, d4 = xmym;
            const float d5 = nxp, d6 = pxp, d7 = nxm, d8 = pxm;
            const float d9 = nyp, d10 = pyp, d11 = nym, d12 = pym;
            const float fyx = (((d1 - d2) - d3) + d4) * 0.25f;
            const float fzx = (((d5 - d6) - d7) + d8) * 0.25f;
            const float fzy = (((d9 - d10) - d11) + d12) * 0.25f;
            const float cross = (fx * (fy * fyx) + fx * (fz * fzx)) + fy * (fz * fzy);
            const float hnum = fmaf(fy * fy + fz * fz, fxx, fmaf(fx * fx + fz * fz, fyy, fmaf(fx * fx + fy * fy, fzz, -2.0f * cross)));
            const float grad = fmaf(fx, fx, fmaf(fy, fy, fz * fz));
            const float hc = grad > 1e-7f ? hnum / grad : 0.0f;
            const float d = clampf(dt * hc, -0.1f, 0.1f);
            float nv = f0 + d;
            if (CLAMP) nv = clampf(nv, 0.0f, 1.0f);
            out[z * BSX * BSX] = nv;
            if (xo) xo[z * BSX] = nv;
            pc = c; pxm = cxm; pxp = cxp; pym = cym; pyp = cyp;
            c = nc; cxm = nxm; cxp = nxp; cym = nym; cyp = nyp;
            if (z + 1 < z1) {
                const int j = i + 2 * PL;
                nc = h[j]; nxm = lp[(z + 2) * lsz]; nxp = rp[(z + 2) * rsz]; nym = h[j - RS]; nyp = h[j + RS];
            }
        }
    }
}

// Pairs of f32 in one 64-bit register and the paired IEEE single-precision
// operations of sm_100 (each half rounded as the scalar operation).  The
// stencil below feeds no paired product directly into a paired sum (the
// code generator may fuse such a pair even with .rn); its products go to
// explicit fused multiply-adds, as in the scalar form.
__device__ __forceinline__ uint64_t sw_pack(float a, float b) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void sw_unpack(uint64_t v, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ uint64_t sw_add(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ uint64_t sw_sub(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ uint64_t sw_mul(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ uint64_t sw_fma(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
__device__ __forceinline__ uint64_t sw_ld2(const float* p) { return *reinterpret_cast<const uint64_t*>(p); }

// The 7-tap stencil over a block staged in the compact layout, two
// x-columns per thread: thread (xp, y) walks columns x = 2 xp and x + 1 along
// z with paired arithmetic, the same operations in the same order per cell
// as compute_compact.  The pair's outer neighbours come from the block rows
// or, at x = 0 and x + 1 = BSX - 1, from the x-halo columns.
template <int BSX, bool CLAMP>
__device__ __forceinline__ void compute_compact_pair(const SweepArgs& a, const float* __restrict__ h, int slot, int tid) {
    using CL = Compact<BSX>;
    constexpr int H = CL::H;
    constexpr int RS = BSX, PL = H * BSX;
    constexpr int N = BSX * BSX * BSX;
    float* payload = (float*)a.payload;
    const int xp = tid % (BSX / 2), y = tid / (BSX / 2), x = 2 * xp;
    float* out = payload + (size_t)slot * N + x + y * BSX;
    float* xo0 = x == 0 ? a.xface + ((size_t)slot * 2 + 0) * (BSX * BSX) + y : nullptr;
    float* xo1 = x + 1 == BSX - 1 ? a.xface + ((size_t)slot * 2 + 1) * (BSX * BSX) + y : nullptr;
    const int i0 = (1 * H + (y + 1)) * BSX + x;  // z = 0, column x
    const float* lp = x > 0 ? h + i0 - 1 : h + CL::MAIN + 1 * CL::XP + 3 + (y + 1);
    const float* rp = x + 2 < BSX ? h + i0 + 2 : h + CL::MAIN + CL::XS + 1 * CL::XP + 3 + (y + 1);
    const int lsz = x > 0 ? PL : CL::XP, rsz = x + 2 < BSX ? PL : CL::XP;
    const uint64_t m6 = sw_pack(-6.0f, -6.0f), half = sw_pack(0.5f, 0.5f), dt2 = sw_pack(a.dt, a.dt);
    uint64_t zb = sw_ld2(h + i0 - PL), c = sw_ld2(h + i0), zf = sw_ld2(h + i0 + PL);
#pragma unroll 4
    for (int z = 0; z < BSX; ++z) {
        const int i = i0 + z * PL;
        float c0, c1;
        sw_unpack(c, c0, c1);
        const uint64_t lx = sw_pack(lp[z * lsz], c0), rx = sw_pack(c1, rp[z * rsz]);
        const uint64_t dyu = sw_ld2(h + i - RS), dyd = sw_ld2(h + i + RS);
        uint64_t nbs = sw_add(lx, rx);
        nbs = sw_add(nbs, dyu);
        nbs = sw_add(nbs, dyd);
        nbs = sw_add(nbs, zb);
        nbs = sw_add(nbs, zf);
        const uint64_t lap = sw_fma(c, m6, nbs);
        const uint64_t fx = sw_mul(sw_sub(rx, lx), half), fy = sw_mul(sw_sub(dyd, dyu), half), fz = sw_mul(sw_sub(zf, zb), half);
        float s0, s1;
        sw_unpack(sw_fma(fx, fx, sw_fma(fy, fy, sw_mul(fz, fz))), s0, s1);
        const uint64_t g = sw_pack(sqrtf(s0), sqrtf(s1));
        float n0, n1;
        sw_unpack(sw_fma(sw_mul(dt2, lap), g, c), n0, n1);
        if (CLAMP) {
            n0 = clampf(n0, 0.0f, 1.0f);
            n1 = clampf(n1, 0.0f, 1.0f);
        }
        *reinterpret_cast<float2*>(out + z * BSX * BSX) = make_float2(n0, n1);
        if (xo0) xo0[z * BSX] = n0;
        if (xo1) xo1[z * BSX] = n1;
        zb = c;
        c = zf;
        if (z + 1 < BSX) zf = sw_ld2(h + i + 2 * PL);
    }
}

// The 19-tap stencil over a block staged in the compact layout, two
// x-columns per thread with paired arithmetic: the same operations in the
// same order per cell as compute_compact (meancurv.rs:50-101).  Sums whose
// operands are products are formed in scalar arithmetic (the code generator
// may contract a paired product feeding a paired sum); 2 f0 is formed as
// f0 + f0, which is the same value.  For the pair (x, x + 1) the columns L =
// x - 1, A = x, B = x + 1 and R = x + 2 of a row give the x-neighbour pairs
// (L, A) and (B, R).
template <int BSX, bool CLAMP>
__device__ __forceinline__ void compute_compact_pair_mc(const SweepArgs& a, const float* __restrict__ h, int slot, int tid) {
    using CL = Compact<BSX>;
    constexpr int H = CL::H;
    constexpr int RS = BSX, PL = H * BSX;
    constexpr int N = BSX * BSX * BSX;
    float* payload = (float*)a.payload;
    const int xp = tid % (BSX / 2), y = tid / (BSX / 2), x = 2 * xp;
    float* out = payload + (size_t)slot * N + x + y * BSX;
    float* xo0 = x == 0 ? a.xface + ((size_t)slot * 2 + 0) * (BSX * BSX) + y : nullptr;
    float* xo1 = x + 1 == BSX - 1 ? a.xface + ((size_t)slot * 2 + 1) * (BSX * BSX) + y : nullptr;
    const int i0 = (1 * H + (y + 1)) * BSX + x;  // z = 0, column x
    // columns x - 1 and x + 2: block rows or x-halo columns
    const float* lp = x > 0 ? h + i0 - 1 : h + CL::MAIN + 1 * CL::XP + 3 + (y + 1);
    const float* rp = x + 2 < BSX ? h + i0 + 2 : h + CL::MAIN + CL::XS + 1 * CL::XP + 3 + (y + 1);
    const int lsz = x > 0 ? PL : CL::XP, lsy = x > 0 ? RS : 1;
    const int rsz = x + 2 < BSX ? PL : CL::XP, rsy = x + 2 < BSX ? RS : 1;
    const uint64_t half2 = sw_pack(0.5f, 0.5f), q2 = sw_pack(0.25f, 0.25f), m2 = sw_pack(-2.0f, -2.0f),
                   dt2 = sw_pack(a.dt, a.dt);
    auto lo = [](uint64_t v) { float p, q; sw_unpack(v, p, q); return p; };
    auto hi = [](uint64_t v) { float p, q; sw_unpack(v, p, q); return q; };
    // planes z - 1 (p), z (c), z + 1 (n): row y as L, (A, B), R; rows y - 1
    // and y + 1 as (A, B)
    float pL = lp[-lsz], pR = rp[-rsz], cL = lp[0], cR = rp[0], nL = lp[lsz], nR = rp[rsz];
    uint64_t pAB = sw_ld2(h + i0 - PL), pABm = sw_ld2(h + i0 - PL - RS), pABp = sw_ld2(h + i0 - PL + RS);
    uint64_t cAB = sw_ld2(h + i0), cABm = sw_ld2(h + i0 - RS), cABp = sw_ld2(h + i0 + RS);
    uint64_t nAB = sw_ld2(h + i0 + PL), nABm = sw_ld2(h + i0 + PL - RS), nABp = sw_ld2(h + i0 + PL + RS);
#pragma unroll 2
    for (int z = 0; z < BSX; ++z) {
        const int i = i0 + z * PL;
        // plane z's diagonal columns: L and R of rows y - 1 and y + 1
        const float cLm = lp[z * lsz - lsy], cLp = lp[z * lsz + lsy], cRm = rp[z * rsz - rsy], cRp = rp[z * rsz + rsy];
        // meancurv.rs:50-101 with f1..f6 = x-, x+, y-, y+, z-, z+
        const uint64_t f0 = cAB, f1 = sw_pack(cL, lo(cAB)), f2 = sw_pack(hi(cAB), cR);
        const uint64_t f3 = cABm, f4 = cABp, f5 = pAB, f6 = nAB;
        const uint64_t fx = sw_mul(sw_sub(f2, f1), half2), fy = sw_mul(sw_sub(f4, f3), half2),
                       fz = sw_mul(sw_sub(f6, f5), half2);
        const uint64_t two_f0 = sw_add(f0, f0);
        const uint64_t fxx = sw_sub(sw_add(f1, f2), two_f0), fyy = sw_sub(sw_add(f3, f4), two_f0),
                       fzz = sw_sub(sw_add(f5, f6), two_f0);
        // d1..d4: (x+1, y+1), (x+1, y-1), (x-1, y+1), (x-1, y-1) in plane z
        const uint64_t d1 = sw_pack(hi(cABp), cRp), d2 = sw_pack(hi(cABm), cRm), d3 = sw_pack(cLp, lo(cABp)),
                       d4 = sw_pack(cLm, lo(cABm));
        // d5..d8: (x+1, z+1), (x+1, z-1), (x-1, z+1), (x-1, z-1) in row y
        const uint64_t d5 = sw_pack(hi(nAB), nR), d6 = sw_pack(hi(pAB), pR), d7 = sw_pack(nL, lo(nAB)),
                       d8 = sw_pack(pL, lo(pAB));
        // d9..d12: (y+1, z+1), (y+1, z-1), (y-1, z+1), (y-1, z-1)
        const uint64_t fyx = sw_mul(sw_add(sw_sub(sw_sub(d1, d2), d3), d4), q2);
        const uint64_t fzx = sw_mul(sw_add(sw_sub(sw_sub(d5, d6), d7), d8), q2);
        const uint64_t fzy = sw_mul(sw_add(sw_sub(sw_sub(nABp, pABp), nABm), pABm), q2);
        // cross = (fx (fy fyx) + fx (fz fzx)) + fy (fz fzy): the inner
        // products paired, the outer products and their sums scalar
        const uint64_t i1 = sw_mul(fy, fyx), i2 = sw_mul(fz, fzx), i3 = sw_mul(fz, fzy);
        const float cr0 = (lo(fx) * lo(i1) + lo(fx) * lo(i2)) + lo(fy) * lo(i3);
        const float cr1 = (hi(fx) * hi(i1) + hi(fx) * hi(i2)) + hi(fy) * hi(i3);
        // squares paired, their sums scalar
        const uint64_t sx = sw_mul(fx, fx), sy = sw_mul(fy, fy), sz = sw_mul(fz, fz);
        const uint64_t syz = sw_pack(lo(sy) + lo(sz), hi(sy) + hi(sz)), sxz = sw_pack(lo(sx) + lo(sz), hi(sx) + hi(sz)),
                       sxy = sw_pack(lo(sx) + lo(sy), hi(sx) + hi(sy));
        const uint64_t hnum = sw_fma(syz, fxx, sw_fma(sxz, fyy, sw_fma(sxy, fzz, sw_mul(m2, sw_pack(cr0, cr1)))));
        const uint64_t grad = sw_fma(fx, fx, sw_fma(fy, fy, sw_mul(fz, fz)));
        const float g0 = lo(grad), g1 = hi(grad);
        const float hc0 = g0 > 1e-7f ? lo(hnum) / g0 : 0.0f, hc1 = g1 > 1e-7f ? hi(hnum) / g1 : 0.0f;
        float dd0, dd1;
        sw_unpack(sw_mul(dt2, sw_pack(hc0, hc1)), dd0, dd1);
        float n0, n1;
        sw_unpack(sw_add(f0, sw_pack(clampf(dd0, -0.1f, 0.1f), clampf(dd1, -0.1f, 0.1f))), n0, n1);
        if (CLAMP) {
            n0 = clampf(n0, 0.0f, 1.0f);
            n1 = clampf(n1, 0.0f, 1.0f);
        }
        *reinterpret_cast<float2*>(out + z * BSX * BSX) = make_float2(n0, n1);
        if (xo0) xo0[z * BSX] = n0;
        if (xo1) xo1[z * BSX] = n1;
        pL = cL; pR = cR; pAB = cAB; pABm = cABm; pABp = cABp;
        cL = nL; cR = nR; cAB = nAB; cABm = nABm; cABp = nABp;
        if (z + 1 < BSX) {
            const int j = i + 2 * PL;
            nL = lp[(z + 2) * lsz];
            nR = rp[(z + 2) * rsz];
            nAB = sw_ld2(h + j);
            nABm = sw_ld2(h + j - RS);
            nABp = sw_ld2(h + j + RS);
        }
    }
}

// Threads of a compact-sweep CTA: two columns per thread (PAIR) or one.
template <int BSX, int ST, bool PAIR = true> struct CompactThreads {
    static constexpr bool pair = PAIR && (ST == MSBG_LAPLACIAN || ST == MSBG_MEAN_CURVATURE) && BSX >= 8;
    static constexpr int v = pair ? BSX * BSX / 2 : BSX * BSX;
};

// The 19-tap stencil takes two columns per thread in colour phases of at
// least this many blocks (B200, 16^3 blocks: 10 sweeps of 56,056 blocks 9.2
// against 10.5 ms), one column otherwise: a phase of a few hundred blocks is
// bound by the latency of one block, which twice the threads shorten (776
// blocks: 0.87 against 0.99 ms).
constexpr int kPairMinPhaseBlocks = 1184;

template <int BSX, int ST, bool CLAMP, bool PAIR>
__global__ void __launch_bounds__(CompactThreads<BSX, ST, PAIR>::v, BSX == 16 ? 4 : 1)
sweep_compact_kernel(SweepArgs a, const int32_t* __restrict__ order, int n) {
    using CL = Compact<BSX>;
    extern __shared__ float4 h4[];
    float* hb = reinterpret_cast<float*>(h4);
    // block metadata in a ring of three slots: the neighbour codes and flags
    // of block t + 2 g are loaded into registers while block t is computed
    // and written to the ring after it, so their latency is hidden
    __shared__ int32_t nbs[3][27];
    __shared__ int32_t flg[3], pis[3];
    __shared__ int8_t ok[3][BSX + 2], dd[3][BSX + 2], ll[3][BSX + 2];
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int g = gridDim.x;
    int t = blockIdx.x;
    if (t >= n) return;
    const bool meta_thread = tid < 27 || tid == nthr - 1;
    auto load_meta = [&](int pi, int32_t& nbv, int32_t& flv) {
        if (tid < 27) nbv = a.nbr[(size_t)pi * 27 + tid];
        if (tid == nthr - 1) flv = a.bxyz[(size_t)pi * 4 + 3];
    };
    auto put_meta = [&](int sl, int pi, int32_t nbv, int32_t flv) {
        if (tid < 27) nbs[sl][tid] = nbv;
        if (tid == nthr - 1) {
            flg[sl] = flv;
            pis[sl] = pi;
        }
    };
    int pi2 = 0;
    if (meta_thread) {
        int32_t nbv = 0, flv = 0;
        const int pi0 = order[t];
        load_meta(pi0, nbv, flv);
        put_meta(0, pi0, nbv, flv);
        if (t + g < n) {
            const int pi1 = order[t + g];
            load_meta(pi1, nbv, flv);
            put_meta(1, pi1, nbv, flv);
        }
        if (t + 2 * g < n) pi2 = order[t + 2 * g];
    }
    __syncthreads();
    constexpr int NT = CompactThreads<BSX, ST, PAIR>::v;
    if (flg[0] & 1) issue_compact<BSX, ST, NT>(a, hb, nbs[0]);
    cp_async_commit();
    for (int j = 0; t < n; t += g, ++j) {
        const int sl = j % 3, sn = (j + 1) % 3, s2 = (j + 2) % 3;
        const int b = j & 1, bn = b ^ 1;
        const int tn = t + g, t2 = t + 2 * g, t3 = t + 3 * g;
        int32_t nb2 = 0, fl2 = 0;
        int pi3 = 0;
        if (meta_thread) {
            if (t2 < n) load_meta(pi2, nb2, fl2);
            if (t3 < n) pi3 = order[t3];
        }
        __syncthreads();  // slot sn visible; every thread is done with buffer bn (the previous block)
        if (tn < n && (flg[sn] & 1)) issue_compact<BSX, ST, NT>(a, hb + bn * CL::BUF, nbs[sn]);
        cp_async_commit();
        if (flg[sl] & 1) cp_async_wait<1>();  // this block's copies have landed
        else stage_general<ElemF32, BSX, ST, true>(a, hb + b * CL::BUF, nbs[sl], pis[sl], &ok[0][0], &dd[0][0], &ll[0][0]);
        __syncthreads();
        if (CompactThreads<BSX, ST, PAIR>::pair && ST == MSBG_LAPLACIAN) compute_compact_pair<BSX, CLAMP>(a, hb + b * CL::BUF, nbs[sl][13], tid);
        else if (CompactThreads<BSX, ST, PAIR>::pair) compute_compact_pair_mc<BSX, CLAMP>(a, hb + b * CL::BUF, nbs[sl][13], tid);
        else compute_compact<BSX, ST, CLAMP>(a, hb + b * CL::BUF, nbs[sl][13], tid);
        if (meta_thread && t2 < n) put_meta(s2, pi2, nb2, fl2);
        pi2 = pi3;
    }
    cp_async_wait<0>();
}

// ---- one-launch sweeps for small active sets -------------------------------
// Every colour phase of every sweep of a call in one launch.  Items are
// (sweep t, block) pairs.  A block of colour c reads its neighbours of lower
// colours after their update in sweep t and those of higher colours before
// it (the crate's colour order, solver.rs:187-217), so item (t, b) waits
// until every neighbour it reads or is read by has completed t + 1 sweeps
// (lower colour) or t sweeps (higher colour), and b itself t sweeps:
// per-slot progress words, each published after the block's stores.  The
// host orders the items by (k = 8 t + c + bz, higher bz first, colour-major
// Morton rank): every item an item waits for comes strictly earlier in that
// order (a dependency at the same or a lower block layer has a smaller k; one
// a layer up has k at most equal, and then comes first by its layer), and
// CTAs claim items from a counter in that order, so a waiting item only waits
// for items already claimed by running CTAs.  The CTAs flow from phase to
// phase without the launch gap and tail of a kernel per phase, which is what
// bounds a phase of a few hundred blocks.  (On large sets the chain of
// dependent phases inside each block layer makes it slower than a kernel per
// phase, whose next block's staging always overlaps the current stencil.)
// The next item's staging is issued while the current block is computed when
// its neighbours are already done, else after the current block is
// published.  Blocks other CTAs update are read through L2.  A wait that runs
// past kWaitLimitNs sets bit 8 of the status word, and every CTA stops at its
// next wait once the bit is set (after its copies in flight have landed); the
// sweep is then incomplete and the next call that reads the status word
// reports it.

// Neighbours (of the 27) a stencil's halo reads: faces for the 7-tap stencil,
// faces and edges for the 19- and 25-tap ones.
template <int ST> __device__ __forceinline__ bool reads_neighbour(int k) {
    const int nout = (k % 3 != 1) + ((k / 3) % 3 != 1) + (k / 9 != 1);
    return ST == MSBG_LAPLACIAN ? nout == 1 : (nout == 1 || nout == 2);
}

template <int BSX, int ST, bool CLAMP>
__global__ void __launch_bounds__(CompactThreads<BSX, ST>::v, BSX == 16 ? 4 : 1)
sweep_wave_kernel(SweepArgs a, const int2* __restrict__ items, int total, int* prog, unsigned int* counter, int* status) {
    using CL = Compact<BSX>;
    constexpr int NT = CompactThreads<BSX, ST>::v;
    extern __shared__ float4 h4[];
    float* hb = reinterpret_cast<float*>(h4);
    __shared__ int32_t nbs[2][27];
    __shared__ int32_t flg[2], pis[2], col[2], swp[2];
    __shared__ int itm[2];
    __shared__ int8_t ok[3][BSX + 2], dd[3][BSX + 2], ll[3][BSX + 2];
    __shared__ int s_stop;
    const int tid = threadIdx.x;
    auto claim = [&](int b) {
        if (tid == 0) itm[b] = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int w = itm[b];
        if (w < total) {
            const int2 it = items[w];
            if (tid < 27) nbs[b][tid] = a.nbr[(size_t)it.y * 27 + tid];
            if (tid == NT - 1) {
                const int32_t* bx = a.bxyz + (size_t)it.y * 4;
                flg[b] = bx[3];
                pis[b] = it.y;
                swp[b] = it.x;
                col[b] = (bx[0] & 1) | ((bx[1] & 1) << 1) | ((bx[2] & 1) << 2);
            }
        }
        __syncthreads();
    };
    // every swept neighbour the block reads or is read by, and the block
    // itself, has completed the sweeps item b needs: the neighbours the
    // stencil reads, and any of the 26 when either block lies at the domain
    // edge (the Neumann rule may reflect an edge block's halo into a diagonal
    // neighbour, which must then also wait for it)
    auto ready = [&](int b) -> bool {
        bool good = true;
        const int fl = flg[b];
        if (tid < 27 && (tid == 13 || !(fl & 1) || ((fl >> (4 + tid)) & 1) || reads_neighbour<ST>(tid))) {
            const int c = nbs[b][tid];
            if (c >= 0) {
                const int nc = col[b] ^ ((tid % 3 != 1) | (((tid / 3) % 3 != 1) << 1) | ((tid / 9 != 1) << 2));
                const int need = nc < col[b] ? swp[b] + 1 : swp[b];
                good = *(volatile int*)(prog + c) >= need;
            }
        }
        __threadfence();
        return __syncthreads_and(good) != 0;
    };
    // false: a wait gave up (here or in another CTA); the kernel then stops
    auto wait_ready = [&](int b) -> bool {
        uint64_t t0 = 0;
        for (uint32_t spins = 0;; ++spins) {
            if (ready(b)) return true;
            if (tid == 0) {
                int stop = (*(volatile int*)status & 8) ? 1 : 0;
                if (!stop && (spins & 15u) == 15u) {
                    const uint64_t now = globaltimer_ns();
                    if (!t0) t0 = now;
                    else if (now - t0 > kWaitLimitNs) {
                        atomicOr(status, 8);
                        stop = 1;
                    }
                }
                s_stop = stop;
            }
            __syncthreads();
            if (s_stop) return false;
            __nanosleep(64);
        }
    };
    auto stage = [&](int b) {  // issues (interior) or performs (edge) the staging of item b into buffer b
        if (flg[b] & 1) issue_compact<BSX, ST, NT, true>(a, hb + b * CL::BUF, nbs[b]);
        else stage_general<ElemF32, BSX, ST, true, true>(a, hb + b * CL::BUF, nbs[b], pis[b], &ok[0][0], &dd[0][0], &ll[0][0]);
        cp_async_commit();
    };
    claim(0);
    if (itm[0] >= total) return;
    if (!wait_ready(0)) return;
    stage(0);
    int b = 0;
    while (true) {
        const int bn = b ^ 1;
        claim(bn);
        const bool more = itm[bn] < total;
        bool early = false;
        if (more && ready(bn)) {
            stage(bn);
            early = true;
        } else {
            cp_async_commit();  // an empty group keeps the wait count uniform
        }
        cp_async_wait<1>();  // the current block's copies have landed
        __syncthreads();
        if (CompactThreads<BSX, ST>::pair && ST == MSBG_LAPLACIAN) compute_compact_pair<BSX, CLAMP>(a, hb + b * CL::BUF, nbs[b][13], tid);
        else if (CompactThreads<BSX, ST>::pair) compute_compact_pair_mc<BSX, CLAMP>(a, hb + b * CL::BUF, nbs[b][13], tid);
        else compute_compact<BSX, ST, CLAMP>(a, hb + b * CL::BUF, nbs[b][13], tid);
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicExch(prog + nbs[b][13], swp[b] + 1);
        }
        if (!more) break;
        if (!early) {
            if (!wait_ready(bn)) break;  // nothing of bn is in flight
            stage(bn);
        }
        b = bn;
    }
    cp_async_wait<0>();
}

// Progress words of a wave sweep: INT_MAX for every slot (blocks that are
// not swept never hold anything up), then 0 for the swept blocks.
__global__ void wave_init_kernel(int* prog, size_t n_slots, unsigned int* counter) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n_slots; i += (size_t)gridDim.x * blockDim.x)
        prog[i] = 0x7fffffff;
    if (blockIdx.x == 0 && threadIdx.x == 0) *counter = 0u;
}
__global__ void wave_zero_kernel(int* prog, const int32_t* __restrict__ nbr, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) prog[nbr[(size_t)i * 27 + 13]] = 0;
}

// Copies the outer x-planes (x = 0 .. xd-1 and x = bsx-1 .. bsx-xd) of the
// listed slots into the side buffer: [slot][plane][z][y].
template <class E, int BSX>
__global__ void xface_init_kernel(const typename E::T* __restrict__ payload, const int32_t* __restrict__ slots, size_t n,
                                  int xd, float* __restrict__ xface) {
    constexpr int LG = Lg<BSX>::v, N = BSX * BSX * BSX, P = BSX * BSX;
    const size_t per = (size_t)2 * xd * P;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n * per; e += (size_t)gridDim.x * blockDim.x) {
        const size_t k = e / per;
        const int r = (int)(e % per), pl = r / P, zy = r % P, z = zy / BSX, y = zy % BSX;
        const int32_t slot = slots[k];
        const int x = pl < xd ? pl : BSX - 1 - (pl - xd);
        xface[((size_t)slot * 2 * xd + pl) * P + zy] = E::load(payload[(size_t)slot * N + x + (y << LG) + (z << (2 * LG))]);
    }
}

template <class E, int BSX>
static void launch_xface_init(msbg_ctx* ctx, const void* payload, const int32_t* slots, size_t n, int xd, float* xface) {
    if (!n) return;
    begin_launch(ctx);
    xface_init_kernel<E, BSX><<<(unsigned)std::min<size_t>((n * 2 * xd * BSX * BSX + 255) / 256, 148 * 32), 256, 0, ctx->stream>>>(
        (const typename E::T*)payload, slots, n, xd, xface);
    after_launch(ctx, "xface_init_kernel");
}

template <class E>
static void xface_init(msbg_ctx* ctx, int bsx, const void* payload, const int32_t* slots, size_t n, int xd, float* xface) {
    switch (bsx) {
        case 4: launch_xface_init<E, 4>(ctx, payload, slots, n, xd, xface); break;
        case 8: launch_xface_init<E, 8>(ctx, payload, slots, n, xd, xface); break;
        case 16: launch_xface_init<E, 16>(ctx, payload, slots, n, xd, xface); break;
        default: launch_xface_init<E, 32>(ctx, payload, slots, n, xd, xface); break;
    }
}

// ---- small colour phases: one block per thread-block cluster ---------------
// A phase of a few hundred blocks leaves most SMs idle with one CTA per
// block and takes one block's latency.  Here a cluster of BSX / ZS CTAs
// shares a block: each stages the planes of its z-slab (and one halo plane
// on either side), the cluster barrier orders every CTA's reads of the block
// before any CTA's in-place writes (the stencil reads the block's values from
// before the phase, as with one CTA), and each computes its ZS planes.
__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <int BSX, int ST, bool CLAMP, int ZS>
__global__ void __launch_bounds__(BSX * BSX) sweep_cluster_kernel(SweepArgs a, const int32_t* __restrict__ order, int n) {
    using CL = Compact<BSX>;
    constexpr int NS = BSX / ZS;  // CTAs of a cluster, one block
    extern __shared__ float4 h4[];
    float* hb = reinterpret_cast<float*>(h4);
    __shared__ int32_t nbs[27];
    __shared__ int32_t flg, pis;
    __shared__ int8_t ok[3][BSX + 2], dd[3][BSX + 2], ll[3][BSX + 2];
    const int tid = threadIdx.x;
    const int t = blockIdx.x / NS, z0 = (int)(blockIdx.x % NS) * ZS;
    const int pi = order[t];
    if (tid < 27) nbs[tid] = a.nbr[(size_t)pi * 27 + tid];
    if (tid == BSX * BSX - 1) {
        flg = a.bxyz[(size_t)pi * 4 + 3];
        pis = pi;
    }
    __syncthreads();
    if (flg & 1) {
        issue_compact<BSX, ST, BSX * BSX, false, true>(a, hb, nbs, z0, z0 + ZS + 1);
        cp_async_commit();
        cp_async_wait<0>();
    } else {
        stage_general<ElemF32, BSX, ST, true>(a, hb, nbs, pis, &ok[0][0], &dd[0][0], &ll[0][0]);
    }
    __syncthreads();
    cluster_barrier();  // every CTA of the block has read it
    compute_compact<BSX, ST, CLAMP, ZS>(a, hb, nbs[13], tid, z0);
}

// Colour phases of at most this many blocks run one block per cluster of 4
// CTAs (16^3 blocks, one-cell halos).
constexpr int kClusterMaxPhaseBlocks = 296;

template <int BSX, int ST, bool CLAMP>
static void launch_cluster(msbg_ctx* ctx, const SweepArgs& a, const int32_t* order, int n) {
    constexpr int ZS = 4, NS = BSX / ZS;
    const size_t smem = sizeof(float) * Compact<BSX>::BUF;
    static bool attr = false;
    if (!attr) {
        CUDA_CHECK(cudaFuncSetAttribute(sweep_cluster_kernel<BSX, ST, CLAMP, ZS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
        attr = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(n * NS));
    cfg.blockDim = dim3(BSX * BSX);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = NS;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    begin_launch(ctx);
    CUDA_CHECK(cudaLaunchKernelEx(&cfg, sweep_cluster_kernel<BSX, ST, CLAMP, ZS>, a, order, n));
    after_launch(ctx, "sweep_cluster_kernel");
}

template <int BSX, int ST, bool CLAMP, bool PAIR>
static void launch_compact_v(msbg_ctx* ctx, const SweepArgs& a, const int32_t* order, int n) {
    const size_t smem = 2 * sizeof(float) * Compact<BSX>::BUF;
    static bool attr = false;
    if (!attr) {
        CUDA_CHECK(cudaFuncSetAttribute(sweep_compact_kernel<BSX, ST, CLAMP, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
        CUDA_CHECK(cudaFuncSetAttribute(sweep_compact_kernel<BSX, ST, CLAMP, PAIR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)cudaSharedmemCarveoutMaxShared));
        attr = true;
    }
    const int threads = CompactThreads<BSX, ST, PAIR>::v;
    int per_sm = 0;
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_compact_kernel<BSX, ST, CLAMP, PAIR>, threads, smem));
    int sms = 0;
    CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    const int grid = std::max(1, std::min(n, std::max(per_sm, 1) * sms));
    begin_launch(ctx);
    sweep_compact_kernel<BSX, ST, CLAMP, PAIR><<<(unsigned)grid, threads, smem, ctx->stream>>>(a, order, n);
    after_launch(ctx, "sweep_compact_kernel");
}

template <int BSX, int ST, bool CLAMP>
static void launch_compact(msbg_ctx* ctx, const SweepArgs& a, const int32_t* order, int n) {
    if constexpr (ST == MSBG_LAPLACIAN) {
        launch_compact_v<BSX, ST, CLAMP, true>(ctx, a, order, n);
    } else {
        if (n >= kPairMinPhaseBlocks) {
            launch_compact_v<BSX, ST, CLAMP, true>(ctx, a, order, n);
            return;
        }
        if constexpr (BSX == 16 && ST == MSBG_MEAN_CURVATURE) {
            if (n <= kClusterMaxPhaseBlocks) {
                launch_cluster<BSX, ST, CLAMP>(ctx, a, order, n);
                return;
            }
        }
        launch_compact_v<BSX, ST, CLAMP, false>(ctx, a, order, n);
    }
}

template <int BSX, int ST, bool CLAMP>
static void launch_wave(msbg_ctx* ctx, const SweepArgs& a, const int2* items, int total, int* prog, unsigned int* counter) {
    const size_t smem = 2 * sizeof(float) * Compact<BSX>::BUF;
    static bool attr = false;
    if (!attr) {
        CUDA_CHECK(cudaFuncSetAttribute(sweep_wave_kernel<BSX, ST, CLAMP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CUDA_CHECK(cudaFuncSetAttribute(sweep_wave_kernel<BSX, ST, CLAMP>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)cudaSharedmemCarveoutMaxShared));
        attr = true;
    }
    const int threads = CompactThreads<BSX, ST>::v;
    int per_sm = 0;
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_wave_kernel<BSX, ST, CLAMP>, threads, smem));
    int sms = 0;
    CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    const int grid = std::max(1, std::min(total, std::max(per_sm, 1) * sms));
    begin_launch(ctx);
    sweep_wave_kernel<BSX, ST, CLAMP><<<(unsigned)grid, threads, smem, ctx->stream>>>(a, items, total, prog, counter,
                                                                                       ctx->status.as<int>());
    after_launch(ctx, "sweep_wave_kernel");
}

template <int BSX>
static void launch_wave_laplacian(msbg_ctx* ctx, const SweepArgs& a, const int2* items, int total, int* prog,
                                  unsigned int* counter) {
    if (a.clamp01) launch_wave<BSX, MSBG_LAPLACIAN, true>(ctx, a, items, total, prog, counter);
    else launch_wave<BSX, MSBG_LAPLACIAN, false>(ctx, a, items, total, prog, counter);
}

// The one-launch sweep runs the 7-tap stencil on active sets of at most
// this many blocks (measured on B200, 10 sweeps: 872 blocks 0.21 against
// 0.51 ms for a kernel per phase, 3,464 blocks 0.47 against 0.66 ms, 14,248
// blocks 1.67 against 1.70 ms, 56,056 blocks 6.46 against 4.82 ms; the
// 19-tap stencil gains nothing measurable at any size).
constexpr size_t kWaveMaxBlocks = 16384;

// The (sweep, plan index) items of `iterations` sweeps in wavefront order:
// by 8 t + colour + bz, then the higher bz, then plan index (colour-major
// Morton rank).
static void wave_items(SweepPlan* plan, msbg_ctx* ctx, int iterations) {
    if (plan->wave_iters == iterations) return;
    const size_t n = plan->n;
    MSBG_REQUIRE(n < (1u << 24), "too many blocks for a one-launch sweep");
    MSBG_REQUIRE(iterations < (1 << 20), "too many sweeps for a one-launch sweep");
    std::vector<std::pair<uint64_t, int2>> keyed;
    keyed.reserve(n * (size_t)iterations);
    for (int t = 0; t < iterations; ++t) {
        for (size_t i = 0; i < n; ++i) {
            const uint64_t bz = (uint64_t)plan->h_bz[i];
            MSBG_REQUIRE(bz < (1u << 21), "block layer out of range");
            const uint64_t k = 8 * (uint64_t)t + plan->h_col[i] + bz;
            // ties of k: the higher block layer first (a dependency one layer
            // up can tie with its dependant; one at the same layer or below
            // never does)
            keyed.push_back({(k << 21) | ((1u << 21) - 1 - bz), make_int2(t, (int)i)});
        }
    }
    std::sort(keyed.begin(), keyed.end(), [](const std::pair<uint64_t, int2>& x, const std::pair<uint64_t, int2>& y) {
        return x.first != y.first ? x.first < y.first : x.second.y < y.second.y;
    });
    std::vector<int2> items(keyed.size());
    for (size_t i = 0; i < keyed.size(); ++i) items[i] = keyed[i].second;
    plan->wave_items.reserve(items.size() * sizeof(int2));
    CUDA_CHECK(cudaMemcpyAsync(plan->wave_items.p, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice,
                               ctx->stream));
    sync(ctx);
    plan->wave_iters = iterations;
}

template <class E, int BSX, int ST>
static void launch_phase(msbg_ctx* ctx, const SweepArgs& a, const int32_t* order, int n) {
    constexpr int HALO = ST == MSBG_BILAPLACIAN ? 2 : 1;
    constexpr int HSX = BSX + 2 * HALO;
    const size_t smem = sizeof(float) * HSX * HSX * Stage<BSX>::RS;
    static bool attr_set = false;  // per instantiation
    if (!attr_set) {
        CUDA_CHECK(cudaFuncSetAttribute(sweep_phase_kernel<E, BSX, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        // all of the SM's unified L1/shared storage as shared memory: more
        // CTAs (and their staging loads) resident per SM
        CUDA_CHECK(cudaFuncSetAttribute(sweep_phase_kernel<E, BSX, ST>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)cudaSharedmemCarveoutMaxShared));
        attr_set = true;
    }
    const int threads = BSX * BSX < 32 ? 32 : BSX * BSX;
    // f32 with one-cell halos: the double-buffered kernel in the compact
    // layout (two 25-tap buffers would leave too few CTAs per SM)
    if (std::is_same<E, ElemF32>::value && BSX >= 8 && ST != MSBG_BILAPLACIAN && a.xface) {
        if (a.clamp01) launch_compact<BSX, ST, true>(ctx, a, order, n);
        else launch_compact<BSX, ST, false>(ctx, a, order, n);
        return;
    }
    if (std::is_same<E, ElemF32>::value && BSX >= 8 && ST != MSBG_BILAPLACIAN) {
        static bool pattr = false;
        if (!pattr) {
            CUDA_CHECK(cudaFuncSetAttribute(sweep_pipe_kernel<BSX, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(2 * smem)));
            CUDA_CHECK(cudaFuncSetAttribute(sweep_pipe_kernel<BSX, ST>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                            (int)cudaSharedmemCarveoutMaxShared));
            pattr = true;
        }
        int per_sm = 0;
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_pipe_kernel<BSX, ST>, threads, 2 * smem));
        int sms = 0;
        CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
        const int grid = std::max(1, std::min(n, std::max(per_sm, 1) * sms));
        begin_launch(ctx);
        sweep_pipe_kernel<BSX, ST><<<(unsigned)grid, threads, 2 * smem, ctx->stream>>>(a, order, n);
        after_launch(ctx, "sweep_pipe_kernel");
        return;
    }
    begin_launch(ctx);
    sweep_phase_kernel<E, BSX, ST><<<(unsigned)n, threads, smem, ctx->stream>>>(a, order, n);
    after_launch(ctx, "sweep_phase_kernel");
}

template <class E, int BSX>
static void launch_phase_st(msbg_ctx* ctx, int st, const SweepArgs& a, const int32_t* order, int n) {
    if (st == MSBG_LAPLACIAN) launch_phase<E, BSX, MSBG_LAPLACIAN>(ctx, a, order, n);
    else if (st == MSBG_MEAN_CURVATURE) launch_phase<E, BSX, MSBG_MEAN_CURVATURE>(ctx, a, order, n);
    else launch_phase<E, BSX, MSBG_BILAPLACIAN>(ctx, a, order, n);
}

template <class E>
static void launch_phase_bsx(msbg_ctx* ctx, int bsx, int st, const SweepArgs& a, const int32_t* order, int n) {
    switch (bsx) {
        case 4: launch_phase_st<E, 4>(ctx, st, a, order, n); break;
        case 8: launch_phase_st<E, 8>(ctx, st, a, order, n); break;
        case 16: launch_phase_st<E, 16>(ctx, st, a, order, n); break;
        default: launch_phase_st<E, 32>(ctx, st, a, order, n); break;
    }
}

static uint64_t fnv(uint64_t h, uint64_t v) {
    for (int i = 0; i < 8; ++i) { h ^= (v >> (8 * i)) & 0xff; h *= 0x100000001b3ULL; }
    return h;
}

// Builds (or reuses) the plan for `active` on grid g (and coarse + levels for
// a multiresolution sweep).
static SweepPlan* get_plan(msbg_grid* g, msbg_grid* coarse, const uint8_t* levels, const uint64_t* active, size_t n) {
    uint64_t key = 0xcbf29ce484222325ULL;
    key = fnv(key, n);
    key = fnv(key, g->version);
    key = fnv(key, (uint64_t)(uintptr_t)coarse);
    if (coarse) {
        key = fnv(key, coarse->version);
        key = fnv(key, coarse->n_slots());
        for (uint64_t b = 0; b < g->n_blocks; b += 1) key = fnv(key, levels[b]);
    }
    for (size_t k = 0; k < n; ++k) key = fnv(key, active[k]);
    if (g->plan && g->plan->key == key) return g->plan;

    std::vector<std::vector<uint64_t>> buckets(8);
    std::unordered_map<uint64_t, char> seen;
    for (size_t k = 0; k < n; ++k) {
        uint64_t bid = active[k];
        MSBG_REQUIRE(bid < g->n_blocks, "active block id out of range");
        if (grid_code(g, bid) < 0) continue;  // dummy or absent: skipped (solver.rs:196-199)
        if (!seen.emplace(bid, 1).second) continue;
        int64_t bx, by, bz;
        block_coords(g, bid, &bx, &by, &bz);
        buckets[(bx & 1) | ((by & 1) << 1) | ((bz & 1) << 2)].push_back(bid);
    }
    auto plan = new SweepPlan;
    plan->key = key;
    std::vector<int32_t> nbr, bxyz, order;
    int32_t pi = 0;
    for (int c = 0; c < 8; ++c) {
        auto& bk = buckets[c];
        std::stable_sort(bk.begin(), bk.end(), [&](uint64_t a, uint64_t b) {
            int64_t ax, ay, az, bx, by, bz;
            block_coords(g, a, &ax, &ay, &az);
            block_coords(g, b, &bx, &by, &bz);
            return morton3(ax, ay, az) < morton3(bx, by, bz);
        });
        plan->color_off[c] = pi;
        for (uint64_t bid : bk) {
            int64_t bx, by, bz;
            block_coords(g, bid, &bx, &by, &bz);
            bxyz.push_back((int32_t)bx);
            bxyz.push_back((int32_t)by);
            bxyz.push_back((int32_t)bz);
            // interior: the block and a halo of h cells lie inside the domain
            int32_t fl = 0;
            for (int hh = 1; hh <= 2; ++hh) {
                const int64_t B = g->bsx;
                bool in = bx * B - hh >= 0 && by * B - hh >= 0 && bz * B - hh >= 0 && (bx + 1) * B + hh <= (int64_t)g->sx &&
                          (by + 1) * B + hh <= (int64_t)g->sy && (bz + 1) * B + hh <= (int64_t)g->sz;
                if (in) fl |= 1 << (hh - 1);
            }
            // bits 4 + k: neighbour k lies at the domain edge (its halo of one
            // cell leaves the domain, so the Neumann rule may reflect its reads
            // into any of its 26 neighbours, this block included)
            for (int k = 0; k < 27; ++k) {
                const int64_t B = g->bsx, X = bx + k % 3 - 1, Y = by + (k / 3) % 3 - 1, Z = bz + k / 9 - 1;
                if (k == 13 || X < 0 || Y < 0 || Z < 0 || X >= (int64_t)g->nx || Y >= (int64_t)g->ny || Z >= (int64_t)g->nz)
                    continue;
                const bool in = X * B - 1 >= 0 && Y * B - 1 >= 0 && Z * B - 1 >= 0 && (X + 1) * B + 1 <= (int64_t)g->sx &&
                                (Y + 1) * B + 1 <= (int64_t)g->sy && (Z + 1) * B + 1 <= (int64_t)g->sz;
                if (!in) fl |= 1 << (4 + k);
            }
            bxyz.push_back(fl);
            plan->h_col.push_back((uint8_t)c);
            plan->h_bz.push_back((int32_t)bz);
            for (int k = 0; k < 27; ++k) {
                int64_t X = bx + k % 3 - 1, Y = by + (k / 3) % 3 - 1, Z = bz + k / 9 - 1;
                int32_t code = kCodeEmpty;
                if (X >= 0 && Y >= 0 && Z >= 0 && X < (int64_t)g->nx && Y < (int64_t)g->ny && Z < (int64_t)g->nz) {
                    uint64_t nbid = (uint64_t)X + (uint64_t)Y * g->nx + (uint64_t)Z * g->nxy;
                    if (coarse && levels[nbid] > levels[bid]) {
                        int32_t cs = grid_code(coarse, nbid);
                        code = cs >= 0 ? kCodeCoarse0 - cs : kCodeEmpty;
                    } else {
                        code = grid_code(g, nbid);
                        if (coarse && code == kCodeFull) code = kCodeEmpty;
                    }
                }
                nbr.push_back(code);
            }
            order.push_back(pi++);
        }
    }
    plan->color_off[8] = pi;
    plan->n = (size_t)pi;
    // slots read through x-planes: x-side neighbours (faces and edges) that are value blocks
    {
        std::vector<int32_t> xs;
        for (size_t k = 0; k < nbr.size(); k += 27)
            for (int j = 0; j < 27; ++j)
                if (j % 3 != 1 && nbr[k + j] >= 0) xs.push_back(nbr[k + j]);
        std::sort(xs.begin(), xs.end());
        xs.erase(std::unique(xs.begin(), xs.end()), xs.end());
        plan->n_xslots = xs.size();
        if (!xs.empty()) {
            plan->xslots.reserve(xs.size() * 4);
            CUDA_CHECK(cudaMemcpyAsync(plan->xslots.p, xs.data(), xs.size() * 4, cudaMemcpyHostToDevice, g->ctx->stream));
            sync(g->ctx);
        }
    }
    if (pi) {
        plan->nbr.reserve(nbr.size() * 4);
        plan->bxyz.reserve(bxyz.size() * 4);
        plan->order.reserve(order.size() * 4);
        CUDA_CHECK(cudaMemcpyAsync(plan->nbr.p, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice, g->ctx->stream));
        CUDA_CHECK(cudaMemcpyAsync(plan->bxyz.p, bxyz.data(), bxyz.size() * 4, cudaMemcpyHostToDevice, g->ctx->stream));
        CUDA_CHECK(cudaMemcpyAsync(plan->order.p, order.data(), order.size() * 4, cudaMemcpyHostToDevice, g->ctx->stream));
        sync(g->ctx);
    }
    if (g->plan && !g->plan->graphs.empty()) sync(g->ctx);  // its graphs may still run
    delete g->plan;
    g->plan = plan;
    return plan;
}

static void sweep(msbg_grid* g, msbg_grid* coarse, const uint8_t* levels, const uint64_t* active, size_t n, int stencil,
                  float dt, int iterations, int clamp01, uint32_t seed = 0xdeadbeefu, int lanes = 16,
                  uint64_t* stream_pos = nullptr) {
    MSBG_REQUIRE(stencil >= 0 && stencil <= 2, "bad stencil");
    MSBG_REQUIRE(iterations >= 0, "negative iteration count");
    MSBG_REQUIRE(g->bsx >= 4, "sweeps need bsx >= 4");
    if (g->dtype == MSBG_U8)
        MSBG_REQUIRE((lanes == 4 || lanes == 8 || lanes == 16) && lanes <= g->bsx,
                     "Density8 sweeps need 4, 8 or 16 generator lanes, at most the block size");
    if (coarse) {
        MSBG_REQUIRE(g->dtype == MSBG_F32 && coarse->dtype == MSBG_F32, "multiresolution sweep needs f32 levels");
        MSBG_REQUIRE(coarse->bsx * 2 == g->bsx && coarse->nx == g->nx && coarse->ny == g->ny && coarse->nz == g->nz,
                     "coarse level must have half the block size on the same block grid");
        MSBG_REQUIRE(levels, "null levels");
    }
    set_device(g->ctx);
    SweepPlan* plan = get_plan(g, coarse, levels, active, n);
    if (!plan->n || !iterations) return;
    SweepArgs a;
    a.payload = g->payload.p;
    a.coarse = coarse ? coarse->payload.as<float>() : nullptr;
    a.nbr = plan->nbr.as<int32_t>();
    a.bxyz = plan->bxyz.as<int32_t>();
    a.sx = (int32_t)g->sx; a.sy = (int32_t)g->sy; a.sz = (int32_t)g->sz;
    a.empty = coarse ? 0.0f : quantize_roundtrip(g->dtype, g->empty_value);
    a.full = coarse ? 0.0f : quantize_roundtrip(g->dtype, g->full_value);
    a.dt = dt;
    a.clamp01 = clamp01 ? 1 : 0;
    int lg = 0;
    while ((1 << lg) < lanes) ++lg;
    for (int l = 0; l < 16; ++l) a.sr_seed[l] = sr_lane_seed(seed, (uint32_t)l);
    a.sr_lg = lg;
    a.sr_zstep = sr_pow((uint64_t)(g->bsx * g->bsx) >> lg);
    const uint64_t chunks_per_sweep = (uint64_t)plan->n * ((uint64_t)g->block_elems >> lg);
    const uint64_t pos0 = stream_pos ? *stream_pos : 0;
    // x-plane side buffer: sized for every slot (here, before any launch: a
    // graph capture below must not allocate), refreshed from the payload at
    // the start of each call (the payload may have changed in between)
    const size_t slots = g->n_slots();
    const int xd = stencil == MSBG_BILAPLACIAN ? 2 : 1;  // x-planes per side the stencil's halo reaches
    if (plan->xface_slots < slots * xd) {
        plan->xface.reserve(slots * 2 * xd * g->bsx * g->bsx * sizeof(float));
        plan->xface_slots = slots * xd;
    }
    a.xface = plan->xface.as<float>();
    const int32_t* order = plan->order.as<int32_t>();
    // the 7-tap stencil on f32 8^3 or 16^3 blocks of a small active set:
    // every colour phase of every sweep in one launch
    const bool wave =
        g->dtype == MSBG_F32 && (g->bsx == 8 || g->bsx == 16) && stencil == MSBG_LAPLACIAN && plan->n <= kWaveMaxBlocks;
    int* prog = nullptr;
    unsigned int* counter = nullptr;
    if (wave) {
        MSBG_REQUIRE((double)plan->n * iterations < 2147483647.0, "too many (sweep, block) items for one launch");
        wave_items(plan, g->ctx, iterations);
        if (plan->wave_slots < slots) {
            plan->wave_prog.reserve(slots * 4 + 256);
            plan->wave_slots = slots;
        }
        prog = plan->wave_prog.as<int>();
        counter = reinterpret_cast<unsigned int*>(plan->wave_prog.as<char>() + ((slots * 4 + 127) & ~size_t(127)));
    }
    auto issue = [&]() {
        const int32_t* xs = plan->xslots.as<int32_t>();
        const size_t nxs = plan->n_xslots;
        if (g->dtype == MSBG_F32) xface_init<ElemF32>(g->ctx, g->bsx, g->payload.p, xs, nxs, xd, a.xface);
        else if (g->dtype == MSBG_U16) xface_init<ElemU16>(g->ctx, g->bsx, g->payload.p, xs, nxs, xd, a.xface);
        else if (g->dtype == MSBG_U8) xface_init<ElemU8>(g->ctx, g->bsx, g->payload.p, xs, nxs, xd, a.xface);
        else if (g->dtype == MSBG_F16) xface_init<ElemF16>(g->ctx, g->bsx, g->payload.p, xs, nxs, xd, a.xface);
        else xface_init<ElemBF16>(g->ctx, g->bsx, g->payload.p, xs, nxs, xd, a.xface);
        if (wave) {
            begin_launch(g->ctx);
            wave_init_kernel<<<(unsigned)std::min<size_t>((slots + 255) / 256 + 1, 148 * 8), 256, 0, g->ctx->stream>>>(
                prog, slots, counter);
            after_launch(g->ctx, "wave_init_kernel");
            begin_launch(g->ctx);
            wave_zero_kernel<<<(unsigned)std::min<size_t>((plan->n + 255) / 256, 148 * 8), 256, 0, g->ctx->stream>>>(
                prog, a.nbr, (int)plan->n);
            after_launch(g->ctx, "wave_zero_kernel");
            const int total = (int)(plan->n * (size_t)iterations);
            const int2* items = plan->wave_items.as<int2>();
            if (g->bsx == 16) launch_wave_laplacian<16>(g->ctx, a, items, total, prog, counter);
            else launch_wave_laplacian<8>(g->ctx, a, items, total, prog, counter);
            return;
        }
        for (int it = 0; it < iterations; ++it) {
            a.sr_base = pos0 + (uint64_t)it * chunks_per_sweep;
            for (int c = 0; c < 8; ++c) {
                int cnt = plan->color_off[c + 1] - plan->color_off[c];
                if (!cnt) continue;
                const int32_t* o = order + plan->color_off[c];
                if (g->dtype == MSBG_F32) launch_phase_bsx<ElemF32>(g->ctx, g->bsx, stencil, a, o, cnt);
                else if (g->dtype == MSBG_U16) launch_phase_bsx<ElemU16>(g->ctx, g->bsx, stencil, a, o, cnt);
                else if (g->dtype == MSBG_U8) launch_phase_bsx<ElemU8>(g->ctx, g->bsx, stencil, a, o, cnt);
                else if (g->dtype == MSBG_F16) launch_phase_bsx<ElemF16>(g->ctx, g->bsx, stencil, a, o, cnt);
                else launch_phase_bsx<ElemBF16>(g->ctx, g->bsx, stencil, a, o, cnt);
            }
        }
    };
    // f32 sweeps: the call's launches (a kernel per colour phase: 80 for 10
    // sweeps) are captured once into a graph and replayed by later calls with
    // the same plan, arguments and buffers, so a phase of a few hundred
    // blocks costs a graph node rather than a host launch.  (Per-kernel
    // timing launches directly; Density8 sweeps advance the generator
    // stream every call.)
    if (g->dtype != MSBG_F32 || g->ctx->timing) {
        issue();
        if (stream_pos && g->dtype == MSBG_U8) *stream_pos = pos0 + (uint64_t)iterations * chunks_per_sweep;
        return;
    }
    uint64_t key = 0xcbf29ce484222325ULL;
    auto bits = [](float f) { uint32_t u; memcpy(&u, &f, 4); return (uint64_t)u; };
    for (uint64_t v : {(uint64_t)iterations, (uint64_t)stencil, bits(dt), (uint64_t)a.clamp01, (uint64_t)(uintptr_t)a.payload,
                       (uint64_t)(uintptr_t)a.coarse, (uint64_t)(uintptr_t)a.xface, (uint64_t)(uintptr_t)prog, bits(a.empty),
                       bits(a.full)})
        key = fnv(key, v);
    SweepPlan::Graph* sg = nullptr;
    for (auto& q : plan->graphs)
        if (q.key == key) sg = &q;
    if (!sg) {
        msbg_ctx* ctx = g->ctx;
        const uint64_t l0 = ctx->launches;
        cudaGraph_t graph = nullptr;
        CUDA_CHECK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        try {
            issue();
        } catch (...) {
            cudaStreamEndCapture(ctx->stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            ctx->launches = l0;
            throw;
        }
        CUDA_CHECK(cudaStreamEndCapture(ctx->stream, &graph));
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) MSBG_THROW(MSBG_ERR_CUDA, std::string("sweep graph: ") + cudaGetErrorString(e));
        if (plan->graphs.size() >= 8) {  // keep the most recent few
            cudaGraphExecDestroy(plan->graphs.front().exec);
            plan->graphs.erase(plan->graphs.begin());
        }
        plan->graphs.push_back({key, exec, (int)(ctx->launches - l0)});
        ctx->launches = l0;
        sg = &plan->graphs.back();
    }
    CUDA_CHECK(cudaGraphLaunch(sg->exec, g->ctx->stream));
    g->ctx->launches += (uint64_t)sg->kernels;
}

}  // namespace msbg

using namespace msbg;

extern "C" {

int msbg_sweep(msbg_grid* g, const uint64_t* active, size_t n, int stencil, float dt, int iterations, int clamp01) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && (active || !n), "null argument");
    sweep(g, nullptr, nullptr, active, n, stencil, dt, iterations, clamp01, 0xdeadbeefu, std::min(16, g->bsx));
    MSBG_API_END
}

int msbg_sweep_stochastic(msbg_grid* g, const uint64_t* active, size_t n, int stencil, float dt, int iterations,
                          int clamp01, uint32_t seed, int lanes, uint64_t* stream_pos) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && (active || !n) && stream_pos, "null argument");
    sweep(g, nullptr, nullptr, active, n, stencil, dt, iterations, clamp01, seed, lanes, stream_pos);
    MSBG_API_END
}

int msbg_sweep_multires(msbg_grid* fine, msbg_grid* coarse, const uint8_t* levels, const uint64_t* active, size_t n,
                        int stencil, float dt, int iterations, int clamp01) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(fine && coarse && (active || !n), "null argument");
    MSBG_REQUIRE(fine->ctx == coarse->ctx, "levels on different contexts");
    sweep(fine, coarse, levels, active, n, stencil, dt, iterations, clamp01);
    MSBG_API_END
}

}  // extern "C"
