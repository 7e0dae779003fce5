// p2g.cu -- particles_to_grid (fluid/p2g.rs:141-412): deterministic,
// atomic-free sum-splat of mass and momentum to the right MAC faces.
//
// Pipeline (all on the context stream):
//  1. Morton key of every particle's cell, stable radix sort -> permutation;
//     payloads gathered into cell-sorted SoA arrays.  A 16^3 block is one
//     contiguous Morton range, so particles end up grouped by block ("particle
//     blocks") and by cell inside a block.
//  2. Per particle block: CSR of its cells, and the union of its particles'
//     footprint blocks (active_blocks, p2g.rs:104-136, reach r_p + 1) as a
//     27-bit mask; the active set is the sorted union over particle blocks.
//  3. Splat: one CTA per (particle block, face direction) accumulates into a
//     (bsx + 2M)^3 staging window in shared memory (M = ceil(r_p)), in FP64.
//     Cells are visited by 2x2x2 tiles in (M+1)^3 colour phases: cells of
//     two tiles of one phase are 2M+1 apart, so their face windows are
//     disjoint and each warp owns its tile's faces -- no atomics, a fixed
//     summation order.  A warp handles a tile's cells in turn: lanes take a
//     cell's (2M+1)^2 candidate face columns, loop over the
//     cell's particles, and evaluate the reference's per-face weight
//     w = max(1 - d^2/r_p^2, 0)^3 with its exact f32 operation order and its
//     exact clamped footprint (p2g.rs:263-330).
//  4. Combine: one CTA per (active block, direction) sums, in the reference's
//     commit order (colour of the contributing particle block, p2g.rs:186-216),
//     the staging windows of the <= 27 neighbouring particle blocks, rounds to
//     f32 and applies normalize_velocity (mac.rs:106-132).
// FP64 accumulation makes the result the correctly rounded sum of the f32
// per-particle terms up to a few ulp; the reference's own f32 sums differ from
// that by their rounding error.
#include <algorithm>

#include "mac.cuh"
#include "sort.cuh"

namespace msbg {

struct SplatArgs {
    const float *px, *py, *pz, *pm, *pv[3];  // cell-sorted particles: x, y, z, velocity
    int ps;                                  // components at px[i ps] .. pv[d][i ps]; mass at pm[i]
    const int32_t* cell_begin;               // [npb][bsx^3] by local Morton code
    const int32_t* cell_end;
    const uint64_t* pb_key;                  // block Morton key per particle block
    const uint64_t* lane_mask[3];            // per direction: clipped footprint as lane and face bits
    double* partial;                         // [npb][3][2][W^3]
    int* status;                             // device status word (bit 4: a tile wait gave up)
    float r_p, inv_r2;
};

template <int BSX> struct P2GLg { static constexpr int v = BSX == 8 ? 3 : BSX == 16 ? 4 : 5; };

struct CombineArgs {
    const double* partial;
    const int32_t* nbr_rank;  // [n_active][27] particle-block rank or -1
    const uint64_t* active;   // sorted active bids
    const int32_t* slots;     // MAC slot per active block
    float* mass[3];
    float* vel[3];
    int64_t nx, ny;
};

template <int BSX, int M>
__global__ void __launch_bounds__(256) p2g_combine_kernel(CombineArgs a) {
    constexpr int W = BSX + 2 * M;
    constexpr int WW = W * W * W;
    constexpr int N = BSX * BSX * BSX;
    constexpr int LG = P2GLg<BSX>::v;
    __shared__ int32_t rank[27];
    const int j = blockIdx.x, dir = blockIdx.y;
    const uint64_t bid = a.active[j];
    const int64_t bx = (int64_t)(bid % a.nx), by = (int64_t)((bid / a.nx) % a.ny), bz = (int64_t)(bid / (a.nx * a.ny));
    if (threadIdx.x < 27) rank[threadIdx.x] = a.nbr_rank[(size_t)j * 27 + threadIdx.x];
    __syncthreads();
    const int px = (int)(bx & 1), py = (int)(by & 1), pz = (int)(bz & 1);
    const int32_t slot = a.slots[j];
    // this direction's output block (selected once: a dynamically indexed
    // parameter array is read through local memory)
    float* const mout = (dir == 0 ? a.mass[0] : dir == 1 ? a.mass[1] : a.mass[2]) + (size_t)slot * N;
    float* const vout = (dir == 0 ? a.vel[0] : dir == 1 ? a.vel[1] : a.vel[2]) + (size_t)slot * N;
    const double* const part = a.partial + (size_t)dir * 2 * WW;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const int lx = i & (BSX - 1), ly = (i >> LG) & (BSX - 1), lz = i >> (2 * LG);
        // Contributions are added in the colour order of the contributing
        // particle block (the reference commits colour by colour).  A face
        // lies in the window of the block itself and, along each axis, of at
        // most one neighbour (-1 within M of the low side, +1 within M of
        // the high side; 2M <= bsx), and the two differ in parity, so each
        // colour names at most one contributing block.
        const int ex = lx < M ? -1 : (lx >= BSX - M ? 1 : 0);
        const int ey = ly < M ? -1 : (ly >= BSX - M ? 1 : 0);
        const int ez = lz < M ? -1 : (lz >= BSX - M ? 1 : 0);
        double sm = 0.0, sv = 0.0;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int ox = (c & 1) == px ? 0 : ex, oy = ((c >> 1) & 1) == py ? 0 : ey, oz = ((c >> 2) & 1) == pz ? 0 : ez;
            if (((c & 1) != px && !ex) || (((c >> 1) & 1) != py && !ey) || (((c >> 2) & 1) != pz && !ez)) continue;
            const int r = rank[(ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)];
            if (r < 0) continue;
            const int sx = lx - BSX * ox + M, sy = ly - BSX * oy + M, sz = lz - BSX * oz + M;
            const double* p = part + (size_t)r * 3 * 2 * WW + (sz * W + sy) * W + sx;
            sm += p[0];
            sv += p[WW];
        }
        const float mf = (float)sm, pf = (float)sv;
        mout[i] = mf;
        vout[i] = mf > 0.0f ? pf / mf : 0.0f;
    }
}

// Cell CSR of one particle block: begin/end index of every cell (by local
// Morton code) in the sorted particle order.
__global__ void cell_csr_kernel(const uint64_t* skeys, const uint64_t* pb_starts, int lg, int32_t* cell_begin,
                                int32_t* cell_end) {
    const int k = blockIdx.x;
    const int n_cells = 1 << (3 * lg);
    const uint64_t cmask = (uint64_t)n_cells - 1;
    int32_t* cb = cell_begin + (size_t)k * n_cells;
    int32_t* ce = cell_end + (size_t)k * n_cells;
    for (int i = threadIdx.x; i < n_cells; i += blockDim.x) cb[i] = ce[i] = 0;
    __syncthreads();
    // particle indices fit int32 (the CSR stores them as int32); a key's
    // neighbours come from the adjacent lanes (the warp's end lanes load
    // theirs), every lane of the CTA taking the same rounds
    const int32_t s = (int32_t)pb_starts[k], e = (int32_t)pb_starts[k + 1];
    const uint32_t cm = (uint32_t)cmask;
    const int lane = threadIdx.x & 31;
    for (int32_t r = s; r < e; r += (int32_t)blockDim.x) {
        const int32_t i = r + (int32_t)threadIdx.x;
        const bool in = i < e;
        const uint32_t c = in ? (uint32_t)skeys[i] & cm : 0u;
        uint32_t prev = __shfl_up_sync(0xffffffffu, c, 1), next = __shfl_down_sync(0xffffffffu, c, 1);
        if (lane == 0 && in && i > s) prev = (uint32_t)skeys[i - 1] & cm;
        if (lane == 31 && i + 1 < e) next = (uint32_t)skeys[i + 1] & cm;
        if (in) {
            if (i == s || prev != c) cb[c] = i;
            if (i == e - 1 || next != c) ce[c] = i + 1;
        }
    }
}

// Payload gather into cell-sorted SoA (only for particles in the caller's
// order, perm != null; sorted particles are read by the splat in place), each
// particle's block-footprint mask (particles/mod.rs:207-212 footprint_axis
// with r_scan = (r_p + 1) / bsx, relative to its own block) and, per face
// direction, its clipped face footprint (p2g.rs:263-270) relative to its own
// cell as the splat kernel's lane and face bits: for direction DIR with face
// axis F and lane axes U, V (U = DIR == 0 ? 1 : 0, V = DIR == 2 ? 1 : 2),
// bit du + (2M+1) dv (du, dv in [0, 2M]) is set when the cell-centred
// footprint (offset 0.5) holds the lane's row, at cell offsets du - M and
// dv - M along U and V, and bit 56 + s (s in [0, 2M]) when the face
// footprint (offset 1.0) along F holds cell offset s - 1 - M.
// MT > 0 fixes M = MT at compile time (the footprint loops unrolled).
template <int MT>
__global__ void p2g_gather_kernel(const float* pos, const float* vel, const float* mass, const uint32_t* perm, size_t n,
                                  int lg, int M_, float r_p, float r_scan_bsx, int64_t nx, int64_t ny, int64_t nz,
                                  float* px, float* py, float* pz, float* pm, float* v0, float* v1, float* v2,
                                  uint32_t* fmask, uint64_t* lane_mask, int* bad) {
    const int M = MT > 0 ? MT : M_;
    const float inv_bsx = 1.0f / (float)(1 << lg);
    const int32_t B = 1 << lg;
    const int WIN = 2 * M + 1;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t s = perm ? perm[i] : i;
        const float x = pos[3 * s], y = pos[3 * s + 1], z = pos[3 * s + 2];
        if (perm) {
            px[i] = x; py[i] = y; pz[i] = z;
            pm[i] = mass[s];
            v0[i] = vel[3 * s]; v1[i] = vel[3 * s + 1]; v2[i] = vel[3 * s + 2];
        }
        const float p[3] = {x, y, z};
        // block counts per axis are below 2^21 (Morton keys take 21 bits per
        // axis), so the cell and block arithmetic fits 32 bits; a coordinate
        // beyond the int32 range converts to INT_MAX, whose block is out of
        // range as well
        const int32_t nn[3] = {(int32_t)nx, (int32_t)ny, (int32_t)nz};
        uint32_t lo[3], hi[3];
        int32_t a1[3][2], a2[3][2], cell[3];
        bool out = false;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const int32_t c = p[ax] > 0.0f ? (int32_t)p[ax] : 0;  // the particle's cell (p as usize)
            const int32_t cb = c >> lg;                              // and block
            if (cb >= nn[ax]) out = true;
            const float b = p[ax] * inv_bsx;  // p / bsx: bsx is a power of two, the product is exact
            const int32_t l = max((int32_t)truncf(b - r_scan_bsx), 0);
            const int32_t h = min((int32_t)truncf(b + r_scan_bsx), nn[ax] - 1);
            lo[ax] = (uint32_t)(min(max(l - cb, -1), 1) + 1);
            hi[ax] = (uint32_t)(min(max(h - cb, -1), 1) + 1);
            const int32_t b0 = cb * B;
            cell[ax] = c - b0;
#pragma unroll
            for (int face = 0; face < 2; ++face) {
                // staging coordinates (global - (b0 - M)) of the clipped footprint
                const float of = face ? 1.0f : 0.5f;
                a1[ax][face] = min(max((int32_t)ceilf((p[ax] - r_p) - of), b0 - M), b0 + B + M - 1) - (b0 - M);
                a2[ax][face] = min(max((int32_t)floorf((p[ax] + r_p) - of), b0 - M), b0 + B + M - 1) - (b0 - M);
            }
        }
        // per axis, the offsets k in [0, 2M] whose staging coordinate
        // cell + k (cell-centred, face 0) or cell + k - 1 (faces, face 1)
        // lies in the clipped footprint: a contiguous run of bits
        uint32_t run[3][2];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax)
#pragma unroll
            for (int face = 0; face < 2; ++face) {
                const int lo = max(a1[ax][face] - cell[ax] + face, 0), hi = min(a2[ax][face] - cell[ax] + face, WIN - 1);
                run[ax][face] = lo > hi ? 0u : ((2u << hi) - 1u) & ~((1u << lo) - 1u);
            }
#pragma unroll
        for (int dir = 0; dir < 3; ++dir) {
            const int F = dir, U = dir == 0 ? 1 : 0, V = dir == 2 ? 1 : 2;
            // lane bit du + WIN dv for du in run U, dv in run V: the U run
            // repeated at the V run's rows (one product, no carries)
            uint64_t rows = 0;
#pragma unroll
            for (int dv = 0; dv < WIN; ++dv)
                if ((run[V][0] >> dv) & 1u) rows |= 1ull << (WIN * dv);
            uint64_t m = (uint64_t)run[U][0] * rows | ((uint64_t)run[F][1] << 56);
            // M = 2: bit 32 when the footprint has the regular r_p = 2 shape
            // (four rows along U and V starting 2 - s before the cell, s = 0
            // or 1, and faces -2 .. +1 along F), bits 33 and 34 the shifts
            // s_U and s_V (the r_p = 2 splat's anchor); lane bits end at 24
            if (M == 2) {
                const uint32_t rU = run[U][0], rV = run[V][0], rF = run[F][1];
                if ((rU == 0x0fu || rU == 0x1eu) && (rV == 0x0fu || rV == 0x1eu) && rF == 0x1eu)
                    m |= (1ull << 32) | ((uint64_t)(rU == 0x1eu) << 33) | ((uint64_t)(rV == 0x1eu) << 34);
            }
            lane_mask[(size_t)dir * n + i] = m;
        }
        if (out) { atomicExch(bad, 1); fmask[i] = 0; continue; }
        // bit dx + 3 dy + 9 dz for dx, dy, dz in [lo, hi] per axis: the x run
        // replicated at the y run's and the z run's offsets (products of
        // disjoint bit patterns, no carries)
        auto rep = [](uint32_t l, uint32_t h, uint32_t step) {
            uint32_t r = 0;
            for (uint32_t d = 0; d < 3; ++d)
                if (l <= d && d <= h) r |= 1u << (step * d);
            return r;
        };
        const uint32_t xr = ((2u << hi[0]) - 1u) & ~((1u << lo[0]) - 1u);
        fmask[i] = xr * rep(lo[1], hi[1], 3) * rep(lo[2], hi[2], 9);
    }
}

// Particles a splat warp stages at once (two float4 each): a whole typical
// tile where the FP64 window leaves room in shared memory, 32 otherwise.
template <int BSX, int M> struct SplatCap {
    static constexpr int v = 2 * 8 * (BSX + 2 * M) * (BSX + 2 * M) * (BSX + 2 * M) <= 131072 ? 128 : 32;
};

// Warps of a splat CTA.  Tiles wait for their overlapping predecessors, so
// more warps mostly wait longer; 20 (one CTA per SM, up to 96 registers a
// thread) measured fastest on B200 among 16, 20, 24 and 32.
constexpr int kSplatWarps = 20;

// Pairs of f32 in one 64-bit register, and the paired IEEE single-precision
// operations of sm_100 (each half rounded to nearest, exactly as the scalar
// operation).  A paired product that feeds a paired sum directly can be
// fused into one paired multiply-add by the code generator even with .rn
// (measured on B200), so callers keep such products scalar.
__device__ __forceinline__ uint64_t f2_pack(float a, float b) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_unpack(uint64_t v, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ uint64_t f2_add(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ uint64_t f2_sub(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ uint64_t f2_mul(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

// Splat kernel: one CTA per (particle block, direction DIR).  The block's
// (bsx + 2M)^3 staging window of face sums lives in shared memory in FP64.
// Cells are grouped in 2x2x2 tiles; a warp takes a whole tile (its 8 cells in
// a fixed order).  The face windows of two tiles overlap only when the tiles
// are at most M apart along every axis, so tiles coloured by tile coordinate
// mod (M+1) never overlap within a colour.  Warps take tiles from a shared
// counter in colour-major order, and before adding into the window a warp
// waits until every overlapping tile of a lower colour is done (per-tile
// flags in shared memory).  Every face therefore receives its cells'
// contributions in colour order, then cell order: a fixed summation order
// with no atomics and no CTA-wide barrier between colours.
//
// Inside a cell, the lanes of the warp take the (2M+1)^2 positions of the
// cell's face window across the two axes other than the face axis, and each
// lane keeps the 2M+1 faces along the face axis in FP64 registers.  For every
// particle of the cell (sorted order) a lane evaluates the reference's f32
// term for each of its faces inside the particle's clipped footprint
// (p2g.rs:263-330, operation by operation; the footprint arrives as the
// particle's lane and face bits), then adds its register sums to the window.
// A tile wait that runs past a second sets bit 4 of the status word and goes
// on (the result is then wrong and the host reports the error).
template <int BSX, int M, int DIR>
__global__ void __launch_bounds__(32 * kSplatWarps, 1) p2g_cells_kernel(SplatArgs a) {
    constexpr int W = BSX + 2 * M;
    constexpr int WW = W * W * W;
    constexpr int WIN = 2 * M + 1;
    constexpr int NUV = WIN * WIN;       // lane positions
    constexpr int Q = (NUV + 31) / 32;   // lane rounds
    constexpr int T = BSX / 2, K = M + 1, NT = T * T * T;
    constexpr int NNB = WIN * WIN * WIN;  // tile offsets in [-M, M]^3
    constexpr int CAP = SplatCap<BSX, M>::v;
    constexpr int NR = (NNB + 31) / 32;   // of them per lane
    // Faces s = 1 .. WIN-1 in pairs; face 0 (offset -M-1) is inside a
    // particle's footprint only when the particle sits exactly on a face
    // plane, so it is evaluated alone, and only for such particles.
    constexpr int NP = (WIN - 1) / 2;    // face pairs (2h+1, 2h+2)
    static_assert(WIN <= 7 && NUV <= 56, "lane and face bits must fit one u64");
    static_assert(NT < 0xffff, "tile indices must fit 16 bits");
    extern __shared__ double st[];       // [2][W^3]: mass, momentum; then per-warp particle slots
    __shared__ uint32_t s_done[NT];
    __shared__ uint16_t s_order[NT];     // tiles in colour-major order
    __shared__ uint32_t s_next;
    const int k_pb = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31;
    float4* wslot = reinterpret_cast<float4*>(st + 2 * WW) + (size_t)(tid >> 5) * 2 * SplatCap<BSX, M>::v;
    for (int i = tid; i < 2 * WW; i += blockDim.x) st[i] = 0.0;
    for (int t = tid; t < NT; t += blockDim.x) {
        s_done[t] = 0;
        const int tx = t % T, ty = (t / T) % T, tz = t / (T * T);
        const int cx = tx % K, cy = ty % K, cz = tz % K;
        const int ci = cx + K * (cy + K * cz);
        int base = 0;
        for (int c = 0; c < ci; ++c) {
            const int ox = c % K, oy = (c / K) % K, oz = c / (K * K);
            base += ((T - ox + K - 1) / K) * ((T - oy + K - 1) / K) * ((T - oz + K - 1) / K);
        }
        const int ntx = (T - cx + K - 1) / K, nty = (T - cy + K - 1) / K;
        s_order[base + (tx / K) + ntx * ((ty / K) + nty * (tz / K))] = (uint16_t)t;
    }
    if (tid == 0) s_next = 0;
    const uint64_t key = a.pb_key[k_pb];
    const int32_t b0[3] = {(int32_t)compact3(key) * BSX, (int32_t)compact3(key >> 1) * BSX,
                           (int32_t)compact3(key >> 2) * BSX};
    // axes: F = face axis (registers), U and V = lane axes
    constexpr int F = DIR, U = DIR == 0 ? 1 : 0, V = DIR == 2 ? 1 : 2;
    const int32_t* cb = a.cell_begin + (size_t)k_pb * BSX * BSX * BSX;
    const int32_t* ce = a.cell_end + (size_t)k_pb * BSX * BSX * BSX;
    const float* __restrict__ pv = a.pv[DIR];
    const uint64_t* __restrict__ lmask = a.lane_mask[DIR];
    const float inv_r2 = a.inv_r2;
    __syncthreads();
    while (true) {
        uint32_t q = 0;
        if (lane == 0) q = atomicAdd(&s_next, 1u);
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= (uint32_t)NT) break;
        const int t = s_order[q];
        const int tc[3] = {t % T, (t / T) % T, t / (T * T)};
        const int ci = tc[0] % K + K * (tc[1] % K + K * (tc[2] % K));
        // the tile's cell ranges, one cell per lane, fetched before the wait
        int cbeg = 0, cend = 0;
        if (lane < 8) {
            const uint32_t lm = (uint32_t)morton3(2 * tc[0] + (lane & 1), 2 * tc[1] + ((lane >> 1) & 1), 2 * tc[2] + (lane >> 2));
            cbeg = cb[lm];
            cend = ce[lm];
        }
        // the overlapping tiles of lower colours: each lane takes up to NR of
        // them; the warp waits for them before its first shared-memory add
        // of this tile (so the tile's first cell is computed meanwhile),
        // drops each as it is seen done, and sleeps between rounds
        uint32_t nbi[(NR + 1) / 2];  // tile indices, two 16-bit fields per word, 0xffff = none
#pragma unroll
        for (int k = 0; k < (NR + 1) / 2; ++k) nbi[k] = 0xffffffffu;
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            const int o = lane + 32 * k;
            const int nx = tc[0] + o % WIN - M, ny = tc[1] + (o / WIN) % WIN - M, nz = tc[2] + o / (WIN * WIN) - M;
            const bool dep = o < NNB && nx >= 0 && ny >= 0 && nz >= 0 && nx < T && ny < T && nz < T &&
                             nx % K + K * (ny % K + K * (nz % K)) < ci;
            if (dep) nbi[k >> 1] &= ~(0xffffu << (16 * (k & 1))) | ((uint32_t)(nx + T * (ny + T * nz)) << (16 * (k & 1)));
        }
        bool deps_pending = true;
        auto wait_deps = [&]() {
            uint64_t t0 = 0;
            uint32_t spins = 0, sleep_ns = 32;
            while (true) {
                bool ready = true;
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    const uint32_t idx = (nbi[k >> 1] >> (16 * (k & 1))) & 0xffffu;
                    if (idx != 0xffffu) {
                        if (*(volatile uint32_t*)&s_done[idx]) nbi[k >> 1] |= 0xffffu << (16 * (k & 1));
                        else ready = false;
                    }
                }
                if (__all_sync(0xffffffffu, ready)) break;
                __nanosleep(sleep_ns);
                sleep_ns = sleep_ns < 512 ? 2 * sleep_ns : 512;
                if ((++spins & 63u) == 0) {
                    const uint64_t now = globaltimer_ns();
                    if (!t0) t0 = now;
                    else if (now - t0 > kWaitLimitNs) {
                        if (lane == 0) atomicOr(a.status, 4);
                        break;
                    }
                }
            }
            __threadfence_block();
            deps_pending = false;
        };
        const int e_tile = (int)__reduce_max_sync(0xffffffffu, lane < 8 ? (uint32_t)cend : 0u);
        int st_lo = 0, st_hi = 0;  // the particles held by the warp's staging slots
        for (int sub = 0; sub < 8; ++sub) {
            // cells of a tile have overlapping face windows: order this
            // cell's shared-memory updates after the previous cell's across
            // the warp's lanes
            __syncwarp();
            const int b = __shfl_sync(0xffffffffu, cbeg, sub), e = __shfl_sync(0xffffffffu, cend, sub);
            if (b >= e) continue;
            int cell[3];
            cell[0] = 2 * tc[0] + (sub & 1);
            cell[1] = 2 * tc[1] + ((sub >> 1) & 1);
            cell[2] = 2 * tc[2] + (sub >> 2);
#pragma unroll
            for (int qq = 0; qq < Q; ++qq) {
                const int uv = lane + 32 * qq;
                const bool on = uv < NUV;
                // staging coordinates of this lane's row: U, V offsets in [-M, M]
                const int su = cell[U] + (uv % WIN), sv = cell[V] + (uv / WIN);
                const float gu = (float)(b0[U] - M + su), gv = (float)(b0[V] - M + sv);
                // face positions along F, in pairs: staging cell[F] + s - 1
                uint64_t gf2[NP];
#pragma unroll
                for (int h = 0; h < NP; ++h)
                    gf2[h] = f2_pack((float)(b0[F] - M + cell[F] + 2 * h), (float)(b0[F] - M + cell[F] + 2 * h + 1));
                const float gf0 = (float)(b0[F] - M + cell[F] - 1);
                double am[WIN], av[WIN];
#pragma unroll
                for (int s = 0; s < WIN; ++s) am[s] = av[s] = 0.0;
                // the cell's particles from the warp's staging slots, which
                // hold up to CAP consecutive particles of the tile (the 8 cells
                // of a tile are one contiguous range of the sorted order):
                // staged with coalesced loads, CAP / 32 per lane, then read by
                // broadcast
                for (int p0 = b; p0 < e;) {
                  if (p0 < st_lo || p0 >= st_hi) {
                      __syncwarp();
                      st_lo = p0;
                      st_hi = min(p0 + CAP, e_tile);
#pragma unroll
                      for (int k = 0; k < CAP / 32; ++k) {
                          const int pl = st_lo + lane + 32 * k;
                          if (pl < st_hi) {
                              const uint64_t f = lmask[pl];
                              const float m = a.pm[pl];
                              const size_t q = (size_t)pl * a.ps;
                              const float pc[3] = {a.px[q] - 0.5f, a.py[q] - 0.5f, a.pz[q] - 0.5f};
                              wslot[pl - st_lo] = make_float4(pc[U], pc[V], pc[F], m);
                              wslot[CAP + pl - st_lo] = make_float4(m * pv[q], __uint_as_float((uint32_t)f),
                                                                    __uint_as_float((uint32_t)(f >> 32)), 0.0f);
                          }
                      }
                      __syncwarp();
                  }
                  const int pend = min(e, st_hi);
                  for (int j = p0; j < pend; ++j) {
                    const float4 P = wslot[j - st_lo];        // U, V, F coordinates (minus 0.5), mass
                    const float4 R = wslot[CAP + j - st_lo];  // momentum, lane bits (low, high)
                    const uint32_t f_lo = __float_as_uint(R.y), f_hi = __float_as_uint(R.z);
                    // bit s: face s inside the footprint, none when the lane's
                    // row is outside it (no branch: the warp stays converged,
                    // and a zero weight adds +0 to a sum that starts at +0)
                    const uint32_t lanebit = on ? (((qq == 0 ? f_lo : f_hi) >> lane) & 1u) : 0u;
                    const uint32_t fbits = (f_hi >> 24) & (0u - lanebit);
                    const float m_p = P.w, scale_mom = R.x;
                    const float du = gu - P.x, dv = gv - P.y;
                    const uint64_t pf2 = f2_pack(P.z, P.z);
                    // p2g.rs:287-325: dz2 = dz*dz; dyz = dz2 + dy*dy; dist_sq = dx*dx + dyz,
                    // with (dx, dy, dz) = (df, du, dv), (du, df, dv) or (du, dv, df)
                    float hoist0 = 0.0f, hoist1 = 0.0f;
                    if (DIR == 0) hoist0 = dv * dv + du * du;  // dyz
                    else if (DIR == 1) { hoist0 = dv * dv; hoist1 = du * du; }  // dz2, dx*dx
                    else { hoist0 = dv * dv; hoist1 = du * du; }                // dy*dy, dx*dx
                    const uint64_t h02 = f2_pack(hoist0, hoist0), h12 = f2_pack(hoist1, hoist1);
#pragma unroll
                    for (int h = 0; h < NP; ++h) {
                        const uint64_t df = f2_sub(gf2[h], pf2);
                        // products that feed a sum stay scalar: a paired
                        // product feeding a paired sum may be contracted
                        float d0, d1;
                        f2_unpack(df, d0, d1);
                        const uint64_t sq = f2_pack(d0 * d0, d1 * d1);
                        uint64_t dist;
                        if (DIR == 0) dist = f2_add(sq, h02);                 // dx*dx + dyz
                        else if (DIR == 1) dist = f2_add(h12, f2_add(h02, sq));  // dx*dx + (dz2 + dy*dy)
                        else dist = f2_add(h12, f2_add(sq, h02));             // dx*dx + (dz2 + dy*dy)
                        const uint64_t df2 = f2_add(f2_add(dist, df), f2_pack(0.25f, 0.25f));
                        float e0, e1;
                        f2_unpack(df2, e0, e1);
                        const uint64_t t = f2_sub(f2_pack(1.0f, 1.0f), f2_pack(e0 * inv_r2, e1 * inv_r2));
                        float w0, w1;
                        f2_unpack(t, w0, w1);
                        w0 = ((fbits >> (2 * h + 1)) & 1u) ? fmaxf(w0, 0.0f) : 0.0f;
                        w1 = ((fbits >> (2 * h + 2)) & 1u) ? fmaxf(w1, 0.0f) : 0.0f;
                        uint64_t w = f2_pack(w0, w1);
                        w = f2_mul(f2_mul(w, w), w);
                        float tm0, tm1, tv0, tv1;
                        f2_unpack(f2_mul(w, f2_pack(m_p, m_p)), tm0, tm1);
                        f2_unpack(f2_mul(w, f2_pack(scale_mom, scale_mom)), tv0, tv1);
                        am[2 * h + 1] += (double)tm0;
                        av[2 * h + 1] += (double)tv0;
                        am[2 * h + 2] += (double)tm1;
                        av[2 * h + 2] += (double)tv1;
                    }
                    if ((f_hi >> 24) & 1u) {  // face 0: the same for every lane of the warp
                        const float df = gf0 - P.z;
                        const float sq = df * df;
                        float dist;
                        if (DIR == 0) dist = sq + hoist0;
                        else if (DIR == 1) dist = hoist1 + (hoist0 + sq);
                        else dist = hoist1 + (sq + hoist0);
                        const float df2 = (dist + df) + 0.25f;
                        float w = 1.0f - df2 * inv_r2;
                        w = (fbits & 1u) ? fmaxf(w, 0.0f) : 0.0f;
                        w = (w * w) * w;
                        am[0] += (double)(w * m_p);
                        av[0] += (double)(w * scale_mom);
                    }
                  }
                  p0 = pend;
                }
                if (deps_pending) wait_deps();
                if (on) {
#pragma unroll
                    for (int s = 0; s < WIN; ++s) {
                        const int sf = cell[F] + s - 1;
                        if (sf < 0 || sf >= W) continue;
                        int sc[3];
                        sc[F] = sf;
                        sc[U] = su;
                        sc[V] = sv;
                        const int si = (sc[2] * W + sc[1]) * W + sc[0];
                        st[si] += am[s];
                        st[WW + si] += av[s];
                    }
                }
            }
        }
        __syncwarp();
        __threadfence_block();
        if (lane == 0) *(volatile uint32_t*)&s_done[t] = 1u;
    }
    __syncthreads();
    double* out = a.partial + ((size_t)k_pb * 3 + DIR) * 2 * WW;
    for (int i = tid; i < 2 * WW; i += blockDim.x) out[i] = st[i];
}

// Splat for r_p = 2 (M = 2), grouped by footprint anchor.  With r_p = 2 the
// clipped footprint of a particle in cell c spans, along each lane axis (U,
// V), the four rows [c - 2 + s, c + 1 + s], s = 0 or 1 by the side of the
// cell centre the particle lies on, and along the face axis F the four faces
// [c - 2, c + 1] -- except when a coordinate lies exactly on a cell centre
// (lane axes) or a face plane (face axis).  Such a "regular" particle's
// footprint is fixed by its anchor (c_U + s_U, c_V + s_V, c_F): the particles
// of one anchor, drawn from four cells, share every footprint row, so a warp
// can keep its lanes' face sums in FP64 registers over all of them and add
// them into the window once.  The block's anchors (0 .. BSX along U and V,
// 0 .. BSX-1 along F) are cut into 2x2x2 anchor tiles; a tile draws its
// particles from 3 x 3 x 2 source cells.  Tile footprints are at most six
// rows wide, so tiles coloured by tile coordinate mod 3 never overlap within
// a colour, and the tile-order waits of p2g_cells_kernel apply unchanged.
// Per tile a warp stages its source cells' particles (each tagged with its
// anchor inside the tile), then takes the tile's eight anchors in turn: lane
// (i, j, h) evaluates faces 2h and 2h + 1 of footprint row (i, j) for every
// particle of the anchor and adds its two sums into the window afterwards.
// Irregular particles (footprint not of that shape) are tagged with their own
// cell and go through the lane-bit path of p2g_cells_kernel.  Every term is
// the reference's f32 operation sequence (p2g.rs:263-330); the sums are FP64
// in a fixed order (colour, tile, anchor, staging order).
// 24 warps with 160 staging slots each (a typical tile stages 144 particles)
// measured fastest on B200 among 16 x 192, 20 x 192, 24 x 160 and 28 x 128
// (6.02 against 7.02, 6.42 and 6.69 ms at 256^3).
constexpr int kSplatR2Warps = 24;
template <int BSX> struct SplatR2 {
    static constexpr int M = 2, W = BSX + 2 * M, WW = W * W * W;
    static constexpr int NA = BSX / 2 + 1;  // anchor tiles along U and V (anchors 0 .. BSX)
    static constexpr int NF = BSX / 2;      // anchor tiles along F
    static constexpr int NT = NA * NA * NF;
    static constexpr int NSRC = 18;         // source cells of a tile
    static constexpr int WARPS = NT < kSplatR2Warps ? NT : kSplatR2Warps;
    // particles a warp stages at once: a whole typical tile (144 at 8 per cell)
    static constexpr int CAP = 160;
    // per warp: CAP x (float4 position/mass, float momentum, u8 anchor-sorted
    // index), source cells (int2), 17 anchor-range offsets and 16 counters
    static constexpr size_t warp_bytes = (size_t)CAP * (16 + 4 + 1 + 1 + 1 + 1) + NSRC * 8 + 17 * 4 + 16 * 4;
    static constexpr size_t smem_bytes = 2 * sizeof(double) * WW + (size_t)WARPS * ((warp_bytes + 15) / 16 * 16);
    static_assert(NT < 0xffff, "tile indices must fit 16 bits");
    static_assert(CAP <= 256 && CAP % 32 == 0, "staging indices must fit a byte");
    static_assert(BSX <= 16, "source-cell Morton codes take 4 bits per axis");
};

// Morton code of a cell inside a block of at most 16^3 cells.
__device__ __forceinline__ uint32_t morton4(uint32_t x, uint32_t y, uint32_t z) {
    auto sp = [](uint32_t v) { return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4) | ((v & 8u) << 6); };
    return sp(x) | (sp(y) << 1) | (sp(z) << 2);
}

template <int BSX, int DIR>
__device__ __forceinline__ void splat_r2_body(const SplatArgs& a, const int k_pb, double* st, uint32_t* s_done,
                                              const uint16_t* s_order, uint32_t* s_next, const uint32_t (*s_dep)[4]) {
    using S = SplatR2<BSX>;
    constexpr int M = 2, W = S::W, WW = S::WW, NA = S::NA, NF = S::NF, NT = S::NT, CAP = S::CAP, NSRC = S::NSRC;
    constexpr int NNB = 125, NR = (NNB + 31) / 32;  // tile offsets in [-2, 2]^3, NR of them per lane
    constexpr int F = DIR, U = DIR == 0 ? 1 : 0, V = DIR == 2 ? 1 : 2;
    constexpr int kStride[3] = {1, W, W * W};  // window index step per axis
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    char* const wbase = reinterpret_cast<char*>(st + 2 * WW) + (size_t)warp * ((S::warp_bytes + 15) / 16 * 16);
    float4* const wp = reinterpret_cast<float4*>(wbase);                    // U, V, F coordinates - 0.5, mass
    float* const wm = reinterpret_cast<float*>(wbase + 16 * CAP);           // momentum m * v[DIR]
    int2* const wc = reinterpret_cast<int2*>(wbase + 20 * CAP);             // (first staging index, first particle)
    int* const woff = reinterpret_cast<int*>(wbase + 20 * CAP + NSRC * 8);  // anchor code ranges [16 + 1]
    int* const wcnt = woff + 17;                                            // per-code counters
    uint8_t* const wlist = reinterpret_cast<uint8_t*>(wcnt + 16);           // staging indices by anchor code
    int8_t* const wcode = reinterpret_cast<int8_t*>(wlist + CAP);            // anchor code per staging index
    uint8_t* const wsrc = reinterpret_cast<uint8_t*>(wcode + CAP);          // source cell per staging index
    uint8_t* const wrank = wsrc + CAP;                                      // rank inside its anchor code
    const uint64_t key = a.pb_key[k_pb];
    const int32_t b0[3] = {(int32_t)compact3(key) * BSX, (int32_t)compact3(key >> 1) * BSX,
                           (int32_t)compact3(key >> 2) * BSX};
    const int32_t* cb = a.cell_begin + (size_t)k_pb * BSX * BSX * BSX;
    const int32_t* ce = a.cell_end + (size_t)k_pb * BSX * BSX * BSX;
    const float* __restrict__ pv = a.pv[DIR];
    const uint64_t* __restrict__ lmask = a.lane_mask[DIR];
    const float inv_r2 = a.inv_r2;
    const uint32_t lt = [] { uint32_t m; asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m)); return m; }();
    // this lane's footprint row inside an anchor, (i, j) along (U, V), and
    // which two of the anchor's four faces along F it evaluates
    const int li = lane & 3, lj = (lane >> 2) & 3, half = lane >> 4;
    // this lane's tile offsets o = lane + 32 k in [-2, 2]^3, packed (ou + 2,
    // ov + 2, of + 2)
    uint32_t opk[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
        const int o = lane + 32 * k;
        opk[k] = (uint32_t)(o % 5) | ((uint32_t)((o / 5) % 5) << 8) | ((uint32_t)(o / 25) << 16);
    }
    while (true) {
        uint32_t q = 0;
        if (lane == 0) q = atomicAdd(s_next, 1u);
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= (uint32_t)NT) break;
        const int t = s_order[q];
        const int tu = t % NA, tv = (t / NA) % NA, tf = t / (NA * NA);
        const int ci = tu % 3 + 3 * (tv % 3 + 3 * (tf % 3));
        // source cells, one per lane: (2tu - 1 + c % 3, 2tv - 1 + (c / 3) % 3, 2tf + c / 9)
        int n_c = 0, b_c = 0;
        if (lane < NSRC) {
            const int cu = 2 * tu - 1 + lane % 3, cv = 2 * tv - 1 + (lane / 3) % 3, cf = 2 * tf + lane / 9;
            if (cu >= 0 && cu < BSX && cv >= 0 && cv < BSX) {
                int c3[3];
                c3[U] = cu;
                c3[V] = cv;
                c3[F] = cf;
                const uint32_t lm = morton4(c3[0], c3[1], c3[2]);
                b_c = cb[lm];
                n_c = ce[lm] - b_c;
            }
        }
        int incl = n_c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        __syncwarp();  // the previous tile's readers of wc are done
        if (lane < NSRC) wc[lane] = make_int2(incl - n_c, b_c);
        // the overlapping tiles of lower colours: each lane takes up to NR of
        // them; the warp waits for them before its first shared-memory add
        // of this tile, drops each as it is seen done, sleeps between rounds
        uint32_t nbi[(NR + 1) / 2];  // tile indices, two 16-bit fields per word, 0xffff = none
#pragma unroll
        for (int k = 0; k < (NR + 1) / 2; ++k) nbi[k] = 0xffffffffu;
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            // offsets of lower colour (per colour class, precomputed), inside the tile grid
            const bool lower = (s_dep[ci][k] >> lane) & 1u;
            const int nu = tu + (int)(opk[k] & 0xffu) - 2, nv = tv + (int)((opk[k] >> 8) & 0xffu) - 2,
                      nf = tf + (int)(opk[k] >> 16) - 2;
            const bool dep = lower && (unsigned)nu < (unsigned)NA && (unsigned)nv < (unsigned)NA && (unsigned)nf < (unsigned)NF;
            if (dep) nbi[k >> 1] &= ~(0xffffu << (16 * (k & 1))) | ((uint32_t)(nu + NA * (nv + NA * nf)) << (16 * (k & 1)));
        }
        bool deps_pending = true;
        auto wait_deps = [&]() {
            uint64_t t0 = 0;
            uint32_t spins = 0, sleep_ns = 32;
            while (true) {
                bool ready = true;
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    const uint32_t idx = (nbi[k >> 1] >> (16 * (k & 1))) & 0xffffu;
                    if (idx != 0xffffu) {
                        if (*(volatile uint32_t*)&s_done[idx]) nbi[k >> 1] |= 0xffffu << (16 * (k & 1));
                        else ready = false;
                    }
                }
                if (__all_sync(0xffffffffu, ready)) break;
                __nanosleep(sleep_ns);
                sleep_ns = sleep_ns < 512 ? 2 * sleep_ns : 512;
                if ((++spins & 63u) == 0) {
                    const uint64_t now = globaltimer_ns();
                    if (!t0) t0 = now;
                    else if (now - t0 > kWaitLimitNs) {
                        if (lane == 0) atomicOr(a.status, 4);
                        break;
                    }
                }
            }
            __threadfence_block();
            deps_pending = false;
        };
        // staging coordinates of this lane's row and first face for the
        // tile's first anchor, their global coordinates in f32, and the
        // window index
        const int su0 = 2 * tu + li, sv0 = 2 * tv + lj, sf0 = 2 * tf + 2 * half;
        const uint64_t guv0 = f2_pack((float)(b0[U] - M + su0), (float)(b0[V] - M + sv0));
        const uint64_t gf20 = f2_pack((float)(b0[F] - M + sf0), (float)(b0[F] - M + sf0 + 1));
        const int si0 = su0 * kStride[U] + sv0 * kStride[V] + sf0 * kStride[F];
        for (int s0 = 0; s0 < total; s0 += CAP) {
            const int ns = min(CAP, total - s0);
            __syncwarp();  // wc written; the previous chunk's readers of the slots are done
            if (lane < 16) wcnt[lane] = 0;
            // source cell of every staging index of the chunk
            if (lane < NSRC) {
                const int2 cc = wc[lane];
                const int lo = max(cc.x, s0), hi = min(cc.x + n_c, s0 + ns);
                for (int g = lo; g < hi; ++g) wsrc[g - s0] = (uint8_t)lane;
            }
            __syncwarp();
            // the anchor code of every staging index (from the lane-mask
            // shape bits alone) and its rank among the chunk's particles of
            // that code (staging order: ranks by lane inside each group of
            // 32, group counts added in order)
            uint32_t fbk[CAP / 32];  // shape bits of the lane masks, all loads issued at once
#pragma unroll
            for (int k = 0; k < CAP / 32; ++k) {
                const int s = lane + 32 * k;
                fbk[k] = 0;
                if (s < ns) {
                    const int2 cc = wc[wsrc[s]];
                    fbk[k] = (uint32_t)(lmask[cc.y + (s0 + s - cc.x)] >> 32);
                }
            }
#pragma unroll
            for (int k = 0; k < CAP / 32; ++k) {
                if (32 * k >= ns) break;
                const int s = lane + 32 * k;
                int code = -1;
                if (s < ns) {
                    const int c = wsrc[s];
                    const uint32_t fb = fbk[k];
                    // the anchor relative to the tile: source cell c sits at
                    // (c % 3 - 1, c / 3 % 3 - 1, c / 9) from the tile's first
                    // anchor; a regular particle's anchor is its cell shifted
                    // by (s_U, s_V), an irregular one's its cell
                    const bool regular = fb & 1u;
                    const int du = c % 3 - 1 + (regular ? (int)((fb >> 1) & 1u) : 0);
                    const int dv = (c / 3) % 3 - 1 + (regular ? (int)((fb >> 2) & 1u) : 0);
                    if ((unsigned)du <= 1u && (unsigned)dv <= 1u) code = du + 2 * dv + 4 * (c / 9) + (regular ? 0 : 8);
                }
                const uint32_t peers = __match_any_sync(0xffffffffu, code);
                const int before = code >= 0 ? wcnt[code] : 0;
                wcode[s] = (int8_t)code;
                wrank[s] = (uint8_t)(before + __popc(peers & lt));
                __syncwarp();
                if (code >= 0 && !(peers & lt)) wcnt[code] = before + __popc(peers);
                __syncwarp();
            }
            {
                const int c = lane < 16 ? wcnt[lane] : 0;
                int inc = c;
#pragma unroll
                for (int o = 1; o < 16; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= o) inc += v;
                }
                if (lane < 16) woff[lane + 1] = inc;
                if (lane == 0) woff[0] = 0;
            }
            __syncwarp();
            // the tile's own particles into their anchor-sorted slots
#pragma unroll 2
            for (int s = lane; s < ns; s += 32) {
                const int code = wcode[s];
                if (code < 0) continue;
                const int dst = woff[code] + wrank[s];
                const int2 cc = wc[wsrc[s]];
                const int pl = cc.y + (s0 + s - cc.x);
                const float m = a.pm[pl];
                const size_t q = (size_t)pl * a.ps;
                const float pp[3] = {a.px[q], a.py[q], a.pz[q]};
                wp[dst] = make_float4(pp[U] - 0.5f, pp[V] - 0.5f, pp[F] - 0.5f, m);
                wm[dst] = m * pv[q];
                wlist[dst] = (uint8_t)s;
            }
            __syncwarp();
#pragma unroll 1
            for (int al = 0; al < 8; ++al) {
                const int beg = woff[al], end = woff[al + 1];
                if (beg == end) continue;
                const int du = al & 1, dv = (al >> 1) & 1, df = al >> 2;
                // this lane's row and first face (exact small integers in f32)
                const uint64_t guv = f2_add(guv0, f2_pack((float)du, (float)dv));
                const uint64_t gf2 = f2_add(gf20, f2_pack((float)df, (float)df));
                double am0 = 0.0, am1 = 0.0, av0 = 0.0, av1 = 0.0;
                // the reference's terms of one particle for this lane's two faces
                auto terms = [&](int i, float& tm0, float& tm1, float& tv0, float& tv1) {
                    const float4 P = wp[i];
                    const float m_p = P.w, scale_mom = wm[i];
                    float duu, dvv;  // du * du, dv * dv (paired)
                    {
                        const uint64_t d2 = f2_sub(guv, f2_pack(P.x, P.y));
                        f2_unpack(f2_mul(d2, d2), duu, dvv);
                    }
                    // p2g.rs:287-325: dz2 = dz*dz; dyz = dz2 + dy*dy; dist_sq = dx*dx + dyz,
                    // with (dx, dy, dz) = (df, du, dv), (du, df, dv) or (du, dv, df)
                    float hoist0 = 0.0f, hoist1 = 0.0f;
                    if (DIR == 0) hoist0 = dvv + duu;
                    else { hoist0 = dvv; hoist1 = duu; }
                    const uint64_t dff = f2_sub(gf2, f2_pack(P.z, P.z));
                    float d0, d1;
                    f2_unpack(dff, d0, d1);
                    // products that feed a sum stay scalar: a paired product
                    // feeding a paired sum may be contracted
                    const uint64_t sq = f2_pack(d0 * d0, d1 * d1);
                    const uint64_t h02 = f2_pack(hoist0, hoist0);
                    uint64_t dist;
                    if (DIR == 0) dist = f2_add(sq, h02);
                    else if (DIR == 1) dist = f2_add(f2_pack(hoist1, hoist1), f2_add(h02, sq));
                    else dist = f2_add(f2_pack(hoist1, hoist1), f2_add(sq, h02));
                    const uint64_t df2 = f2_add(f2_add(dist, dff), f2_pack(0.25f, 0.25f));
                    float e0, e1;
                    f2_unpack(df2, e0, e1);
                    const uint64_t tt = f2_sub(f2_pack(1.0f, 1.0f), f2_pack(e0 * inv_r2, e1 * inv_r2));
                    float w0, w1;
                    f2_unpack(tt, w0, w1);
                    uint64_t w = f2_pack(fmaxf(w0, 0.0f), fmaxf(w1, 0.0f));
                    w = f2_mul(f2_mul(w, w), w);
                    f2_unpack(f2_mul(w, f2_pack(m_p, m_p)), tm0, tm1);
                    f2_unpack(f2_mul(w, f2_pack(scale_mom, scale_mom)), tv0, tv1);
                };
                // two particles per round (independent arithmetic), added in
                // list order
                int j = beg;
#pragma unroll 1
                for (; j + 1 < end; j += 2) {
                    float a0, a1, a2, a3, c0, c1, c2, c3;
                    terms(j, a0, a1, a2, a3);
                    terms(j + 1, c0, c1, c2, c3);
                    am0 += (double)a0;
                    am1 += (double)a1;
                    av0 += (double)a2;
                    av1 += (double)a3;
                    am0 += (double)c0;
                    am1 += (double)c1;
                    av0 += (double)c2;
                    av1 += (double)c3;
                }
                if (j < end) {
                    float a0, a1, a2, a3;
                    terms(j, a0, a1, a2, a3);
                    am0 += (double)a0;
                    am1 += (double)a1;
                    av0 += (double)a2;
                    av1 += (double)a3;
                }
                if (deps_pending) wait_deps();
                {
                    const int si = si0 + du * kStride[U] + dv * kStride[V] + df * kStride[F];
                    constexpr int step = kStride[F];
                    st[si] += am0;
                    st[WW + si] += av0;
                    st[si + step] += am1;
                    st[WW + si + step] += av1;
                }
                __syncwarp();  // anchors of a tile share faces: order their adds
            }
            // irregular particles (codes 8 .. 15, their own cell): lanes take
            // the 5 x 5 rows around the cell, faces by the lane bits
#pragma unroll 1
            for (int j = woff[8]; j < woff[16]; ++j) {
                if (deps_pending) wait_deps();
                int al = 8;
                while (woff[al + 1] <= j) ++al;
                const int jj = wlist[j];  // staging index
                const int2 cc = wc[wsrc[jj]];
                const int pl = cc.y + (s0 + jj - cc.x);
                const float4 P = wp[j];
                const float smom = wm[j];
                const uint64_t fb = lmask[pl];
                const uint32_t f_lo = (uint32_t)fb, f_hi = (uint32_t)(fb >> 32);
                int cell[3];  // the particle's cell inside the block
                cell[U] = 2 * tu + (al & 1);
                cell[V] = 2 * tv + ((al >> 1) & 1);
                cell[F] = 2 * tf + ((al >> 2) & 1);
                const bool on = lane < 25;
                const uint32_t lanebit = on ? ((f_lo >> lane) & 1u) : 0u;
                const uint32_t fbits = (f_hi >> 24) & (0u - lanebit);
                const int su = cell[U] + lane % 5, sv = cell[V] + lane / 5;
                const float du_ = (float)(b0[U] - M + su) - P.x, dv_ = (float)(b0[V] - M + sv) - P.y;
                float hoist0 = 0.0f, hoist1 = 0.0f;
                if (DIR == 0) hoist0 = dv_ * dv_ + du_ * du_;
                else { hoist0 = dv_ * dv_; hoist1 = du_ * du_; }
                if (on) {
#pragma unroll
                    for (int s = 0; s < 5; ++s) {
                        const int sf = cell[F] + s - 1;
                        if (sf < 0 || sf >= W || !((fbits >> s) & 1u)) continue;
                        const float dff = (float)(b0[F] - M + sf) - P.z;
                        const float sq = dff * dff;
                        float dist;
                        if (DIR == 0) dist = sq + hoist0;
                        else if (DIR == 1) dist = hoist1 + (hoist0 + sq);
                        else dist = hoist1 + (sq + hoist0);
                        const float df2 = (dist + dff) + 0.25f;
                        float w = fmaxf(1.0f - df2 * inv_r2, 0.0f);
                        w = (w * w) * w;
                        int sc[3];
                        sc[F] = sf;
                        sc[U] = su;
                        sc[V] = sv;
                        const int si = (sc[2] * W + sc[1]) * W + sc[0];
                        st[si] += (double)(w * P.w);
                        st[WW + si] += (double)(w * smom);
                    }
                }
                __syncwarp();
            }
        }
        __syncwarp();
        __threadfence_block();
        if (lane == 0) *(volatile uint32_t*)&s_done[t] = 1u;
    }
    __syncthreads();
    double* out = a.partial + ((size_t)k_pb * 3 + DIR) * 2 * WW;
    for (int i = tid; i < 2 * WW; i += blockDim.x) out[i] = st[i];
}

template <int BSX>
__global__ void __launch_bounds__(32 * kSplatR2Warps, 1) p2g_r2_kernel(SplatArgs a) {
    using S = SplatR2<BSX>;
    constexpr int WW = S::WW, NA = S::NA, NF = S::NF, NT = S::NT;
    extern __shared__ double st[];  // [2][W^3]: mass, momentum; then per-warp staging slots
    __shared__ uint32_t s_done[NT];
    __shared__ uint16_t s_order[NT];  // anchor tiles in colour-major order
    __shared__ uint32_t s_dep[27][4];  // per colour class: the tile offsets in [-2, 2]^3 of lower colour
    __shared__ uint32_t s_next;
    const int tid = threadIdx.x;
    for (int i = tid; i < 2 * WW; i += blockDim.x) st[i] = 0.0;
    for (int i = tid; i < 27 * 4; i += blockDim.x) {
        const int ci = i / 4, k = i % 4;
        const int cu = ci % 3, cv = (ci / 3) % 3, cf = ci / 9;
        uint32_t m = 0;
        for (int l = 0; l < 32; ++l) {
            const int o = l + 32 * k;
            if (o >= 125) break;
            const int nu = cu + 3 + o % 5 - 2, nv = cv + 3 + (o / 5) % 5 - 2, nf = cf + 3 + o / 25 - 2;
            if (nu % 3 + 3 * (nv % 3 + 3 * (nf % 3)) < ci) m |= 1u << l;
        }
        s_dep[ci][k] = m;
    }
    for (int t = tid; t < NT; t += blockDim.x) {
        s_done[t] = 0;
        const int tu = t % NA, tv = (t / NA) % NA, tf = t / (NA * NA);
        const int cu = tu % 3, cv = tv % 3, cf = tf % 3;
        const int ci = cu + 3 * (cv + 3 * cf);
        int base = 0;
        for (int c = 0; c < ci; ++c) {
            const int ou = c % 3, ov = (c / 3) % 3, of = c / 9;
            base += ((NA - ou + 2) / 3) * ((NA - ov + 2) / 3) * ((NF - of + 2) / 3);
        }
        const int nu = (NA - cu + 2) / 3, nv = (NA - cv + 2) / 3;
        s_order[base + tu / 3 + nu * (tv / 3 + nv * (tf / 3))] = (uint16_t)t;
    }
    if (tid == 0) s_next = 0;
    __syncthreads();
    const int k_pb = blockIdx.x / 3;
    switch (blockIdx.x % 3) {
        case 0: splat_r2_body<BSX, 0>(a, k_pb, st, s_done, s_order, &s_next, s_dep); break;
        case 1: splat_r2_body<BSX, 1>(a, k_pb, st, s_done, s_order, &s_next, s_dep); break;
        default: splat_r2_body<BSX, 2>(a, k_pb, st, s_done, s_order, &s_next, s_dep); break;
    }
}

// OR of the footprint masks over each particle block's particles, expanded to
// candidate block ids (n_blocks = "none").
__global__ void pb_candidates_kernel(const uint32_t* fmask, const uint64_t* pb_starts, const uint64_t* pb_key, size_t npb,
                                     int64_t nx, int64_t ny, int64_t nz, uint64_t* cand) {
    for (size_t k = blockIdx.x; k < npb; k += gridDim.x) {
        uint32_t m = 0;
        const uint32_t* f = fmask + pb_starts[k];
        const uint32_t cnt = (uint32_t)(pb_starts[k + 1] - pb_starts[k]);  // particles of one block
#pragma unroll 4
        for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) m |= f[i];
        for (int o = 16; o; o >>= 1) m |= __shfl_xor_sync(0xffffffffu, m, o);
        __shared__ uint32_t wm[32];
        if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x < 27) {
            uint32_t all = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) all |= wm[w];
            const uint64_t key = pb_key[k];
            const int64_t X = (int64_t)compact3(key) + threadIdx.x % 3 - 1, Y = (int64_t)compact3(key >> 1) + (threadIdx.x / 3) % 3 - 1,
                          Z = (int64_t)compact3(key >> 2) + threadIdx.x / 9 - 1;
            const bool on = (all >> threadIdx.x) & 1u;
            cand[k * 27 + threadIdx.x] = on && X >= 0 && Y >= 0 && Z >= 0 && X < nx && Y < ny && Z < nz
                                             ? (uint64_t)X + (uint64_t)Y * nx + (uint64_t)Z * nx * ny
                                             : (uint64_t)(nx * ny * nz);
        }
        __syncthreads();
    }
}

// For every active block, the particle-block rank of each of its 27
// neighbours (binary search of the neighbour's Morton key among the sorted
// particle-block keys), or -1.
__global__ void active_nbr_kernel(const uint64_t* active, size_t n_active, const uint64_t* pb_key, size_t npb, int64_t nx,
                                  int64_t ny, int64_t nz, int32_t* nbr_rank) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n_active * 27; t += (size_t)gridDim.x * blockDim.x) {
        const size_t j = t / 27;
        const int d = (int)(t % 27);
        const uint64_t bid = active[j];
        const int64_t X = (int64_t)(bid % nx) + d % 3 - 1, Y = (int64_t)((bid / nx) % ny) + (d / 3) % 3 - 1,
                      Z = (int64_t)(bid / (nx * ny)) + d / 9 - 1;
        int32_t r = -1;
        if (X >= 0 && Y >= 0 && Z >= 0 && X < nx && Y < ny && Z < nz) {
            const uint64_t key = morton3(X, Y, Z);
            size_t lo = 0, hi = npb;
            while (lo < hi) {
                const size_t mid = (lo + hi) / 2;
                if (pb_key[mid] < key) lo = mid + 1;
                else hi = mid;
            }
            if (lo < npb && pb_key[lo] == key) r = (int32_t)lo;
        }
        nbr_rank[t] = r;
    }
}

static unsigned grid_for(size_t n) { return (unsigned)std::min<size_t>(std::max<size_t>(div_up(n, 256), 1), 8192); }

template <int BSX, int M, int DIR>
static void launch_splat_dir(msbg_ctx* ctx, const SplatArgs& a, size_t npb) {
    constexpr int W = BSX + 2 * M;
    constexpr int T = BSX / 2, NT = T * T * T;
    constexpr int WARPS = NT < kSplatWarps ? NT : kSplatWarps;
    const size_t smem = 2 * sizeof(double) * W * W * W + (size_t)WARPS * 2 * SplatCap<BSX, M>::v * sizeof(float4);
    static bool attr = false;
    if (!attr) {
        CUDA_CHECK(cudaFuncSetAttribute(p2g_cells_kernel<BSX, M, DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = true;
    }
    begin_launch(ctx);
    p2g_cells_kernel<BSX, M, DIR><<<(unsigned)npb, 32 * WARPS, smem, ctx->stream>>>(a);
    after_launch(ctx, "p2g_cells_kernel");
}

template <int BSX, int M>
static void launch_splat(msbg_ctx* ctx, const SplatArgs& a, size_t npb) {
    if (M == 2 && a.r_p == 2.0f) {
        constexpr int WARPS = SplatR2<BSX>::WARPS;
        const size_t smem = SplatR2<BSX>::smem_bytes;
        static bool attr = false;
        if (!attr) {
            CUDA_CHECK(cudaFuncSetAttribute(p2g_r2_kernel<BSX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr = true;
        }
        begin_launch(ctx);
        p2g_r2_kernel<BSX><<<(unsigned)(3 * npb), 32 * WARPS, smem, ctx->stream>>>(a);
        after_launch(ctx, "p2g_r2_kernel");
        return;
    }
    launch_splat_dir<BSX, M, 0>(ctx, a, npb);
    launch_splat_dir<BSX, M, 1>(ctx, a, npb);
    launch_splat_dir<BSX, M, 2>(ctx, a, npb);
}

template <int BSX, int M>
static void launch_combine(msbg_ctx* ctx, const CombineArgs& a, size_t n_active) {
    begin_launch(ctx);
    p2g_combine_kernel<BSX, M><<<dim3((unsigned)n_active, 3), 256, 0, ctx->stream>>>(a);
    after_launch(ctx, "p2g_combine_kernel");
}

template <int BSX>
static void dispatch_m(msbg_ctx* ctx, int M, const SplatArgs* s, size_t npb, const CombineArgs* c, size_t na) {
    switch (M) {
        case 1: if (s) launch_splat<BSX, 1>(ctx, *s, npb); else launch_combine<BSX, 1>(ctx, *c, na); break;
        case 2: if (s) launch_splat<BSX, 2>(ctx, *s, npb); else launch_combine<BSX, 2>(ctx, *c, na); break;
        default: if (s) launch_splat<BSX, 3>(ctx, *s, npb); else launch_combine<BSX, 3>(ctx, *c, na); break;
    }
}

static void dispatch(msbg_ctx* ctx, int bsx, int M, const SplatArgs* s, size_t npb, const CombineArgs* c, size_t na) {
    if (bsx == 8) dispatch_m<8>(ctx, M, s, npb, c, na);
    else dispatch_m<16>(ctx, M, s, npb, c, na);
}

static size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

// d_sorted_keys: optional sorted Morton keys (msbg_morton_sort_device); the
// internal sort is skipped.  With d_perm null the particle arrays are already
// in that order (msbg_permute_device); otherwise they are in the caller's
// order and d_perm[i] is the caller index of sorted particle i, which the
// gather follows.
void p2g_device(msbg_mac* mac, const float* d_pos, const float* d_vel, const float* d_mass, size_t n, float r_p,
                size_t* n_active_out, const uint64_t* d_sorted_keys, const uint32_t* d_perm) {
    msbg_ctx* ctx = mac->ctx;
    msbg_grid* u = mac->ch[0];
    const int bsx = u->bsx, lg = u->lg;
    MSBG_REQUIRE(bsx == 8 || bsx == 16, "P2G supports bsx 8 and 16");
    MSBG_REQUIRE(u->sx % bsx == 0 && u->sy % bsx == 0 && u->sz % bsx == 0, "P2G needs domain extents that are multiples of bsx");
    MSBG_REQUIRE(r_p > 0.0f && r_p <= 3.0f, "P2G supports 0 < r_p <= 3");
    const int M = (int)ceilf(r_p);
    MSBG_REQUIRE(2 * M <= bsx, "r_p too large for the block size");
    MSBG_REQUIRE(n < (1ULL << 31), "P2G supports < 2^31 particles");
    MSBG_REQUIRE(u->sx <= (1u << 21) && u->sy <= (1u << 21) && u->sz <= (1u << 21), "domain exceeds 21-bit Morton keys");
    const uint64_t smax = std::max(u->sx, std::max(u->sy, u->sz));
    const int key_bits = 3 * ilog2i(smax);
    const int W = bsx + 2 * M;
    const size_t WW = (size_t)W * W * W, NC = (size_t)bsx * bsx * bsx;
    if (n == 0) {
        mac->active.clear();
        if (n_active_out) *n_active_out = 0;
        return;
    }
    // ---- phase 1: sort, gather, particle blocks -------------------------------
    ScratchLayout L1;
    // the cell-sorted SoA copy exists only for particles in the caller's order
    const bool sorted_in_place = d_sorted_keys && !d_perm;
    const size_t o_keys = L1.add<uint64_t>(n), o_skeys = L1.add<uint64_t>(n), o_perm = L1.add<uint32_t>(n),
                 o_soa = L1.add<float>(sorted_in_place ? 1 : 7 * n), o_fm = L1.add<uint32_t>(n), o_fp = L1.add<uint64_t>(3 * n),
                 o_pbk = L1.add<uint64_t>(n + 1),
                 o_pbs = L1.add<uint64_t>(n + 2), o_tmp = L1.add<char>(std::max(radix_sort_scratch_bytes(n), segment_scratch_bytes(n))),
                 o_bad = L1.add<int>(4);
    // phase-2 buffers go after phase 1's (sized once npb is known)
    char* base = scratch(ctx, L1);
    uint64_t* keys = ScratchLayout::at<uint64_t>(base, o_keys);
    const uint64_t* skeys = ScratchLayout::at<uint64_t>(base, o_skeys);
    uint32_t* perm = ScratchLayout::at<uint32_t>(base, o_perm);
    float* soa = ScratchLayout::at<float>(base, o_soa);
    uint32_t* fmask = ScratchLayout::at<uint32_t>(base, o_fm);
    uint64_t* fpk = ScratchLayout::at<uint64_t>(base, o_fp);
    uint64_t* pb_key = ScratchLayout::at<uint64_t>(base, o_pbk);
    uint64_t* pb_starts = ScratchLayout::at<uint64_t>(base, o_pbs);
    int* bad = ScratchLayout::at<int>(base, o_bad);
    CUDA_CHECK(cudaMemsetAsync(bad, 0, 4, ctx->stream));
    if (d_sorted_keys) {
        skeys = d_sorted_keys;
        perm = const_cast<uint32_t*>(d_perm);
    } else {
        morton_keys(ctx, d_pos, n, keys);
        radix_sort_pairs(ctx, keys, nullptr, ScratchLayout::at<uint64_t>(base, o_skeys), perm, n, key_bits,
                         ScratchLayout::at<char>(base, o_tmp));
    }
    float *px = soa, *py = soa + n, *pz = soa + 2 * n, *pm = soa + 3 * n, *v0 = soa + 4 * n, *v1 = soa + 5 * n, *v2 = soa + 6 * n;
    begin_launch(ctx);
    if (M == 2)
        p2g_gather_kernel<2><<<grid_for(n), 256, 0, ctx->stream>>>(d_pos, d_vel, d_mass, perm, n, lg, M, r_p,
                                                                   (r_p + 1.0f) / (float)bsx, (int64_t)u->nx, (int64_t)u->ny,
                                                                   (int64_t)u->nz, px, py, pz, pm, v0, v1, v2, fmask, fpk, bad);
    else
        p2g_gather_kernel<0><<<grid_for(n), 256, 0, ctx->stream>>>(d_pos, d_vel, d_mass, perm, n, lg, M, r_p,
                                                                   (r_p + 1.0f) / (float)bsx, (int64_t)u->nx, (int64_t)u->ny,
                                                                   (int64_t)u->nz, px, py, pz, pm, v0, v1, v2, fmask, fpk, bad);
    after_launch(ctx, "p2g_gather_kernel");
    const size_t npb = sorted_segments(ctx, skeys, n, (uint64_t)(3 * lg), pb_key, pb_starts, ScratchLayout::at<char>(base, o_tmp));
    int hbad = 0, hstatus = 0;
    {
        SmallReads rd(ctx);
        rd.add(&hbad, bad, 4);
        rd.add(&hstatus, ctx->status.p, 4);
        rd.wait();
    }
    raise_device_status(ctx, hstatus);
    MSBG_REQUIRE(!hbad, "a particle lies outside the domain");

    // ---- phase 2: active set ------------------------------------------------
    ScratchLayout L2 = L1;
    const size_t o_cand = L2.add<uint64_t>(npb * 27), o_csort = L2.add<uint64_t>(npb * 27), o_cperm = L2.add<uint32_t>(npb * 27),
                 o_act = L2.add<uint64_t>(npb * 27 + 1), o_ast = L2.add<uint64_t>(npb * 27 + 2),
                 o_ctmp = L2.add<char>(std::max(radix_sort_scratch_bytes(npb * 27), segment_scratch_bytes(npb * 27))),
                 o_cb = L2.add<int32_t>(npb * NC), o_ce = L2.add<int32_t>(npb * NC), o_part = L2.add<double>(npb * 6 * WW);
    base = scratch(ctx, L2);  // may move: re-derive phase-1 pointers
    if (!d_sorted_keys) skeys = ScratchLayout::at<uint64_t>(base, o_skeys);
    fpk = ScratchLayout::at<uint64_t>(base, o_fp);
    soa = ScratchLayout::at<float>(base, o_soa);
    fmask = ScratchLayout::at<uint32_t>(base, o_fm);
    pb_key = ScratchLayout::at<uint64_t>(base, o_pbk);
    pb_starts = ScratchLayout::at<uint64_t>(base, o_pbs);
    px = soa; py = soa + n; pz = soa + 2 * n; pm = soa + 3 * n; v0 = soa + 4 * n; v1 = soa + 5 * n; v2 = soa + 6 * n;
    uint64_t* cand = ScratchLayout::at<uint64_t>(base, o_cand);
    uint64_t* csort = ScratchLayout::at<uint64_t>(base, o_csort);
    uint32_t* cperm = ScratchLayout::at<uint32_t>(base, o_cperm);
    uint64_t* act = ScratchLayout::at<uint64_t>(base, o_act);
    uint64_t* ast = ScratchLayout::at<uint64_t>(base, o_ast);
    int32_t* cell_begin = ScratchLayout::at<int32_t>(base, o_cb);
    int32_t* cell_end = ScratchLayout::at<int32_t>(base, o_ce);
    double* partial = ScratchLayout::at<double>(base, o_part);

    begin_launch(ctx);
    pb_candidates_kernel<<<(unsigned)std::min<size_t>(npb, 65535), 256, 0, ctx->stream>>>(
        fmask, pb_starts, pb_key, npb, (int64_t)u->nx, (int64_t)u->ny, (int64_t)u->nz, cand);
    after_launch(ctx, "pb_candidates_kernel");
    const int cbits = ilog2i(u->n_blocks + 1) + 1;
    radix_sort_pairs(ctx, cand, nullptr, csort, cperm, npb * 27, cbits, ScratchLayout::at<char>(base, o_ctmp));
    size_t nuniq = sorted_segments(ctx, csort, npb * 27, 0, act, ast, ScratchLayout::at<char>(base, o_ctmp));
    std::vector<uint64_t> active(nuniq);
    {
        SmallReads rd(ctx);
        rd.add(active.data(), act, nuniq * 8);
        rd.add(&hstatus, ctx->status.p, 4);
        rd.wait();
    }
    raise_device_status(ctx, hstatus);
    if (!active.empty() && active.back() == u->n_blocks) active.pop_back();  // the "none" sentinel
    const size_t na = active.size();
    std::vector<int32_t> slots(na);
    mac_ensure(mac, active.data(), na, slots.data());  // may grow the six payloads
    mac->active = active;

    // ---- phase 3: splat + combine -------------------------------------------
    ScratchLayout L3 = L2;
    const size_t o_nr = L3.add<int32_t>(na * 27), o_sl = L3.add<int32_t>(na);
    base = scratch(ctx, L3);
    if (!d_sorted_keys) skeys = ScratchLayout::at<uint64_t>(base, o_skeys);
    fpk = ScratchLayout::at<uint64_t>(base, o_fp);
    soa = ScratchLayout::at<float>(base, o_soa);
    pb_key = ScratchLayout::at<uint64_t>(base, o_pbk);
    pb_starts = ScratchLayout::at<uint64_t>(base, o_pbs);
    px = soa; py = soa + n; pz = soa + 2 * n; pm = soa + 3 * n; v0 = soa + 4 * n; v1 = soa + 5 * n; v2 = soa + 6 * n;
    act = ScratchLayout::at<uint64_t>(base, o_act);
    cell_begin = ScratchLayout::at<int32_t>(base, o_cb);
    cell_end = ScratchLayout::at<int32_t>(base, o_ce);
    partial = ScratchLayout::at<double>(base, o_part);
    int32_t* nbr_rank = ScratchLayout::at<int32_t>(base, o_nr);
    int32_t* d_slots = ScratchLayout::at<int32_t>(base, o_sl);
    CUDA_CHECK(cudaMemcpyAsync(d_slots, slots.data(), na * 4, cudaMemcpyHostToDevice, ctx->stream));

    begin_launch(ctx);
    cell_csr_kernel<<<(unsigned)npb, 256, 0, ctx->stream>>>(skeys, pb_starts, lg, cell_begin, cell_end);
    after_launch(ctx, "cell_csr_kernel");
    begin_launch(ctx);
    active_nbr_kernel<<<grid_for(na * 27), 256, 0, ctx->stream>>>(act, na, pb_key, npb, (int64_t)u->nx, (int64_t)u->ny,
                                                                  (int64_t)u->nz, nbr_rank);
    after_launch(ctx, "active_nbr_kernel");
    SplatArgs s;
    if (perm) {  // the gathered cell-sorted SoA
        s.px = px; s.py = py; s.pz = pz; s.pm = pm;
        s.pv[0] = v0; s.pv[1] = v1; s.pv[2] = v2;
        s.ps = 1;
    } else {  // already sorted: the caller's arrays in place
        s.px = d_pos; s.py = d_pos + 1; s.pz = d_pos + 2; s.pm = d_mass;
        s.pv[0] = d_vel; s.pv[1] = d_vel + 1; s.pv[2] = d_vel + 2;
        s.ps = 3;
    }
    s.cell_begin = cell_begin;
    s.cell_end = cell_end;
    s.pb_key = pb_key;
    for (int d = 0; d < 3; ++d) s.lane_mask[d] = fpk + (size_t)d * n;
    s.status = ctx->status.as<int>();
    s.partial = partial;
    s.r_p = r_p;
    s.inv_r2 = 1.0f / (r_p * r_p);
    dispatch(ctx, bsx, M, &s, npb, nullptr, 0);
    CombineArgs c;
    c.partial = partial;
    c.nbr_rank = nbr_rank;
    c.active = act;
    c.slots = d_slots;
    for (int a = 0; a < 3; ++a) {
        c.vel[a] = mac->ch[a]->payload.as<float>();
        c.mass[a] = mac->ch[3 + a]->payload.as<float>();
    }
    c.nx = (int64_t)u->nx;
    c.ny = (int64_t)u->ny;
    if (na) dispatch(ctx, bsx, M, nullptr, 0, &c, na);
    read_small(ctx, &hstatus, ctx->status.p, 4);  // waits: `slots` (host) and the scratch layout end here
    raise_device_status(ctx, hstatus);
    if (n_active_out) *n_active_out = na;
    (void)a256;
}

}  // namespace msbg

using namespace msbg;

extern "C" {

int msbg_p2g_device(msbg_mac* m, const float* d_pos, const float* d_vel, const float* d_mass, size_t n, float r_p,
                    size_t* n_active_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && ((d_pos && d_vel && d_mass) || !n), "null argument");
    set_device(m->ctx);
    p2g_device(m, d_pos, d_vel, d_mass, n, r_p, n_active_out, nullptr, nullptr);
    MSBG_API_END
}

int msbg_p2g_sorted_device(msbg_mac* m, const float* d_pos, const float* d_vel, const float* d_mass,
                           const uint64_t* d_keys, size_t n, float r_p, size_t* n_active_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && ((d_pos && d_vel && d_mass && d_keys) || !n), "null argument");
    set_device(m->ctx);
    p2g_device(m, d_pos, d_vel, d_mass, n, r_p, n_active_out, d_keys, nullptr);
    MSBG_API_END
}

int msbg_p2g_permuted_device(msbg_mac* m, const float* d_pos, const float* d_vel, const float* d_mass,
                             const uint64_t* d_keys, const uint32_t* d_perm, size_t n, float r_p, size_t* n_active_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && ((d_pos && d_vel && d_mass && d_keys && d_perm) || !n), "null argument");
    set_device(m->ctx);
    p2g_device(m, d_pos, d_vel, d_mass, n, r_p, n_active_out, d_keys, d_perm);
    MSBG_API_END
}

int msbg_p2g(msbg_mac* m, const float* pos, const float* vel, const float* mass, size_t n, float r_p, size_t* n_active_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && ((pos && vel && mass) || !n), "null argument");
    set_device(m->ctx);
    DevBuf io;
    const size_t b3 = (n * 12 + 255) & ~size_t(255), b1 = (n * 4 + 255) & ~size_t(255);
    io.reserve(2 * b3 + b1 + 256);
    float* dp = io.as<float>();
    float* dv = (float*)((char*)io.p + b3);
    float* dm = (float*)((char*)io.p + 2 * b3);
    if (n) {
        CUDA_CHECK(cudaMemcpyAsync(dp, pos, n * 12, cudaMemcpyHostToDevice, m->ctx->stream));
        CUDA_CHECK(cudaMemcpyAsync(dv, vel, n * 12, cudaMemcpyHostToDevice, m->ctx->stream));
        CUDA_CHECK(cudaMemcpyAsync(dm, mass, n * 4, cudaMemcpyHostToDevice, m->ctx->stream));
    }
    p2g_device(m, dp, dv, dm, n, r_p, n_active_out, nullptr, nullptr);
    sync(m->ctx);
    MSBG_API_END
}

}  // extern "C"
