// surface.cu -- surface reconstruction from particles (particles/mod.rs:220-302):
// instanced placement (particles/sort.rs:31-144), the min-splat of normalised
// squared distances (particles/splat.rs:92-319), finalize to a [0, 1]
// density (particles/finalize.rs:35-71) and the mean-curvature smoothing of
// reconstruct_and_smooth.
//
// Splat on the device: particles are Morton-sorted, so each 16^3 block's
// particles are one contiguous range ("particle blocks").  One CTA per
// particle block stages its (bsx + 2m)^3 window (m = ceil(r_scan)) in shared
// memory as 32-bit words (the quantised Density value, or the bits of the
// non-negative f32 ratio, whose order is the float order) and takes the
// minimum with shared atomics; the window's touched voxels are then committed
// with global atomic minima into a 32-bit field over the grid's slots, which a
// last kernel converts into the grid's payload.  A minimum does not depend on
// the order of its operands, so the result is deterministic and equals the
// crate's staged, colour-ordered commit bit for bit.
#include <algorithm>

#include "grid.cuh"
#include "sort.cuh"

namespace msbg {

struct SurfArgs {
    const float* pos;          // Morton-sorted [n][3]
    const uint64_t* pb_key;    // per particle block: its block's Morton key
    const uint64_t* pb_starts; // [npb + 1]
    uint32_t* minfield;        // [slots][bsx^3]
    const int32_t* dense;      // bid -> slot code, or null (hash)
    DevHash hash;
    int64_t sx, sy, sz, nx, ny;
    int lg, m, W;
    float r_scan, dmax, inv;
    int qmax;                  // stored integer scale: 65535 Density, 255 Density8, 0 f32
    uint32_t full;
};

__device__ __forceinline__ int32_t surf_code(const SurfArgs& a, uint64_t bid) {
    return a.dense ? a.dense[bid] : hash_find(a.hash, bid);
}

// Per particle: its footprint blocks (particles/mod.rs:202-212 footprint_axis,
// reach r_scan) relative to its own block, as a 27-bit mask (r_scan < bsx).
__global__ void sf_footprint_kernel(const float* __restrict__ pos, size_t n, int lg, float r_scan_bsx, int64_t nx,
                                    int64_t ny, int64_t nz, uint32_t* __restrict__ fmask) {
    const float bsx = (float)(1 << lg);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        const int64_t nn[3] = {nx, ny, nz};
        uint32_t lo[3], hi[3];
        for (int ax = 0; ax < 3; ++ax) {
            const int64_t cb = (int64_t)(p[ax] > 0.0f ? (int32_t)p[ax] : 0) >> lg;
            const float b = p[ax] / bsx;
            const int64_t l = max((int64_t)(int32_t)truncf(b - r_scan_bsx), (int64_t)0);
            const int64_t h = min((int64_t)(int32_t)truncf(b + r_scan_bsx), nn[ax] - 1);
            lo[ax] = (uint32_t)(min(max(l - cb, (int64_t)-1), (int64_t)1) + 1);
            hi[ax] = (uint32_t)(min(max(h - cb, (int64_t)-1), (int64_t)1) + 1);
        }
        uint32_t m = 0;
        for (uint32_t dz = lo[2]; dz <= hi[2]; ++dz)
            for (uint32_t dy = lo[1]; dy <= hi[1]; ++dy)
                for (uint32_t dx = lo[0]; dx <= hi[0]; ++dx) m |= 1u << (dx + 3 * dy + 9 * dz);
        fmask[i] = m;
    }
}

// OR of each particle block's masks, expanded to candidate bids (n_blocks = none).
__global__ void sf_candidates_kernel(const uint32_t* __restrict__ fmask, const uint64_t* __restrict__ pb_starts,
                                     const uint64_t* __restrict__ pb_key, size_t npb, int64_t nx, int64_t ny, int64_t nz,
                                     uint64_t* __restrict__ cand) {
    __shared__ uint32_t wm[32];
    for (size_t k = blockIdx.x; k < npb; k += gridDim.x) {
        uint32_t m = 0;
        for (uint64_t i = pb_starts[k] + threadIdx.x; i < pb_starts[k + 1]; i += blockDim.x) m |= fmask[i];
        for (int o = 16; o; o >>= 1) m |= __shfl_xor_sync(0xffffffffu, m, o);
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

__global__ void sf_fill_kernel(uint32_t* __restrict__ f, size_t n, uint32_t v) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) f[i] = v;
}

// One CTA per particle block: stage (min in shared memory), then commit the
// touched window voxels (global atomic min).  Each warp takes a particle; its
// lanes take the footprint rows (iy, iz) and walk x, evaluating the crate's
// f32 distance in its order (splat.rs:217-250: dz2 = dz dz, dyz = dz2 + dy dy,
// dist_sq = dx dx + dyz) and quantising as channel.rs:392-417.
__global__ void __launch_bounds__(256) sf_splat_kernel(SurfArgs a) {
    extern __shared__ uint32_t win[];
    const int W = a.W, WW = W * W * W, bsx = 1 << a.lg, m = a.m;
    for (int i = threadIdx.x; i < WW; i += blockDim.x) win[i] = a.full;
    const uint64_t key = a.pb_key[blockIdx.x];
    const int32_t b0[3] = {(int32_t)compact3(key) * bsx, (int32_t)compact3(key >> 1) * bsx, (int32_t)compact3(key >> 2) * bsx};
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint64_t s = a.pb_starts[blockIdx.x], e = a.pb_starts[blockIdx.x + 1];
    for (uint64_t i = s + warp; i < e; i += nw) {
        const float p[3] = {a.pos[3 * i], a.pos[3 * i + 1], a.pos[3 * i + 2]};
        int32_t lo[3], hi[3];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            lo[ax] = min(max((int32_t)ceilf((p[ax] - a.r_scan) - 0.5f), b0[ax] - m), b0[ax] + bsx + m - 1);
            hi[ax] = min(max((int32_t)floorf((p[ax] + a.r_scan) - 0.5f), b0[ax] - m), b0[ax] + bsx + m - 1);
        }
        const float px0 = p[0] - 0.5f, py0 = p[1] - 0.5f, pz0 = p[2] - 0.5f;
        const int ny_ = hi[1] - lo[1] + 1, nrows = ny_ * (hi[2] - lo[2] + 1);
        for (int r = lane; r < nrows; r += 32) {
            const int iy = lo[1] + r % ny_, iz = lo[2] + r / ny_;
            const float dz = (float)iz - pz0;
            const float dz2 = dz * dz;
            const float dy = (float)iy - py0;
            const float dyz = dz2 + dy * dy;
            const int row = ((iz - (b0[2] - m)) * W + (iy - (b0[1] - m))) * W - (b0[0] - m);  // + ix >= 0
            for (int ix = lo[0]; ix <= hi[0]; ++ix) {
                const float dx = (float)ix - px0;
                const float d2 = dx * dx + dyz;
                if (d2 <= a.dmax) {
                    const float t = d2 * a.inv;
                    const uint32_t q = a.qmax ? ((uint32_t)(int32_t)roundf(t * (float)a.qmax) & (uint32_t)a.qmax)
                                              : __float_as_uint(t);
                    atomicMin(win + row + ix, q);
                }
            }
        }
    }
    __syncthreads();
    const int N = bsx * bsx * bsx, msk = bsx - 1;
    for (int i = threadIdx.x; i < WW; i += blockDim.x) {
        const uint32_t v = win[i];
        if (v == a.full) continue;
        const int64_t gx = b0[0] - m + i % W, gy = b0[1] - m + (i / W) % W, gz = b0[2] - m + i / (W * W);
        if (gx < 0 || gy < 0 || gz < 0 || gx >= a.sx || gy >= a.sy || gz >= a.sz) continue;
        const int32_t code = surf_code(a, (uint64_t)(gx >> a.lg) + (uint64_t)(gy >> a.lg) * a.nx +
                                              (uint64_t)(gz >> a.lg) * a.nx * a.ny);
        if (code < 0) continue;
        atomicMin(a.minfield + (size_t)code * N + ((gx & msk) | ((gy & msk) << a.lg) | ((gz & msk) << (2 * a.lg))), v);
    }
}

// The min field of the listed slots into the grid payload (u16, u8 or f32).
__global__ void sf_writeback_kernel(const uint32_t* __restrict__ f, const int32_t* __restrict__ slots, size_t n_slots,
                                    int N, int qmax, void* payload) {
    const size_t total = n_slots * (size_t)N;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t k = i / N, v = i % N;
        const size_t at = (size_t)slots[k] * N + v;
        const uint32_t x = f[at];
        if (qmax == 65535) static_cast<uint16_t*>(payload)[at] = (uint16_t)x;
        else if (qmax == 255) static_cast<uint8_t*>(payload)[at] = (uint8_t)x;
        else static_cast<float*>(payload)[at] = __uint_as_float(x);
    }
}

// finalize.rs:35-71 on the listed slots, in place: ratio = dequantised value,
// touched = ratio < 0.999, f = 1 - clamp((sqrt(ratio r^2) - r_p + r_p) /
// (2 r_p + nb), 0, 1), 0 when untouched; Density / Density8 read q * inv_q
// (Quant::dequant_chunk) and store round(f * qmax) (Quant::quant_chunk,
// channel.rs:303-447).
__global__ void sf_finalize_kernel(const int32_t* __restrict__ slots, size_t n_slots, int N, int qmax, float inv_q,
                                   void* payload, float dmax, float r_particle, float denom) {
    const size_t total = n_slots * (size_t)N;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t at = (size_t)slots[i / N] * N + i % N;
        const float ratio = qmax == 65535 ? __fmul_rn((float)static_cast<uint16_t*>(payload)[at], inv_q)
                            : qmax == 255 ? __fmul_rn((float)static_cast<uint8_t*>(payload)[at], inv_q)
                                          : static_cast<float*>(payload)[at];
        const bool touched = ratio < 0.999f;
        const float dist = __fsqrt_rn(ratio * dmax) - r_particle;
        float t = __fdiv_rn(dist + r_particle, denom);
        t = fminf(fmaxf(t, 0.0f), 1.0f);
        const float f = touched ? 1.0f - t : 0.0f;
        if (qmax == 65535) static_cast<uint16_t*>(payload)[at] = (uint16_t)(int32_t)roundf(__fmul_rn(f, 65535.0f));
        else if (qmax == 255) static_cast<uint8_t*>(payload)[at] = (uint8_t)(int32_t)roundf(__fmul_rn(f, 255.0f));
        else static_cast<float*>(payload)[at] = f;
    }
}

// particles/sort.rs:31-144 place over (instance i, base point j) pairs:
// keep[i n_base + j] = 1 when the placed point lies in the domain bounds and
// its truncated cell in the grid; pass 2 writes the kept points in
// instance-major order at their exclusive-scan offsets.
struct PlaceArgs {
    const float* base;
    int64_t n_base, n_inst;
    float bbox[3], dom_min[3], dom_max[3];
    float smax, base_scale, inst_scale;
    int64_t sx, sy, sz;
};

__device__ __forceinline__ bool place_point(const PlaceArgs& a, int64_t i, int64_t j, float p[3]) {
    bool in = true;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const float origin = 0.2f * a.smax + ((0.6f * a.smax) * a.base_scale) * (a.base[3 * i + ax] - a.bbox[ax]);
        p[ax] = origin + a.inst_scale * (a.base[3 * j + ax] - a.bbox[ax]);
        if (!(p[ax] >= a.dom_min[ax] && p[ax] <= a.dom_max[ax])) in = false;
    }
    const int64_t dims[3] = {a.sx, a.sy, a.sz};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int32_t ip = (int32_t)p[ax];
        if (ip < 0 || ip >= dims[ax]) in = false;
    }
    return in;
}

__global__ void sf_place_flags_kernel(PlaceArgs a, uint32_t* __restrict__ keep) {
    const int64_t total = a.n_inst * a.n_base;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        float p[3];
        keep[t] = place_point(a, t / a.n_base, t % a.n_base, p) ? 1u : 0u;
    }
}

__global__ void sf_place_write_kernel(PlaceArgs a, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ off,
                                      float* __restrict__ out) {
    const int64_t total = a.n_inst * a.n_base;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        if (!keep[t]) continue;
        float p[3];
        place_point(a, t / a.n_base, t % a.n_base, p);
        const size_t o = off[t];
        out[3 * o] = p[0];
        out[3 * o + 1] = p[1];
        out[3 * o + 2] = p[2];
    }
}

static unsigned sf_grid(size_t n) { return (unsigned)std::min<size_t>(std::max<size_t>(div_up(n, 256), 1), 148 * 16); }

static void check(int st) {
    if (st != MSBG_OK) MSBG_THROW(st, msbg_last_error());
}

static int surface_qmax(const msbg_grid* g) { return g->dtype == MSBG_U16 ? 65535 : g->dtype == MSBG_U8 ? 255 : 0; }

static void surface_checks(msbg_grid* g, float r_particle, float nb_dist) {
    MSBG_REQUIRE(g->dtype == MSBG_F32 || g->dtype == MSBG_U16 || g->dtype == MSBG_U8,
                 "surface grids hold f32, Density (u16) or Density8 (u8) values");
    MSBG_REQUIRE(g->sx % g->bsx == 0 && g->sy % g->bsx == 0 && g->sz % g->bsx == 0,
                 "the surface splat needs domain extents that are multiples of bsx");
    MSBG_REQUIRE(r_particle > 0.0f && nb_dist >= 0.0f, "r_particle must be > 0 and nb_dist >= 0");
    const float r_scan = r_particle + nb_dist;
    MSBG_REQUIRE(r_scan + 0.5f < (float)g->bsx, "r_particle + nb_dist must be below bsx - 1/2 (8-colour splat)");
    const int m = (int)ceilf(r_scan), W = g->bsx + 2 * m;
    MSBG_REQUIRE((size_t)W * W * W * 4 <= 200 * 1024, "splat window too large for shared memory");
    MSBG_REQUIRE(g->sx <= (1u << 21) && g->sy <= (1u << 21) && g->sz <= (1u << 21), "domain exceeds 21-bit Morton keys");
}

// Returns the active bids (sorted); the grid holds the splatted field there.
static std::vector<uint64_t> surface_splat(msbg_grid* g, const float* d_pos, size_t n, float r_particle, float nb_dist) {
    msbg_ctx* ctx = g->ctx;
    surface_checks(g, r_particle, nb_dist);
    std::vector<uint64_t> active;
    if (!n) return active;
    MSBG_REQUIRE(n < (1ULL << 31), "the surface splat supports < 2^31 particles");
    const int lg = g->lg, bsx = g->bsx;
    const float r_scan = r_particle + nb_dist;
    const int key_bits = 3 * ilog2i(std::max(g->sx, std::max(g->sy, g->sz)));
    // ---- sort, particle blocks, footprints -------------------------------
    ScratchLayout L1;
    const size_t o_keys = L1.add<uint64_t>(n), o_sk = L1.add<uint64_t>(n), o_perm = L1.add<uint32_t>(n),
                 o_sp = L1.add<float>(3 * n), o_fm = L1.add<uint32_t>(n), o_pbk = L1.add<uint64_t>(n + 1),
                 o_pbs = L1.add<uint64_t>(n + 2),
                 o_tmp = L1.add<char>(std::max(radix_sort_scratch_bytes(n), segment_scratch_bytes(n)));
    char* base = scratch(ctx, L1);
    morton_keys(ctx, d_pos, n, ScratchLayout::at<uint64_t>(base, o_keys));
    radix_sort_pairs(ctx, ScratchLayout::at<uint64_t>(base, o_keys), nullptr, ScratchLayout::at<uint64_t>(base, o_sk),
                     ScratchLayout::at<uint32_t>(base, o_perm), n, key_bits, ScratchLayout::at<char>(base, o_tmp));
    check(msbg_permute_device(ctx, ScratchLayout::at<uint32_t>(base, o_perm), n, 3, d_pos, ScratchLayout::at<float>(base, o_sp)));
    begin_launch(ctx);
    sf_footprint_kernel<<<sf_grid(n), 256, 0, ctx->stream>>>(ScratchLayout::at<float>(base, o_sp), n, lg, r_scan / (float)bsx,
                                                             (int64_t)g->nx, (int64_t)g->ny, (int64_t)g->nz,
                                                             ScratchLayout::at<uint32_t>(base, o_fm));
    after_launch(ctx, "sf_footprint_kernel");
    const size_t npb = sorted_segments(ctx, ScratchLayout::at<uint64_t>(base, o_sk), n, (uint64_t)(3 * lg),
                                       ScratchLayout::at<uint64_t>(base, o_pbk), ScratchLayout::at<uint64_t>(base, o_pbs),
                                       ScratchLayout::at<char>(base, o_tmp));
    // ---- active set: union of the particle blocks' footprints --------------
    ScratchLayout L2 = L1;
    const size_t o_cand = L2.add<uint64_t>(npb * 27), o_cs = L2.add<uint64_t>(npb * 27), o_cp = L2.add<uint32_t>(npb * 27),
                 o_act = L2.add<uint64_t>(npb * 27 + 1), o_ast = L2.add<uint64_t>(npb * 27 + 2),
                 o_ctmp = L2.add<char>(std::max(radix_sort_scratch_bytes(npb * 27), segment_scratch_bytes(npb * 27)));
    base = scratch(ctx, L2);
    begin_launch(ctx);
    sf_candidates_kernel<<<(unsigned)std::min<size_t>(npb, 65535), 256, 0, ctx->stream>>>(
        ScratchLayout::at<uint32_t>(base, o_fm), ScratchLayout::at<uint64_t>(base, o_pbs),
        ScratchLayout::at<uint64_t>(base, o_pbk), npb, (int64_t)g->nx, (int64_t)g->ny, (int64_t)g->nz,
        ScratchLayout::at<uint64_t>(base, o_cand));
    after_launch(ctx, "sf_candidates_kernel");
    radix_sort_pairs(ctx, ScratchLayout::at<uint64_t>(base, o_cand), nullptr, ScratchLayout::at<uint64_t>(base, o_cs),
                     ScratchLayout::at<uint32_t>(base, o_cp), npb * 27, ilog2i(g->n_blocks + 1) + 1,
                     ScratchLayout::at<char>(base, o_ctmp));
    const size_t nuniq = sorted_segments(ctx, ScratchLayout::at<uint64_t>(base, o_cs), npb * 27, 0,
                                         ScratchLayout::at<uint64_t>(base, o_act), ScratchLayout::at<uint64_t>(base, o_ast),
                                         ScratchLayout::at<char>(base, o_ctmp));
    active.resize(nuniq);
    int hstatus = 0;
    {
        SmallReads rd(ctx);
        rd.add(active.data(), ScratchLayout::at<uint64_t>(base, o_act), nuniq * 8);
        rd.add(&hstatus, ctx->status.p, 4);
        rd.wait();
    }
    raise_device_status(ctx, hstatus);
    if (!active.empty() && active.back() == g->n_blocks) active.pop_back();
    // ---- allocate the active blocks, stage + commit, write back ------------
    std::vector<int32_t> slots(active.size());
    grid_ensure(g, active.data(), active.size(), slots.data());
    const int m = (int)ceilf(r_scan), W = bsx + 2 * m, N = bsx * bsx * bsx;
    ScratchLayout L3 = L2;
    const size_t o_min = L3.add<uint32_t>(g->n_slots() * (size_t)N), o_sl = L3.add<int32_t>(active.size());
    base = scratch(ctx, L3);
    const int qmax = surface_qmax(g);
    const uint32_t full = qmax ? (uint32_t)qmax : 0x3f800000u;  // Density(u16::MAX), Density8(u8::MAX) or 1.0f
    uint32_t* minfield = ScratchLayout::at<uint32_t>(base, o_min);
    int32_t* d_slots = ScratchLayout::at<int32_t>(base, o_sl);
    CUDA_CHECK(cudaMemcpyAsync(d_slots, slots.data(), slots.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    begin_launch(ctx);
    sf_fill_kernel<<<sf_grid(g->n_slots() * N), 256, 0, ctx->stream>>>(minfield, g->n_slots() * (size_t)N, full);
    after_launch(ctx, "sf_fill_kernel");
    SurfArgs a;
    a.pos = ScratchLayout::at<float>(base, o_sp);
    a.pb_key = ScratchLayout::at<uint64_t>(base, o_pbk);
    a.pb_starts = ScratchLayout::at<uint64_t>(base, o_pbs);
    a.minfield = minfield;
    a.dense = device_dense(g);
    a.hash = device_hash(g);
    a.sx = (int64_t)g->sx; a.sy = (int64_t)g->sy; a.sz = (int64_t)g->sz;
    a.nx = (int64_t)g->nx; a.ny = (int64_t)g->ny;
    a.lg = lg; a.m = m; a.W = W;
    a.r_scan = r_scan;
    a.dmax = r_scan * r_scan;
    a.inv = 1.0f / a.dmax;
    a.qmax = qmax;
    a.full = full;
    const size_t smem = (size_t)W * W * W * 4;
    CUDA_CHECK(cudaFuncSetAttribute(sf_splat_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    begin_launch(ctx);
    sf_splat_kernel<<<(unsigned)npb, 256, smem, ctx->stream>>>(a);
    after_launch(ctx, "sf_splat_kernel");
    if (!active.empty()) {
        begin_launch(ctx);
        sf_writeback_kernel<<<sf_grid(active.size() * N), 256, 0, ctx->stream>>>(minfield, d_slots, active.size(), N,
                                                                               a.qmax, g->payload.p);
        after_launch(ctx, "sf_writeback_kernel");
    }
    sync(ctx);  // slots (host) and the scratch layout end here
    return active;
}

static void surface_finalize(msbg_grid* g, const uint64_t* active, size_t n, float r_particle, float nb_dist) {
    msbg_ctx* ctx = g->ctx;
    surface_checks(g, r_particle, nb_dist);
    if (!n) return;
    std::vector<int32_t> slots(n);
    for (size_t i = 0; i < n; ++i) {
        auto it = g->map.find(active[i]);
        MSBG_REQUIRE(it != g->map.end() && it->second >= 0, "finalize: a listed block is not a value block of the grid");
        slots[i] = it->second;
    }
    ScratchLayout L;
    const size_t o_sl = L.add<int32_t>(n);
    char* base = scratch(ctx, L);
    int32_t* d_slots = ScratchLayout::at<int32_t>(base, o_sl);
    CUDA_CHECK(cudaMemcpyAsync(d_slots, slots.data(), n * 4, cudaMemcpyHostToDevice, ctx->stream));
    const float r_scan = r_particle + nb_dist;
    const int N = g->bsx * g->bsx * g->bsx;
    begin_launch(ctx);
    const int qmax = surface_qmax(g);
    sf_finalize_kernel<<<sf_grid(n * N), 256, 0, ctx->stream>>>(d_slots, n, N, qmax, qmax ? 1.0f / (float)qmax : 0.0f,
                                                                g->payload.p, r_scan * r_scan, r_particle,
                                                                2.0f * r_particle + nb_dist);
    after_launch(ctx, "sf_finalize_kernel");
    sync(ctx);
}

static void copy_active(const std::vector<uint64_t>& act, uint64_t* out, size_t cap, size_t* n_out) {
    if (n_out) *n_out = act.size();
    if (out) {
        MSBG_REQUIRE(cap >= act.size(), "active_out is smaller than the active set (give the grid's block count)");
        std::copy(act.begin(), act.end(), out);
    }
}

}  // namespace msbg

using namespace msbg;

extern "C" {

int msbg_surface_splat_device(msbg_grid* g, const float* d_pos, size_t n, float r_particle, float nb_dist,
                              uint64_t* active_out, size_t cap, size_t* n_active_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && (d_pos || !n), "null argument");
    set_device(g->ctx);
    copy_active(surface_splat(g, d_pos, n, r_particle, nb_dist), active_out, cap, n_active_out);
    MSBG_API_END
}

int msbg_surface_finalize(msbg_grid* g, const uint64_t* active, size_t n, float r_particle, float nb_dist) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && (active || !n), "null argument");
    set_device(g->ctx);
    surface_finalize(g, active, n, r_particle, nb_dist);
    MSBG_API_END
}

int msbg_reconstruct_and_smooth(msbg_grid* g, const float* pos, size_t n, float r_particle, float nb_dist,
                                int iterations, float dt, uint64_t* active_out, size_t cap, size_t* n_active_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && (pos || !n), "null argument");
    MSBG_REQUIRE(iterations >= 0, "iterations must be >= 0");
    set_device(g->ctx);
    DevBuf io;
    io.reserve(std::max<size_t>(n * 12, 16));
    if (n) CUDA_CHECK(cudaMemcpyAsync(io.p, pos, n * 12, cudaMemcpyHostToDevice, g->ctx->stream));
    const std::vector<uint64_t> act = surface_splat(g, io.as<float>(), n, r_particle, nb_dist);
    surface_finalize(g, act.data(), act.size(), r_particle, nb_dist);
    if (iterations > 0 && !act.empty())
        check(msbg_sweep(g, act.data(), act.size(), MSBG_MEAN_CURVATURE, dt, iterations, 1));
    copy_active(act, active_out, cap, n_active_out);
    sync(g->ctx);
    MSBG_API_END
}

int msbg_place_instances(msbg_ctx* ctx, const float* base, size_t n_base, const float* bbox_min, float span_max,
                         uint64_t sx, uint64_t sy, uint64_t sz, float instance_scale_factor, size_t n_instances,
                         float* pos_out, size_t cap, size_t* n_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && n_out && (base || !n_base) && bbox_min, "null argument");
    MSBG_REQUIRE(span_max > 0.0f, "span_max must be > 0");
    MSBG_REQUIRE(n_instances <= n_base, "more instances than base points");
    const uint64_t total = (uint64_t)n_base * n_instances;
    MSBG_REQUIRE(total < (1ULL << 32), "placement supports < 2^32 (instance, point) pairs");
    set_device(ctx);
    *n_out = 0;
    if (!total) return MSBG_OK;
    PlaceArgs a;
    a.n_base = (int64_t)n_base;
    a.n_inst = (int64_t)n_instances;
    const double sc = 16777215.0 / 32768.0;
    const uint64_t dims[3] = {sx, sy, sz};
    for (int ax = 0; ax < 3; ++ax) {
        a.bbox[ax] = bbox_min[ax];
        a.dom_min[ax] = (float)(std::floor(sc * 0.005 + 0.5) / sc);
        a.dom_max[ax] = (float)(std::floor(sc * ((double)dims[ax] - 0.005) + 0.5) / sc);
    }
    a.smax = (float)std::max(sx, std::max(sy, sz));
    a.base_scale = 1.0f / span_max;
    a.inst_scale = ((float)std::min(sx, std::min(sy, sz)) * instance_scale_factor) * a.base_scale;
    a.sx = (int64_t)sx; a.sy = (int64_t)sy; a.sz = (int64_t)sz;
    ScratchLayout L;
    const size_t o_b = L.add<float>(3 * n_base), o_k = L.add<uint32_t>(total), o_o = L.add<uint32_t>(total),
                 o_t = L.add<uint32_t>(4), o_s = L.add<char>(scan_scratch_bytes(total)), o_p = L.add<float>(3 * total);
    char* b = scratch(ctx, L);
    CUDA_CHECK(cudaMemcpyAsync(ScratchLayout::at<float>(b, o_b), base, n_base * 12, cudaMemcpyHostToDevice, ctx->stream));
    a.base = ScratchLayout::at<float>(b, o_b);
    begin_launch(ctx);
    sf_place_flags_kernel<<<sf_grid(total), 256, 0, ctx->stream>>>(a, ScratchLayout::at<uint32_t>(b, o_k));
    after_launch(ctx, "sf_place_flags_kernel");
    exclusive_scan_u32(ctx, ScratchLayout::at<uint32_t>(b, o_k), ScratchLayout::at<uint32_t>(b, o_o), total,
                       ScratchLayout::at<uint32_t>(b, o_t), ScratchLayout::at<char>(b, o_s));
    begin_launch(ctx);
    sf_place_write_kernel<<<sf_grid(total), 256, 0, ctx->stream>>>(a, ScratchLayout::at<uint32_t>(b, o_k),
                                                                   ScratchLayout::at<uint32_t>(b, o_o),
                                                                   ScratchLayout::at<float>(b, o_p));
    after_launch(ctx, "sf_place_write_kernel");
    uint32_t count = 0;
    read_small(ctx, &count, ScratchLayout::at<uint32_t>(b, o_t), 4);
    *n_out = count;
    if (pos_out) {
        MSBG_REQUIRE(cap >= count, "pos_out is smaller than the number of placed particles");
        if (count) CUDA_CHECK(cudaMemcpyAsync(pos_out, ScratchLayout::at<float>(b, o_p), (size_t)count * 12,
                                              cudaMemcpyDeviceToHost, ctx->stream));
    }
    sync(ctx);
    MSBG_API_END
}

}  // extern "C"
