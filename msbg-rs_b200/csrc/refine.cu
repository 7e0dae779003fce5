// refine.cu -- the refinement map of the multiresolution grid on the device:
// regularize_refinement_map (multires/refinement.rs:63-107, the 2:1 rule) and
// the block topology of set_refinement_map (refinement.rs:124-208).
//
// Regularisation is n_levels - 2 Jacobi passes over the block grid (each pass
// reads the previous map and writes the next, as the crate's `prev` copy
// does), one thread per block with its 26 neighbours.  The topology is one
// pass computing every block's flags, then an ordered compaction per level
// of the FINE_COARSE blocks (scan of flags), so the lists come out in block
// order as the crate's serial collection makes them.
#include <algorithm>

#include "common.cuh"
#include "sort.cuh"

namespace msbg {

constexpr uint16_t kBlkDomBorder = 1u << 1, kBlkCoarseFine = 1u << 2, kBlkFineCoarse = 1u << 3, kBlkExists = 1u << 12;

__global__ void rf_regularize_kernel(const uint8_t* __restrict__ prev, uint8_t* __restrict__ out, int64_t nx, int64_t ny,
                                     int64_t nz, int ll, int n_levels) {
    const int64_t n = nx * ny * nz;
    for (int64_t bid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; bid < n; bid += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t level = prev[bid];
        uint8_t o = level;
        if (level >= ll) {
            const int64_t bx = bid % nx, by = (bid / nx) % ny, bz = bid / (nx * ny);
            uint8_t level2 = (uint8_t)(n_levels - 1);
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (!dx && !dy && !dz) continue;
                        const int64_t X = bx + dx, Y = by + dy, Z = bz + dz;
                        if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
                        level2 = min(level2, prev[X + Y * nx + Z * nx * ny]);
                    }
            if (level2 == ll - 1) o = (uint8_t)ll;
        }
        out[bid] = o;
    }
}

// Block flags; fc[l * n + bid] = 1 when bid is a FINE_COARSE block of level l;
// exists counts EXISTS blocks.
__global__ void rf_topology_kernel(const uint8_t* __restrict__ map, const uint16_t* __restrict__ user, int64_t nx, int64_t ny,
                                   int64_t nz, int n_levels, uint16_t* __restrict__ flags, uint32_t* __restrict__ fc,
                                   unsigned long long* __restrict__ exists) {
    const int64_t n = nx * ny * nz;
    for (int64_t bid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; bid < n; bid += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t level = map[bid];
        uint16_t f = user ? user[bid] : 0;
        const int64_t bx = bid % nx, by = (bid / nx) % ny, bz = bid / (nx * ny);
        if (bx == 0 || bx == nx - 1 || by == 0 || by == ny - 1 || bz == 0 || bz == nz - 1) f |= kBlkDomBorder;
        uint8_t lmax = 0, lmin = (uint8_t)(n_levels - 1);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (!dx && !dy && !dz) continue;
                    const int64_t X = bx + dx, Y = by + dy, Z = bz + dz;
                    if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
                    const uint8_t l2 = map[X + Y * nx + Z * nx * ny];
                    lmax = max(lmax, l2);
                    lmin = min(lmin, l2);
                }
        if (lmax > level) f |= kBlkFineCoarse;
        if (lmin < level) f |= kBlkCoarseFine;
        flags[bid] = f;
        for (int l = 0; l < n_levels; ++l) fc[(int64_t)l * n + bid] = (l == level && (f & kBlkFineCoarse)) ? 1u : 0u;
        if (f & kBlkExists) atomicAdd(exists, 1ull);
    }
}

__global__ void rf_compact_kernel(const uint32_t* __restrict__ fc, const uint32_t* __restrict__ off, int64_t n,
                                  uint64_t* __restrict__ out) {
    for (int64_t bid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; bid < n; bid += (int64_t)gridDim.x * blockDim.x)
        if (fc[bid]) out[off[bid]] = (uint64_t)bid;
}

__global__ void rf_check_kernel(const uint8_t* __restrict__ map, int64_t n, int n_levels, int* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (map[i] >= n_levels) atomicExch(bad, 1);
}

static unsigned rf_grid(int64_t n) { return (unsigned)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 16); }

static void check_levels(msbg_ctx* ctx, const uint8_t* d_map, int64_t n, int n_levels, int* word) {
    CUDA_CHECK(cudaMemsetAsync(word, 0, 4, ctx->stream));
    begin_launch(ctx);
    rf_check_kernel<<<rf_grid(n), 256, 0, ctx->stream>>>(d_map, n, n_levels, word);
    after_launch(ctx, "rf_check_kernel");
    int h = 0;
    read_small(ctx, &h, word, 4);
    MSBG_REQUIRE(!h, "a block level is >= n_levels");
}

static void regularize(msbg_ctx* ctx, uint8_t* d_map, int64_t nx, int64_t ny, int64_t nz, int n_levels) {
    const int64_t n = nx * ny * nz;
    if (n_levels <= 2 || !n) return;
    DevBuf tmp;
    tmp.reserve((size_t)n + 16);
    uint8_t* a = d_map;
    uint8_t* b = tmp.as<uint8_t>();
    for (int ll = 1; ll <= n_levels - 2; ++ll) {
        begin_launch(ctx);
        rf_regularize_kernel<<<rf_grid(n), 256, 0, ctx->stream>>>(a, b, nx, ny, nz, ll, n_levels);
        after_launch(ctx, "rf_regularize_kernel");
        std::swap(a, b);
    }
    if (a != d_map) CUDA_CHECK(cudaMemcpyAsync(d_map, a, (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
    sync(ctx);  // tmp dies at return
}

}  // namespace msbg

using namespace msbg;

extern "C" {

int msbg_regularize_refinement_map_device(msbg_ctx* ctx, uint8_t* d_levels, uint64_t nx, uint64_t ny, uint64_t nz,
                                          int n_levels) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && (d_levels || nx * ny * nz == 0), "null argument");
    MSBG_REQUIRE(n_levels >= 1 && n_levels <= 255, "n_levels must be 1..255");
    set_device(ctx);
    regularize(ctx, d_levels, (int64_t)nx, (int64_t)ny, (int64_t)nz, n_levels);
    MSBG_API_END
}

int msbg_regularize_refinement_map(msbg_ctx* ctx, uint8_t* levels, uint64_t nx, uint64_t ny, uint64_t nz, int n_levels) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && (levels || nx * ny * nz == 0), "null argument");
    MSBG_REQUIRE(n_levels >= 1 && n_levels <= 255, "n_levels must be 1..255");
    set_device(ctx);
    const int64_t n = (int64_t)(nx * ny * nz);
    if (!n) return MSBG_OK;
    DevBuf d;
    d.reserve((size_t)n + 16);
    CUDA_CHECK(cudaMemcpyAsync(d.p, levels, (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    regularize(ctx, d.as<uint8_t>(), (int64_t)nx, (int64_t)ny, (int64_t)nz, n_levels);
    CUDA_CHECK(cudaMemcpyAsync(levels, d.p, (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    MSBG_API_END
}

int msbg_block_topology(msbg_ctx* ctx, const uint8_t* levels, uint64_t nx, uint64_t ny, uint64_t nz, int n_levels,
                        const uint16_t* user_flags, uint16_t* flags_out, uint64_t* fine_coarse_out,
                        uint64_t* fine_coarse_counts, uint64_t* n_exists_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && levels && flags_out && fine_coarse_counts, "null argument");
    MSBG_REQUIRE(n_levels >= 1 && n_levels <= 255, "n_levels must be 1..255");
    set_device(ctx);
    const int64_t n = (int64_t)(nx * ny * nz);
    MSBG_REQUIRE(n > 0 && n < (1LL << 31), "block grid must hold 1 .. 2^31 - 1 blocks");
    ScratchLayout L;
    const size_t o_m = L.add<uint8_t>(n), o_u = L.add<uint16_t>(n), o_f = L.add<uint16_t>(n),
                 o_fc = L.add<uint32_t>((size_t)n * n_levels), o_off = L.add<uint32_t>(n), o_t = L.add<uint32_t>(4),
                 o_s = L.add<char>(scan_scratch_bytes(n)), o_l = L.add<uint64_t>(n), o_e = L.add<uint64_t>(2),
                 o_w = L.add<int>(4);
    char* b = scratch(ctx, L);
    CUDA_CHECK(cudaMemcpyAsync(ScratchLayout::at<uint8_t>(b, o_m), levels, (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    check_levels(ctx, ScratchLayout::at<uint8_t>(b, o_m), n, n_levels, ScratchLayout::at<int>(b, o_w));
    if (user_flags)
        CUDA_CHECK(cudaMemcpyAsync(ScratchLayout::at<uint16_t>(b, o_u), user_flags, (size_t)n * 2, cudaMemcpyHostToDevice,
                                   ctx->stream));
    CUDA_CHECK(cudaMemsetAsync(ScratchLayout::at<uint64_t>(b, o_e), 0, 8, ctx->stream));
    begin_launch(ctx);
    rf_topology_kernel<<<rf_grid(n), 256, 0, ctx->stream>>>(
        ScratchLayout::at<uint8_t>(b, o_m), user_flags ? ScratchLayout::at<uint16_t>(b, o_u) : nullptr, (int64_t)nx,
        (int64_t)ny, (int64_t)nz, n_levels, ScratchLayout::at<uint16_t>(b, o_f), ScratchLayout::at<uint32_t>(b, o_fc),
        ScratchLayout::at<unsigned long long>(b, o_e));
    after_launch(ctx, "rf_topology_kernel");
    CUDA_CHECK(cudaMemcpyAsync(flags_out, ScratchLayout::at<uint16_t>(b, o_f), (size_t)n * 2, cudaMemcpyDeviceToHost,
                               ctx->stream));
    for (int l = 0; l < n_levels; ++l) {
        const uint32_t* fc = ScratchLayout::at<uint32_t>(b, o_fc) + (size_t)l * n;
        exclusive_scan_u32(ctx, fc, ScratchLayout::at<uint32_t>(b, o_off), (size_t)n, ScratchLayout::at<uint32_t>(b, o_t),
                           ScratchLayout::at<char>(b, o_s));
        uint32_t cnt = 0;
        read_small(ctx, &cnt, ScratchLayout::at<uint32_t>(b, o_t), 4);
        fine_coarse_counts[l] = cnt;
        if (fine_coarse_out && cnt) {
            begin_launch(ctx);
            rf_compact_kernel<<<rf_grid(n), 256, 0, ctx->stream>>>(fc, ScratchLayout::at<uint32_t>(b, o_off), n,
                                                                   ScratchLayout::at<uint64_t>(b, o_l));
            after_launch(ctx, "rf_compact_kernel");
            CUDA_CHECK(cudaMemcpyAsync(fine_coarse_out + (size_t)l * n, ScratchLayout::at<uint64_t>(b, o_l), (size_t)cnt * 8,
                                       cudaMemcpyDeviceToHost, ctx->stream));
        }
    }
    uint64_t ex = 0;
    read_small(ctx, &ex, ScratchLayout::at<uint64_t>(b, o_e), 8);
    if (n_exists_out) *n_exists_out = ex;
    sync(ctx);
    MSBG_API_END
}

}  // extern "C"
