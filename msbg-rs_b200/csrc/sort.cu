// sort.cu -- stable onesweep LSD radix sort (8-bit digits), device scans,
// per-particle Morton keys (multires/sort.rs:5-22), bucket_indices
// (particles/sort.rs:174-269) and sort_block_list_morton (multires/sort.rs:35-57).
//
// The sort reads the keys once to histogram every digit at the same time
// (os_hist_kernel), then runs one kernel per digit (os_pass_kernel).  In a
// pass, each CTA takes the next tile id from a counter (so every lower tile
// belongs to a CTA that is already running), ranks its tile's keys stably in
// shared memory, publishes the tile's per-digit counts, and finds the counts
// of all lower tiles by decoupled look-back over a status array of 64-bit
// words (flag and count in one word, so a reader never sees one without the
// other).  The keys then leave shared memory in digit order, so each digit's
// run is written contiguously.  Stable, so sorting (key, index) pairs
// reproduces a stable CPU sort exactly.
#include <algorithm>
#include <mutex>

#include "sort.cuh"

namespace msbg {

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Block-wide exclusive scan of one value per thread (blockDim.x <= 1024, a
// multiple of 32).  Returns the exclusive prefix; *total gets the block sum.
__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t wsum[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < nw ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        wsum[lane] = s;  // inclusive prefix over warps
    }
    __syncthreads();
    uint32_t warp_ex = warp ? wsum[warp - 1] : 0;
    *total = wsum[nw - 1];
    __syncthreads();
    return warp_ex + x - v;
}

// One CTA per row: exclusive scan of the row in place, row total to totals.
__global__ void __launch_bounds__(1024) scan_rows_kernel(uint32_t* data, size_t row_len, uint32_t* totals) {
    uint32_t* row = data + (size_t)blockIdx.x * row_len;
    uint32_t carry = 0;
    for (size_t b = 0; b < row_len; b += blockDim.x) {
        size_t i = b + threadIdx.x;
        uint32_t v = i < row_len ? row[i] : 0, tot;
        uint32_t ex = block_exclusive_scan(v, &tot);
        if (i < row_len) row[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && totals) totals[blockIdx.x] = carry;
}

constexpr int OS_THREADS = 256;
constexpr int OS_ITEMS = 8;  // even, and 32 * OS_ITEMS < 65536
constexpr int OS_TILE = OS_THREADS * OS_ITEMS;
constexpr int OS_WARPS = OS_THREADS / 32;
constexpr int OS_MAX_PASSES = 8;
constexpr int OH_ITEMS = 8;
constexpr int OS_LOOKBACK = 8;  // predecessor tiles read per look-back round
constexpr uint64_t OS_AGGREGATE = 1ull << 32;  // word holds this tile's own count
constexpr uint64_t OS_INCLUSIVE = 2ull << 32;  // word holds the count of tiles 0..k
constexpr size_t OS_PASS_SMEM = (size_t)OS_TILE * (8 + 4);  // 64-bit keys; 32-bit ones use OS_TILE * 8

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Histogram of every digit of every key, and zeroing of the first pass's
// status array.  Each thread takes OH_ITEMS consecutive keys and adds runs of
// equal digits with one shared atomic (keys that are nearly sorted already,
// such as particles sorted in the previous step, share their high digits).
__global__ void __launch_bounds__(256) os_hist_kernel(const uint64_t* __restrict__ keys, size_t n, int passes,
                                                      uint32_t* __restrict__ hist, uint64_t* __restrict__ zero,
                                                      size_t n_zero) {
    __shared__ uint32_t h[OS_MAX_PASSES * 256];
    for (int q = threadIdx.x; q < OS_MAX_PASSES * 256; q += blockDim.x) h[q] = 0;
    __syncthreads();
    const size_t chunk = (size_t)blockDim.x * OH_ITEMS;
    for (size_t b = blockIdx.x * chunk; b < n; b += (size_t)gridDim.x * chunk) {
        const size_t i0 = b + (size_t)threadIdx.x * OH_ITEMS;
        const int cnt = i0 >= n ? 0 : (n - i0 < (size_t)OH_ITEMS ? (int)(n - i0) : OH_ITEMS);
        uint64_t k[OH_ITEMS];
#pragma unroll
        for (int j = 0; j < OH_ITEMS; ++j) k[j] = j < cnt ? keys[i0 + j] : 0;
        if (!cnt) continue;
        for (int p = 0; p < passes; ++p) {
            const int sh = 8 * p;
            uint32_t cur = (uint32_t)(k[0] >> sh) & 255u, run = 0;
#pragma unroll
            for (int j = 0; j < OH_ITEMS; ++j) {
                if (j < cnt) {
                    const uint32_t d = (uint32_t)(k[j] >> sh) & 255u;
                    if (d != cur) {
                        atomicAdd(&h[p * 256 + cur], run);
                        cur = d;
                        run = 0;
                    }
                    ++run;
                }
            }
            atomicAdd(&h[p * 256 + cur], run);
        }
    }
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n_zero; i += (size_t)gridDim.x * blockDim.x)
        zero[i] = 0;
    __syncthreads();
    for (int q = threadIdx.x; q < passes * 256; q += blockDim.x)
        if (h[q]) atomicAdd(&hist[q], h[q]);
}

// One digit pass.  Tile t holds keys [t*OS_TILE, (t+1)*OS_TILE); warp w of the
// CTA ranks the tile's w-th run of 32*OS_ITEMS keys, item j of lane l being
// key w*32*OS_ITEMS + j*32 + l, so (warp, item, lane) order is index order and
// the local sort is stable.  `status` holds tiles*256 words for this pass
// (zeroed before the launch); `status_next` (the next pass's array, or null)
// is zeroed here, tile by tile.  A look-back that waits more than limit_ns
// (one second in a sort) sets bit 2 of *err and carries on with what it has
// (the result is then wrong and the host reports the error), so no CTA can
// spin forever.  KI, KO: the key types read and written; KS: the type a key
// has inside the pass (32 bits when every key fits: half the shared-memory
// and global traffic of the keys in the passes between the first and last).
template <class KI, class KO, class KS>
__global__ void __launch_bounds__(OS_THREADS, 5)
    os_pass_kernel(const KI* __restrict__ kin, const uint32_t* __restrict__ vin, KO* __restrict__ kout,
                   uint32_t* __restrict__ vout, size_t n, int shift, const uint32_t* __restrict__ hist,
                   uint64_t* status, uint64_t* __restrict__ status_next, uint32_t* tile_counter, int* err,
                   uint64_t limit_ns) {
    extern __shared__ __align__(16) unsigned char os_smem[];
    KS* s_keys = reinterpret_cast<KS*>(os_smem);
    uint32_t* s_vals = reinterpret_cast<uint32_t*>(os_smem + (size_t)OS_TILE * sizeof(KS));
    __shared__ uint32_t s_wc[OS_WARPS][256];    // per-warp digit counts, then offsets
    __shared__ uint32_t s_match[OS_WARPS][256];  // per-warp lane masks of one round
    __shared__ uint32_t s_base[256];
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
    const uint32_t hist_d = hist[tid];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        s_wc[w][lane + 32 * q] = 0;
        s_match[w][lane + 32 * q] = 0;
    }
    __syncthreads();
    const size_t tile = s_tile;
    const size_t tile_base = tile * OS_TILE;
    const size_t wbase = tile_base + (size_t)w * 32 * OS_ITEMS;
    const uint32_t lt = lanemask_lt();

    // keys of this warp still inside the array (0 for warps past the end)
    const int rem = wbase >= n ? 0 : (n - wbase >= (size_t)(32 * OS_ITEMS) ? 32 * OS_ITEMS : (int)(n - wbase));
    KS key[OS_ITEMS];
#pragma unroll
    for (int j = 0; j < OS_ITEMS; ++j) key[j] = j * 32 + lane < rem ? (KS)kin[wbase + lane + j * 32] : (KS)0;
    // warp-level stable ranking, one round per item: every lane ORs its bit
    // into its digit's mask, so the mask read back holds the lanes with the
    // same digit; the lowest of them adds the group's size to the warp's
    // count and clears the mask for the next round
    uint32_t rank[OS_ITEMS / 2];  // two 16-bit ranks per word (a warp ranks at most 32*OS_ITEMS keys)
    uint32_t* wc = s_wc[w];
    uint32_t* wm = s_match[w];
#pragma unroll
    for (int j = 0; j < OS_ITEMS; ++j) {
        const bool valid = j * 32 + lane < rem;
        const uint32_t d = (uint32_t)(key[j] >> shift) & 255u;
        if (valid) atomicOr(&wm[d], 1u << lane);
        __syncwarp();
        const uint32_t peers = valid ? wm[d] : 0u;
        const uint32_t lower = __popc(peers & lt);
        const uint32_t c = valid ? wc[d] : 0u;
        __syncwarp();
        if (valid && lower == 0) {
            wc[d] = c + __popc(peers);
            wm[d] = 0;
        }
        __syncwarp();
        if (j & 1) rank[j >> 1] |= (c + lower) << 16;
        else rank[j >> 1] = c + lower;
    }
    __syncthreads();

    // thread tid owns digit tid: tile count, publish, then each warp's
    // offset of the digit inside the tile's local sort
    uint32_t count = 0;
#pragma unroll
    for (int q = 0; q < OS_WARPS; ++q) count += s_wc[q][tid];
    uint64_t* my_status = status + tile * 256 + tid;
    st_relaxed_u64(my_status, (tile == 0 ? OS_INCLUSIVE : OS_AGGREGATE) | count);
    if (status_next) status_next[tile * 256 + tid] = 0;
    uint32_t total;
    const uint32_t local = block_exclusive_scan(count, &total);
    const uint32_t global = block_exclusive_scan(hist_d, &total);
    {
        uint32_t run = local;
#pragma unroll
        for (int q = 0; q < OS_WARPS; ++q) {
            const uint32_t c = s_wc[q][tid];
            s_wc[q][tid] = run;
            run += c;
        }
    }
    __syncthreads();

    // local sort into shared memory
#pragma unroll
    for (int j = 0; j < OS_ITEMS; ++j) {
        if (j * 32 + lane < rem) {
            const uint32_t d = (uint32_t)(key[j] >> shift) & 255u;
            const uint32_t pos = wc[d] + ((rank[j >> 1] >> (16 * (j & 1))) & 0xffffu);
            s_keys[pos] = key[j];
            s_vals[pos] = vin ? vin[wbase + lane + j * 32] : (uint32_t)(wbase + lane + j * 32);
        }
    }

    // decoupled look-back for digit tid, OS_LOOKBACK predecessors per round:
    // add aggregates until an inclusive count; stop at a tile that has not
    // published yet and read again from there
    uint32_t before = 0;
    if (tile > 0) {
        size_t k = tile - 1;  // highest tile not yet added
        uint64_t t0 = 0;
        uint32_t spins = 0;
        while (true) {
            uint64_t sv[OS_LOOKBACK];
#pragma unroll
            for (int q = 0; q < OS_LOOKBACK; ++q)
                sv[q] = k >= (size_t)q ? ld_relaxed_u64(status + (k - q) * 256 + tid) : OS_INCLUSIVE;
            int used = 0;
            bool done = false;
#pragma unroll
            for (int q = 0; q < OS_LOOKBACK; ++q) {
                if (used == q && !done) {
                    const uint64_t flag = sv[q] & (3ull << 32);
                    if (flag != 0) {
                        before += (uint32_t)sv[q];
                        done = flag == OS_INCLUSIVE;
                        ++used;
                    }
                }
            }
            if (done) break;
            k -= used;
            if (used < OS_LOOKBACK && (++spins & 15u) == 0) {
                const uint64_t now = globaltimer_ns();
                if (!t0) t0 = now;
                else if (now - t0 > limit_ns) {
                    atomicOr(err, 2);
                    break;
                }
            }
        }
        st_relaxed_u64(my_status, OS_INCLUSIVE | (before + count));
    }
    s_base[tid] = global + before - local;
    __syncthreads();

    const int in_tile = n - tile_base < (size_t)OS_TILE ? (int)(n - tile_base) : OS_TILE;
    for (int i = tid; i < in_tile; i += OS_THREADS) {
        const KS k = s_keys[i];
        const uint32_t dst = s_base[(uint32_t)(k >> shift) & 255u] + (uint32_t)i;  // modulo 2^32, as s_base is
        if (dst < n) {  // always true unless a look-back gave up
            kout[dst] = (KO)k;
            vout[dst] = s_vals[i];
        }
    }
}

__global__ void iota_copy_kernel(const uint64_t* kin, const uint32_t* vin, uint64_t* kout, uint32_t* vout, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        kout[i] = kin[i];
        vout[i] = vin ? vin[i] : (uint32_t)i;
    }
}

static constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Scratch of the onesweep sort: ping-pong keys and values, the digit
// histograms with one tile counter per pass, and two status arrays (pass p
// uses array p % 2 and clears the other for pass p + 1).
static constexpr size_t onesweep_scratch_bytes(size_t n) {
    return align256(n * 8) + align256(n * 4) + align256(OS_MAX_PASSES * 256 * 4 + OS_MAX_PASSES * 4) +
           2 * align256(((n + OS_TILE - 1) / OS_TILE) * 256 * 8);
}

size_t radix_sort_scratch_bytes(size_t n) { return onesweep_scratch_bytes(n); }

void radix_sort_pairs(msbg_ctx* ctx, const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out,
                      uint32_t* vals_out, size_t n, int end_bit, void* tmp) {
    if (!n) return;
    MSBG_REQUIRE(n < (1ULL << 32), "radix sort supports < 2^32 items");
    MSBG_REQUIRE(end_bit >= 0 && end_bit <= 64, "radix sort end_bit out of range");
    const int passes = (end_bit + 7) / 8;
    if (passes == 0) {
        begin_launch(ctx);
        iota_copy_kernel<<<std::min<size_t>(div_up(n, 256), 4096), 256, 0, ctx->stream>>>(keys_in, vals_in, keys_out, vals_out, n);
        after_launch(ctx, "iota_copy_kernel");
        return;
    }
    const size_t tiles = (n + OS_TILE - 1) / OS_TILE;
    char* t = (char*)tmp;
    uint64_t* kt = (uint64_t*)t;
    t += align256(n * 8);
    uint32_t* vt = (uint32_t*)t;
    t += align256(n * 4);
    uint32_t* hist = (uint32_t*)t;
    uint32_t* counters = hist + OS_MAX_PASSES * 256;
    t += align256(OS_MAX_PASSES * 256 * 4 + OS_MAX_PASSES * 4);
    uint64_t* status[2] = {(uint64_t*)t, (uint64_t*)(t + align256(tiles * 256 * 8))};
    CUDA_CHECK(cudaMemsetAsync(hist, 0, OS_MAX_PASSES * 256 * 4 + OS_MAX_PASSES * 4, ctx->stream));
    begin_launch(ctx);
    os_hist_kernel<<<(unsigned)std::min<size_t>(div_up(n, 256 * OH_ITEMS), 148 * 8), 256, 0, ctx->stream>>>(
        keys_in, n, passes, hist, status[0], tiles * 256);
    after_launch(ctx, "os_hist_kernel");
    // keys of at most 32 bits move as 32-bit words between the passes (the
    // first pass narrows, the last widens); the ping-pong buffers hold either
    const bool narrow = end_bit <= 32;
    const void* ki = keys_in;
    const uint32_t* vi = vals_in;
    for (int p = 0; p < passes; ++p) {
        const bool to_out = ((passes - 1 - p) % 2) == 0;
        void* ko = to_out ? (void*)keys_out : (void*)kt;
        uint32_t* vo = to_out ? vals_out : vt;
        const bool first = p == 0, last = p + 1 == passes;
        uint64_t* st_next = p + 1 < passes ? status[(p + 1) & 1] : nullptr;
        begin_launch(ctx);
#define OS_PASS(KI, KO, KS)                                                                                              \
    os_pass_kernel<KI, KO, KS><<<(unsigned)tiles, OS_THREADS, (size_t)OS_TILE * (sizeof(KS) + 4), ctx->stream>>>(     \
        (const KI*)ki, vi, (KO*)ko, vo, n, 8 * p, hist + p * 256, status[p & 1], st_next, counters + p,                 \
        ctx->status.as<int>(), kWaitLimitNs)
        if (!narrow) OS_PASS(uint64_t, uint64_t, uint64_t);
        else if (first && last) OS_PASS(uint64_t, uint64_t, uint32_t);
        else if (first) OS_PASS(uint64_t, uint32_t, uint32_t);
        else if (last) OS_PASS(uint32_t, uint64_t, uint32_t);
        else OS_PASS(uint32_t, uint32_t, uint32_t);
#undef OS_PASS
        after_launch(ctx, "os_pass_kernel");
        ki = ko;
        vi = vo;
    }
}

// ---- exclusive scan of u32 --------------------------------------------------
constexpr int SC_THREADS = 1024;
constexpr int SC_ITEMS = 4;
constexpr int SC_TILE = SC_THREADS * SC_ITEMS;

__global__ void __launch_bounds__(SC_THREADS) scan_tile_sums_kernel(const uint32_t* in, size_t n, uint32_t* sums) {
    const size_t base = (size_t)blockIdx.x * SC_TILE;
    uint32_t s = 0;
    for (int j = 0; j < SC_ITEMS; ++j) {
        size_t i = base + (size_t)threadIdx.x * SC_ITEMS + j;
        if (i < n) s += in[i];
    }
    uint32_t tot;
    block_exclusive_scan(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SC_THREADS) scan_tiles_kernel(const uint32_t* in, uint32_t* out, size_t n, const uint32_t* offs) {
    const size_t base = (size_t)blockIdx.x * SC_TILE;
    uint32_t v[SC_ITEMS], s = 0;
    for (int j = 0; j < SC_ITEMS; ++j) {
        size_t i = base + (size_t)threadIdx.x * SC_ITEMS + j;
        v[j] = i < n ? in[i] : 0;
        s += v[j];
    }
    uint32_t tot;
    uint32_t ex = block_exclusive_scan(s, &tot) + offs[blockIdx.x];
    for (int j = 0; j < SC_ITEMS; ++j) {
        size_t i = base + (size_t)threadIdx.x * SC_ITEMS + j;
        if (i < n) out[i] = ex;
        ex += v[j];
    }
}

size_t scan_scratch_bytes(size_t n) { return align256(((n + SC_TILE - 1) / SC_TILE + 1) * 4) + 256; }

__global__ void copy_u32_kernel(const uint32_t* a, uint32_t* b) { *b = *a; }

void exclusive_scan_u32(msbg_ctx* ctx, const uint32_t* in, uint32_t* out, size_t n, uint32_t* d_total, void* tmp) {
    if (!n) return;
    const unsigned tiles = (unsigned)((n + SC_TILE - 1) / SC_TILE);
    uint32_t* sums = (uint32_t*)tmp;
    uint32_t* total = sums + tiles;  // scan_rows writes the row total here
    begin_launch(ctx);
    scan_tile_sums_kernel<<<tiles, SC_THREADS, 0, ctx->stream>>>(in, n, sums);
    after_launch(ctx, "scan_tile_sums_kernel");
    begin_launch(ctx);
    scan_rows_kernel<<<1, 1024, 0, ctx->stream>>>(sums, tiles, total);
    after_launch(ctx, "scan_rows_kernel");
    begin_launch(ctx);
    scan_tiles_kernel<<<tiles, SC_THREADS, 0, ctx->stream>>>(in, out, n, sums);
    after_launch(ctx, "scan_tiles_kernel");
    if (d_total) {
        begin_launch(ctx);
        copy_u32_kernel<<<1, 1, 0, ctx->stream>>>(total, d_total);
        after_launch(ctx, "copy_u32_kernel");
    }
}

__global__ void max_u64_kernel(const uint64_t* k, size_t n, unsigned long long* out) {
    unsigned long long m = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        m = max(m, (unsigned long long)k[i]);
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

int key_bits(msbg_ctx* ctx, const uint64_t* d_keys, size_t n, void* tmp8) {
    if (!n) return 0;
    CUDA_CHECK(cudaMemsetAsync(tmp8, 0, 8, ctx->stream));
    begin_launch(ctx);
    max_u64_kernel<<<std::min<size_t>(div_up(n, 256), 1184), 256, 0, ctx->stream>>>(d_keys, n, (unsigned long long*)tmp8);
    after_launch(ctx, "max_u64_kernel");
    uint64_t m = 0;
    read_small(ctx, &m, tmp8, 8);
    int b = 0;
    while (b < 64 && (m >> b)) ++b;
    return b;
}

// Runs of equal key >> shift in sorted keys, in two passes over the keys:
// each tile of SEG_TILE keys counts its run starts, the counts are scanned,
// then each tile writes its runs' keys and start indices in index order
// (warp w of a tile owns the tile's w-th range of 32 * SEG_ITEMS keys and
// walks it in rounds of 32).
constexpr int SEG_THREADS = 256, SEG_ITEMS = 16, SEG_TILE = SEG_THREADS * SEG_ITEMS;

__device__ __forceinline__ bool seg_start(const uint64_t* k, size_t i, uint64_t shift) {
    return i == 0 || (k[i] >> shift) != (k[i - 1] >> shift);
}

__global__ void __launch_bounds__(SEG_THREADS) seg_count_kernel(const uint64_t* __restrict__ k, size_t n, uint64_t shift,
                                                                uint32_t* __restrict__ tile_cnt) {
    const size_t base = (size_t)blockIdx.x * SEG_TILE;
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < SEG_ITEMS; ++j) {
        const size_t i = base + (size_t)j * SEG_THREADS + threadIdx.x;
        if (i < n && seg_start(k, i, shift)) ++c;
    }
    uint32_t total;
    block_exclusive_scan(c, &total);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SEG_THREADS) seg_emit_kernel(const uint64_t* __restrict__ k, size_t n, uint64_t shift,
                                                               const uint32_t* __restrict__ tile_off,
                                                               uint64_t* __restrict__ uniq, uint64_t* __restrict__ starts,
                                                               const uint32_t* __restrict__ count) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const size_t wbase = (size_t)blockIdx.x * SEG_TILE + (size_t)w * 32 * SEG_ITEMS;
    uint32_t fl = 0;  // bit j: item wbase + 32 j + lane starts a run
    uint32_t wc = 0;  // run starts in the warp's range
#pragma unroll
    for (int j = 0; j < SEG_ITEMS; ++j) {
        const size_t i = wbase + 32 * j + lane;
        const bool st = i < n && seg_start(k, i, shift);
        fl |= (uint32_t)st << j;
        wc += __popc(__ballot_sync(0xffffffffu, st));
    }
    uint32_t total;
    uint32_t off = block_exclusive_scan(lane == 0 ? wc : 0u, &total);
    off = __shfl_sync(0xffffffffu, off, 0) + tile_off[blockIdx.x];
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int j = 0; j < SEG_ITEMS; ++j) {
        const bool st = (fl >> j) & 1u;
        const uint32_t b = __ballot_sync(0xffffffffu, st);
        if (st) {
            const size_t i = wbase + 32 * j + lane;
            const uint32_t d = off + __popc(b & lt);
            uniq[d] = k[i] >> shift;
            starts[d] = i;
        }
        off += __popc(b);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) starts[*count] = n;
}

size_t segment_scratch_bytes(size_t n) { return align256(n * 4) * 2 + scan_scratch_bytes(n) + 256; }

size_t sorted_segments(msbg_ctx* ctx, const uint64_t* d_sorted, size_t n, uint64_t shift, uint64_t* d_uniq,
                       uint64_t* d_starts, void* tmp) {
    if (!n) {
        uint64_t z = 0;
        CUDA_CHECK(cudaMemcpyAsync(d_starts, &z, 8, cudaMemcpyHostToDevice, ctx->stream));
        sync(ctx);
        return 0;
    }
    const size_t tiles = div_up(n, (size_t)SEG_TILE);
    char* t = (char*)tmp;
    uint32_t* tile_cnt = (uint32_t*)t;
    t += align256(tiles * 4);
    uint32_t* tile_off = (uint32_t*)t;
    t += align256(tiles * 4);
    uint32_t* count = (uint32_t*)t;
    t += 256;
    begin_launch(ctx);
    seg_count_kernel<<<(unsigned)tiles, SEG_THREADS, 0, ctx->stream>>>(d_sorted, n, shift, tile_cnt);
    after_launch(ctx, "seg_count_kernel");
    exclusive_scan_u32(ctx, tile_cnt, tile_off, tiles, count, t);
    begin_launch(ctx);
    seg_emit_kernel<<<(unsigned)tiles, SEG_THREADS, 0, ctx->stream>>>(d_sorted, n, shift, tile_off, d_uniq, d_starts, count);
    after_launch(ctx, "seg_emit_kernel");
    uint32_t c = 0;
    read_small(ctx, &c, count, 4);
    return c;
}

// ---- Morton keys ------------------------------------------------------------
// `p as usize` (p2g.rs:149-157): truncation toward zero, negatives and NaN to 0.
__device__ __forceinline__ uint64_t trunc_coord(float p) { return p > 0.0f ? (uint64_t)p : 0; }

__global__ void morton_keys_kernel(const float* pos, size_t n, uint64_t* keys) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        keys[i] = morton3(trunc_coord(pos[3 * i]), trunc_coord(pos[3 * i + 1]), trunc_coord(pos[3 * i + 2]));
}

// The same keys and their maximum (atomicMax into *kmax, zeroed before), so
// the sort learns its digit count without a second pass over the keys.
__global__ void morton_keys_max_kernel(const float* pos, size_t n, uint64_t* keys, unsigned long long* kmax) {
    unsigned long long m = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t k = morton3(trunc_coord(pos[3 * i]), trunc_coord(pos[3 * i + 1]), trunc_coord(pos[3 * i + 2]));
        keys[i] = k;
        m = max(m, (unsigned long long)k);
    }
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(kmax, m);
}

__global__ void morton3_kernel(const uint64_t* xyz, size_t n, uint64_t* keys) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        keys[i] = morton3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
}

// multires/sort.rs:35-57 key.
__global__ void block_list_key_kernel(const uint64_t* blocks, size_t n, uint64_t nx, uint64_t ny, const uint8_t* levels,
                                      int n_levels, uint64_t* keys) {
    const uint64_t ref_shift = (uint64_t)(n_levels - 1);
    const uint64_t mask = (1ULL << ref_shift) - 1;
    const uint64_t fine_bits = 3 * ref_shift;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint64_t bid = blocks[i];
        uint64_t bx = bid % nx, by = (bid / nx) % ny, bz = bid / (nx * ny);
        uint64_t lvl = levels[i];
        uint64_t coarse = morton3(bx >> ref_shift, by >> ref_shift, bz >> ref_shift);
        uint64_t priority = ref_shift - lvl;
        uint64_t fine = morton3(bx & mask, by & mask, bz & mask);
        keys[i] = (coarse << (fine_bits + ref_shift)) | (priority << fine_bits) | fine;
    }
}

__global__ void gather_u64_kernel(const uint64_t* src, const uint32_t* perm, uint64_t* dst, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[perm[i]];
}

// dst[i] = src[perm[i]] for items of `width` floats.
// dst[i] = src[perm[i]] for rows of `width` floats: one thread per row (one
// index load, the row's floats gathered together); W > 0 fixes the width at
// compile time, W = 0 reads it from `width`.
template <int W>
__global__ void permute_kernel(const uint32_t* __restrict__ perm, size_t n, int width, const float* __restrict__ src,
                               float* __restrict__ dst) {
    const int w = W > 0 ? W : width;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float* s = src + (size_t)__ldg(perm + i) * w;
        float* d = dst + i * w;
        if (W > 0) {
            float v[W > 0 ? W : 1];
#pragma unroll
            for (int c = 0; c < W; ++c) v[c] = __ldg(s + c);
#pragma unroll
            for (int c = 0; c < W; ++c) d[c] = v[c];
        } else {
            for (int c = 0; c < w; ++c) d[c] = __ldg(s + c);
        }
    }
}

static unsigned grid_for(size_t n) { return (unsigned)std::min<size_t>(std::max<size_t>(div_up(n, 256), 1), 8192); }

void morton_keys(msbg_ctx* ctx, const float* d_pos, size_t n, uint64_t* d_keys) {
    if (!n) return;
    begin_launch(ctx);
    morton_keys_kernel<<<grid_for(n), 256, 0, ctx->stream>>>(d_pos, n, d_keys);
    after_launch(ctx, "morton_keys_kernel");
}

void morton_sort_device(msbg_ctx* ctx, const float* d_pos, size_t n, uint64_t* d_keys_out, uint32_t* d_perm_out) {
    if (!n) return;
    ScratchLayout L;
    size_t ok = L.add<uint64_t>(n), ot = L.add<char>(radix_sort_scratch_bytes(n)), o8 = L.add<uint64_t>(1);
    char* base = scratch(ctx, L);
    uint64_t* keys = ScratchLayout::at<uint64_t>(base, ok);
    unsigned long long* kmax = ScratchLayout::at<unsigned long long>(base, o8);
    CUDA_CHECK(cudaMemsetAsync(kmax, 0, 8, ctx->stream));
    begin_launch(ctx);
    morton_keys_max_kernel<<<grid_for(n), 256, 0, ctx->stream>>>(d_pos, n, keys, kmax);
    after_launch(ctx, "morton_keys_kernel");
    uint64_t m = 0;
    read_small(ctx, &m, kmax, 8);
    int bits = 0;
    while (bits < 64 && (m >> bits)) ++bits;
    radix_sort_pairs(ctx, keys, nullptr, d_keys_out, d_perm_out, n, bits, ScratchLayout::at<char>(base, ot));
}

size_t bucket_indices_device(msbg_ctx* ctx, const uint64_t* d_bids, size_t n, uint64_t* d_blocks, uint64_t* d_starts,
                             uint32_t* d_perm) {
    if (!n) {
        uint64_t z = 0;
        CUDA_CHECK(cudaMemcpyAsync(d_starts, &z, 8, cudaMemcpyHostToDevice, ctx->stream));
        sync(ctx);
        return 0;
    }
    ScratchLayout L;
    size_t osk = L.add<uint64_t>(n), ot = L.add<char>(std::max(radix_sort_scratch_bytes(n), segment_scratch_bytes(n))),
           o8 = L.add<uint64_t>(1);
    char* base = scratch(ctx, L);
    uint64_t* sk = ScratchLayout::at<uint64_t>(base, osk);
    int bits = key_bits(ctx, d_bids, n, ScratchLayout::at<char>(base, o8));
    radix_sort_pairs(ctx, d_bids, nullptr, sk, d_perm, n, bits, ScratchLayout::at<char>(base, ot));
    return sorted_segments(ctx, sk, n, 0, d_blocks, d_starts, ScratchLayout::at<char>(base, ot));
}

// ---- Morton sort without device allocation ----------------------------------
// Some callers cannot allocate device memory on the calling path: hosts that
// embed the library in a real-time loop, inside a memory-pool-managed
// allocator callback, or in a process whose device memory is fully reserved
// up front.  For them msbg_morton_sort_noalloc_device sorts up to
// kNoAllocMaxParticles particles using a fixed scratch area that is part of
// the library image: a file-scope device array, allocated by the CUDA driver
// when the library's module is loaded on a device and held by every device
// that loads the library until the process exits (about 5 MB).
constexpr size_t kNoAllocMaxParticles = size_t(1) << 18;
constexpr size_t a256c(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kNoAllocKeysBytes = a256c(kNoAllocMaxParticles * 8);
constexpr size_t kNoAllocSortBytes = onesweep_scratch_bytes(kNoAllocMaxParticles);
constexpr size_t kNoAllocScratchBytes = kNoAllocKeysBytes + kNoAllocSortBytes + 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch, looked up once per device with that
// device current (the host-side name of the array is not a device address).
static std::mutex g_noalloc_mu;
static char* g_noalloc_ptr[128] = {};

static char* noalloc_scratch(int device) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    MSBG_REQUIRE(device >= 0 && device < 128, "device ordinal out of range for the fixed scratch table");
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            MSBG_THROW(MSBG_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
        g_noalloc_ptr[device] = (char*)p;
    }
    return g_noalloc_ptr[device];
}

}  // namespace msbg

using namespace msbg;

extern "C" {

int msbg_morton3(msbg_ctx* ctx, const uint64_t* xyz, size_t n, uint64_t* keys_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && ((xyz && keys_out) || !n), "null argument");
    if (!n) return MSBG_OK;
    set_device(ctx);
    ScratchLayout L;
    size_t oi = L.add<uint64_t>(3 * n), oo = L.add<uint64_t>(n);
    char* base = scratch(ctx, L);
    uint64_t* di = ScratchLayout::at<uint64_t>(base, oi);
    uint64_t* dout = ScratchLayout::at<uint64_t>(base, oo);
    CUDA_CHECK(cudaMemcpyAsync(di, xyz, 3 * n * 8, cudaMemcpyHostToDevice, ctx->stream));
    begin_launch(ctx);
    morton3_kernel<<<grid_for(n), 256, 0, ctx->stream>>>(di, n, dout);
    after_launch(ctx, "morton3_kernel");
    CUDA_CHECK(cudaMemcpyAsync(keys_out, dout, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    MSBG_API_END
}

int msbg_sort_block_list_morton(msbg_ctx* ctx, uint64_t* blocks, size_t n, uint64_t nx, uint64_t ny,
                                const uint8_t* levels, size_t n_levels_array, int n_levels) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && ((blocks && levels) || !n), "null argument");
    MSBG_REQUIRE(n_levels >= 1 && n_levels <= 8, "n_levels out of range");
    if (!n) return MSBG_OK;
    set_device(ctx);
    std::vector<uint8_t> lv(n);
    for (size_t i = 0; i < n; ++i) {
        MSBG_REQUIRE(blocks[i] < n_levels_array, "block id outside the levels array");
        lv[i] = levels[blocks[i]];
        MSBG_REQUIRE(lv[i] < n_levels, "block level >= n_levels");
    }
    ScratchLayout L;
    size_t ob = L.add<uint64_t>(n), ol = L.add<uint8_t>(n), ok = L.add<uint64_t>(n), osk = L.add<uint64_t>(n),
           op = L.add<uint32_t>(n), ot = L.add<char>(radix_sort_scratch_bytes(n)), o8 = L.add<uint64_t>(1);
    char* base = scratch(ctx, L);
    uint64_t* db = ScratchLayout::at<uint64_t>(base, ob);
    uint8_t* dl = ScratchLayout::at<uint8_t>(base, ol);
    uint64_t* dk = ScratchLayout::at<uint64_t>(base, ok);
    uint64_t* dsk = ScratchLayout::at<uint64_t>(base, osk);
    uint32_t* dp = ScratchLayout::at<uint32_t>(base, op);
    CUDA_CHECK(cudaMemcpyAsync(db, blocks, n * 8, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_CHECK(cudaMemcpyAsync(dl, lv.data(), n, cudaMemcpyHostToDevice, ctx->stream));
    begin_launch(ctx);
    block_list_key_kernel<<<grid_for(n), 256, 0, ctx->stream>>>(db, n, nx, ny, dl, n_levels, dk);
    after_launch(ctx, "block_list_key_kernel");
    int bits = key_bits(ctx, dk, n, ScratchLayout::at<char>(base, o8));
    radix_sort_pairs(ctx, dk, nullptr, dsk, dp, n, bits, ScratchLayout::at<char>(base, ot));
    begin_launch(ctx);
    gather_u64_kernel<<<grid_for(n), 256, 0, ctx->stream>>>(db, dp, dk, n);
    after_launch(ctx, "gather_u64_kernel");
    CUDA_CHECK(cudaMemcpyAsync(blocks, dk, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    check_device_status(ctx);
    MSBG_API_END
}

int msbg_morton_sort_device(msbg_ctx* ctx, const float* d_pos, size_t n, uint64_t* d_keys_out, uint32_t* d_perm_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && ((d_pos && d_keys_out && d_perm_out) || !n), "null argument");
    set_device(ctx);
    morton_sort_device(ctx, d_pos, n, d_keys_out, d_perm_out);
    check_device_status(ctx);
    MSBG_API_END
}

// Same result as msbg_morton_sort_device for n <= 262144 particles, without
// allocating: the temporaries live in the library's fixed device scratch
// array.  The first call on a device looks up the array's device address
// (cudaGetSymbolAddress), so make that first call before capturing the
// stream into a CUDA graph; the address is kept for the life of the process,
// so a cudaDeviceReset while the library is loaded is not supported.  Each
// call blocks the host until the sort is done (it reads the largest key and
// the status word back).  All calls share the one array: calls whose GPU
// work overlaps in time (different streams or contexts on one device) race on
// it; calls ordered on one stream do not.  Every scratch word is written
// before it is read in a call (the key-bits word is cleared on the stream),
// so nothing depends on what a previous call left there.
int msbg_morton_sort_noalloc_device(msbg_ctx* ctx, const float* d_pos, size_t n, uint64_t* d_keys_out,
                                    uint32_t* d_perm_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && ((d_pos && d_keys_out && d_perm_out) || !n), "null argument");
    if (n > kNoAllocMaxParticles)
        MSBG_THROW(MSBG_ERR_ARG, "msbg_morton_sort_noalloc_device: n = " + std::to_string(n) +
                                     " exceeds the maximum of " + std::to_string(kNoAllocMaxParticles) +
                                     " particles of the fixed scratch area; use msbg_morton_sort_device");
    if (ctx->timing)
        MSBG_THROW(MSBG_ERR_STATE, "msbg_morton_sort_noalloc_device: per-kernel timing is on and would create CUDA events");
    set_device(ctx);
    if (!n) return MSBG_OK;
    char* base = noalloc_scratch(ctx->device);
    uint64_t* keys = reinterpret_cast<uint64_t*>(base);
    char* sort_tmp = base + kNoAllocKeysBytes;
    char* bits_word = base + kNoAllocKeysBytes + kNoAllocSortBytes;
    if (radix_sort_scratch_bytes(n) > kNoAllocSortBytes)
        MSBG_THROW(MSBG_ERR_STATE, "fixed scratch area smaller than the radix sort needs");
    morton_keys(ctx, d_pos, n, keys);
    const int bits = key_bits(ctx, keys, n, bits_word);
    radix_sort_pairs(ctx, keys, nullptr, d_keys_out, d_perm_out, n, bits, sort_tmp);
    check_device_status(ctx);
    MSBG_API_END
}

// Test hook for the bounded look-back wait: one digit pass of two tiles runs
// with a single CTA that takes tile 1, so the tile-0 counts it waits for are
// never published.  The wait gives up after limit_ns, sets the radix-sort bit
// of the status word, and the call returns MSBG_ERR_TIMEOUT with the word
// cleared, leaving the context usable.
int msbg_test_sort_lookback_timeout(msbg_ctx* ctx, uint64_t limit_ns) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx, "null argument");
    MSBG_REQUIRE(limit_ns >= 100000ull && limit_ns <= kWaitLimitNs, "limit_ns must lie in [1e5, 1e9]");
    set_device(ctx);
    const size_t n = 2 * (size_t)OS_TILE;
    ScratchLayout L;
    const size_t ok = L.add<uint64_t>(n), ov = L.add<uint32_t>(n), oko = L.add<uint64_t>(n), ovo = L.add<uint32_t>(n),
                 oh = L.add<uint32_t>(256), ost = L.add<uint64_t>(2 * 256), oc = L.add<uint32_t>(1);
    char* base = scratch(ctx, L);
    uint64_t* keys = ScratchLayout::at<uint64_t>(base, ok);
    uint32_t* hist = ScratchLayout::at<uint32_t>(base, oh);
    uint64_t* status = ScratchLayout::at<uint64_t>(base, ost);
    uint32_t* counter = ScratchLayout::at<uint32_t>(base, oc);
    CUDA_CHECK(cudaMemsetAsync(keys, 0, n * 8, ctx->stream));
    CUDA_CHECK(cudaMemsetAsync(hist, 0, 256 * 4, ctx->stream));
    CUDA_CHECK(cudaMemsetAsync(status, 0, 2 * 256 * 8, ctx->stream));
    const uint32_t one = 1;  // the CTA's tile id: tile 0 never runs
    CUDA_CHECK(cudaMemcpyAsync(counter, &one, 4, cudaMemcpyHostToDevice, ctx->stream));
    begin_launch(ctx);
    os_pass_kernel<uint64_t, uint64_t, uint64_t><<<1, OS_THREADS, OS_PASS_SMEM, ctx->stream>>>(
        keys, nullptr, ScratchLayout::at<uint64_t>(base, oko), ScratchLayout::at<uint32_t>(base, ovo), n, 0, hist, status,
        nullptr, counter, ctx->status.as<int>(), limit_ns);
    after_launch(ctx, "os_pass_kernel");
    check_device_status(ctx);
    MSBG_API_END
}

int msbg_morton_sort(msbg_ctx* ctx, const float* pos, size_t n, uint64_t* keys_out, uint32_t* perm_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && ((pos && keys_out && perm_out) || !n), "null argument");
    if (!n) return MSBG_OK;
    set_device(ctx);
    DevBuf io;
    io.reserve(n * 12 + n * 8 + n * 4 + 1024);
    float* dpos = io.as<float>();
    uint64_t* dk = (uint64_t*)((char*)io.p + ((n * 12 + 255) & ~size_t(255)));
    uint32_t* dp = (uint32_t*)((char*)dk + ((n * 8 + 255) & ~size_t(255)));
    CUDA_CHECK(cudaMemcpyAsync(dpos, pos, n * 12, cudaMemcpyHostToDevice, ctx->stream));
    morton_sort_device(ctx, dpos, n, dk, dp);
    CUDA_CHECK(cudaMemcpyAsync(keys_out, dk, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_CHECK(cudaMemcpyAsync(perm_out, dp, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    check_device_status(ctx);
    MSBG_API_END
}

int msbg_permute_device(msbg_ctx* ctx, const uint32_t* d_perm, size_t n, int width, const float* d_src, float* d_dst) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && ((d_perm && d_src && d_dst) || !n), "null argument");
    MSBG_REQUIRE(width >= 1 && width <= 16, "width must be 1..16");
    MSBG_REQUIRE(d_src != d_dst, "permute cannot run in place");
    if (!n) return MSBG_OK;
    set_device(ctx);
    begin_launch(ctx);
    const unsigned g = (unsigned)std::max<size_t>(div_up(n, 256), 1);
    if (width == 1) permute_kernel<1><<<g, 256, 0, ctx->stream>>>(d_perm, n, width, d_src, d_dst);
    else if (width == 3) permute_kernel<3><<<g, 256, 0, ctx->stream>>>(d_perm, n, width, d_src, d_dst);
    else permute_kernel<0><<<g, 256, 0, ctx->stream>>>(d_perm, n, width, d_src, d_dst);
    after_launch(ctx, "permute_kernel");
    MSBG_API_END
}

int msbg_bucket_indices_device(msbg_ctx* ctx, const uint64_t* d_bids, size_t n, uint64_t* d_particle_blocks,
                               uint64_t* d_starts, uint32_t* d_perm, size_t* n_blocks_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && d_starts && n_blocks_out && ((d_bids && d_particle_blocks && d_perm) || !n), "null argument");
    set_device(ctx);
    *n_blocks_out = bucket_indices_device(ctx, d_bids, n, d_particle_blocks, d_starts, d_perm);
    check_device_status(ctx);
    MSBG_API_END
}

int msbg_bucket_indices(msbg_ctx* ctx, const uint64_t* bids, size_t n, uint64_t* particle_blocks, uint64_t* starts,
                        uint32_t* perm, size_t* n_blocks_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && starts && n_blocks_out && ((bids && particle_blocks && perm) || !n), "null argument");
    set_device(ctx);
    if (!n) {
        starts[0] = 0;
        *n_blocks_out = 0;
        return MSBG_OK;
    }
    DevBuf io;
    size_t a = (n * 8 + 255) & ~size_t(255), p = (n * 4 + 255) & ~size_t(255);
    io.reserve(a * 3 + p + 512);
    uint64_t* db = io.as<uint64_t>();
    uint64_t* dblk = (uint64_t*)((char*)io.p + a);
    uint64_t* dst = (uint64_t*)((char*)io.p + 2 * a);
    uint32_t* dp = (uint32_t*)((char*)io.p + 3 * a + 256);
    CUDA_CHECK(cudaMemcpyAsync(db, bids, n * 8, cudaMemcpyHostToDevice, ctx->stream));
    size_t nb = bucket_indices_device(ctx, db, n, dblk, dst, dp);
    CUDA_CHECK(cudaMemcpyAsync(particle_blocks, dblk, nb * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_CHECK(cudaMemcpyAsync(starts, dst, (nb + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_CHECK(cudaMemcpyAsync(perm, dp, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    check_device_status(ctx);
    *n_blocks_out = nb;
    MSBG_API_END
}

}  // extern "C"
