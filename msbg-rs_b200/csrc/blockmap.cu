// blockmap.cu -- BlockMap (blockmap.rs:35-209) in device memory: an
// open-addressing hash from 64-bit block ids to 32-bit values, probed
// linearly from (key * 0x9e3779b97f4a7c15) & mask as the crate does, with
// EMPTY and TOMBSTONE sentinels and growth to twice the capacity when live
// entries plus tombstones would pass 3/4 of it.
//
// Batches run one thread per key.  A slot is claimed with a compare-and-swap
// of its key word; a thread first walks the probe chain to the first EMPTY
// slot looking for its key, so a key is never stored twice (the crate's
// insert reuses the first tombstone it meets without looking further, which
// can duplicate a key that was re-inserted after a removal on its chain).
// insert: batches are sorted by key first and the last value of each key is
// kept, as inserting the batch in order would.  update_add (the counting form
// of BlockMap::update(key, 1, |c| c + 1) that bucket_indices uses,
// particles/sort.rs:174-200) claims only EMPTY slots, whose value word is
// zero, and adds with integer atomics, so duplicate keys in one batch count
// exactly.
#include <algorithm>

#include "common.cuh"
#include "sort.cuh"

struct msbg_blockmap {
    msbg_ctx* ctx = nullptr;
    msbg::DevBuf keys, vals;     // [cap] u64, u32
    msbg::DevBuf counters;       // u64 [2]: live entries, tombstones
    uint64_t cap = 0;
};

namespace msbg {

constexpr uint64_t kBmEmpty = ~0ull;
constexpr uint64_t kBmTomb = ~0ull - 1;

__device__ __forceinline__ uint64_t bm_mix(uint64_t key) { return key * 0x9e3779b97f4a7c15ull; }

struct BmView {
    unsigned long long* keys;
    uint32_t* vals;
    unsigned long long* counters;
    uint64_t mask;
};

// Insert (key, val) for a key that appears once in its batch.
__global__ void bm_insert_kernel(BmView m, const uint64_t* __restrict__ in_keys, const uint32_t* __restrict__ in_vals,
                                 size_t n) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long key = in_keys[t];
        const uint32_t val = in_vals[t];
        uint64_t i = bm_mix(key) & m.mask;
        // existing entry on the chain?
        bool done = false;
        for (uint64_t probe = 0; probe <= m.mask; ++probe) {
            const unsigned long long k = m.keys[i];
            if (k == key) {
                m.vals[i] = val;
                done = true;
                break;
            }
            if (k == kBmEmpty) break;
            i = (i + 1) & m.mask;
        }
        if (done) continue;
        // claim the first free (EMPTY or TOMBSTONE) slot of the chain
        i = bm_mix(key) & m.mask;
        for (uint64_t probe = 0; probe <= m.mask; ++probe) {
            unsigned long long k = m.keys[i];
            while (k == kBmEmpty || k == kBmTomb) {
                const unsigned long long prev = atomicCAS(m.keys + i, k, key);
                if (prev == k) {
                    m.vals[i] = val;
                    atomicAdd(m.counters, 1ull);
                    if (k == kBmTomb) atomicAdd(m.counters + 1, ~0ull);  // one tombstone fewer
                    done = true;
                    break;
                }
                k = prev;
            }
            if (done) break;
            i = (i + 1) & m.mask;
        }
    }
}

// count(key) += 1, a missing key entering with count 1.
__global__ void bm_update_add_kernel(BmView m, const uint64_t* __restrict__ in_keys, size_t n) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long key = in_keys[t];
        uint64_t i = bm_mix(key) & m.mask;
        for (uint64_t probe = 0; probe <= m.mask; ++probe) {
            unsigned long long k = m.keys[i];
            if (k == kBmEmpty) {
                const unsigned long long prev = atomicCAS(m.keys + i, kBmEmpty, key);
                if (prev == kBmEmpty) {
                    atomicAdd(m.counters, 1ull);
                    k = key;
                } else {
                    k = prev;
                }
            }
            if (k == key) {
                atomicAdd(m.vals + i, 1u);
                break;
            }
            i = (i + 1) & m.mask;
        }
    }
}

__global__ void bm_get_kernel(BmView m, const uint64_t* __restrict__ in_keys, size_t n, uint32_t missing,
                              uint32_t* __restrict__ out) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long key = in_keys[t];
        uint64_t i = bm_mix(key) & m.mask;
        uint32_t v = missing;
        for (uint64_t probe = 0; probe <= m.mask; ++probe) {
            const unsigned long long k = m.keys[i];
            if (k == key) {
                v = m.vals[i];
                break;
            }
            if (k == kBmEmpty) break;
            i = (i + 1) & m.mask;
        }
        out[t] = v;
    }
}

__global__ void bm_remove_kernel(BmView m, const uint64_t* __restrict__ in_keys, size_t n) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long key = in_keys[t];
        uint64_t i = bm_mix(key) & m.mask;
        for (uint64_t probe = 0; probe <= m.mask; ++probe) {
            const unsigned long long k = m.keys[i];
            if (k == key) {
                if (atomicCAS(m.keys + i, key, kBmTomb) == key) {
                    atomicAdd(m.counters, ~0ull);  // one entry fewer
                    atomicAdd(m.counters + 1, 1ull);
                }
                break;
            }
            if (k == kBmEmpty) break;
            i = (i + 1) & m.mask;
        }
    }
}

// live flags of the table slots (for compaction)
__global__ void bm_live_kernel(const unsigned long long* __restrict__ keys, uint64_t cap, uint32_t* __restrict__ flags) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cap; i += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        flags[i] = (k != kBmEmpty && k != kBmTomb) ? 1u : 0u;
    }
}

__global__ void bm_gather_kernel(const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ vals,
                                 uint64_t cap, const uint32_t* __restrict__ flags, const uint32_t* __restrict__ off,
                                 uint64_t* __restrict__ out_keys, uint32_t* __restrict__ out_vals) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cap; i += (size_t)gridDim.x * blockDim.x) {
        if (!flags[i]) continue;
        out_keys[off[i]] = keys[i];
        out_vals[off[i]] = vals[i];
    }
}

// The last entry of each run of equal keys in a sorted batch (sorted by key,
// stably, so the last one is the batch's last occurrence).
__global__ void bm_last_of_run_kernel(const uint64_t* __restrict__ k, size_t n, uint32_t* __restrict__ flags) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        flags[i] = (i + 1 == n || k[i + 1] != k[i]) ? 1u : 0u;
}

__global__ void bm_compact_kernel(const uint64_t* __restrict__ k, const uint32_t* __restrict__ perm,
                                  const uint32_t* __restrict__ vals, size_t n, const uint32_t* __restrict__ flags,
                                  const uint32_t* __restrict__ off, uint64_t* __restrict__ ok, uint32_t* __restrict__ ov) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (!flags[i]) continue;
        ok[off[i]] = k[i];
        ov[off[i]] = vals[perm[i]];
    }
}

__global__ void bm_check_keys_kernel(const uint64_t* __restrict__ k, size_t n, int* __restrict__ bad) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (k[i] >= kBmTomb) atomicExch(bad, 1);
}

static unsigned bm_grid(size_t n) { return (unsigned)std::min<size_t>(std::max<size_t>(div_up(n, 256), 1), 148 * 16); }

static BmView view(msbg_blockmap* m) {
    return BmView{m->keys.as<unsigned long long>(), m->vals.as<uint32_t>(), m->counters.as<unsigned long long>(), m->cap - 1};
}

static void bm_counts(msbg_blockmap* m, uint64_t* live, uint64_t* tomb) {
    uint64_t c[2] = {0, 0};
    read_small(m->ctx, c, m->counters.p, 16);
    if (live) *live = c[0];
    if (tomb) *tomb = c[1];
}

static void bm_alloc(msbg_blockmap* m, uint64_t cap) {
    m->keys.reserve(cap * 8);
    m->vals.reserve(cap * 4);
    CUDA_CHECK(cudaMemsetAsync(m->keys.p, 0xff, cap * 8, m->ctx->stream));  // EMPTY
    CUDA_CHECK(cudaMemsetAsync(m->vals.p, 0, cap * 4, m->ctx->stream));
    CUDA_CHECK(cudaMemsetAsync(m->counters.p, 0, 16, m->ctx->stream));
    m->cap = cap;
}

static void require_keys(msbg_blockmap* m, const uint64_t* d_keys, size_t n, void* word) {
    int* bad = (int*)word;
    CUDA_CHECK(cudaMemsetAsync(bad, 0, 4, m->ctx->stream));
    begin_launch(m->ctx);
    bm_check_keys_kernel<<<bm_grid(n), 256, 0, m->ctx->stream>>>(d_keys, n, bad);
    after_launch(m->ctx, "bm_check_keys_kernel");
    int h = 0;
    read_small(m->ctx, &h, bad, 4);
    MSBG_REQUIRE(!h, "a block id collides with a sentinel (2^64 - 1 or 2^64 - 2)");
}

// Live entries, sorted by key (sorted_pairs, blockmap.rs:177-187); returns the count.
static size_t bm_pairs(msbg_blockmap* m, uint64_t* d_keys_out, uint32_t* d_vals_out) {
    msbg_ctx* ctx = m->ctx;
    uint64_t live = 0;
    bm_counts(m, &live, nullptr);
    if (!live) return 0;
    ScratchLayout L;
    const size_t o_f = L.add<uint32_t>(m->cap), o_o = L.add<uint32_t>(m->cap), o_t = L.add<uint32_t>(4),
                 o_s = L.add<char>(scan_scratch_bytes(m->cap)), o_k = L.add<uint64_t>(live), o_v = L.add<uint32_t>(live),
                 o_rt = L.add<char>(radix_sort_scratch_bytes(live));
    char* b = scratch(ctx, L);
    begin_launch(ctx);
    bm_live_kernel<<<bm_grid(m->cap), 256, 0, ctx->stream>>>(m->keys.as<unsigned long long>(), m->cap,
                                                             ScratchLayout::at<uint32_t>(b, o_f));
    after_launch(ctx, "bm_live_kernel");
    exclusive_scan_u32(ctx, ScratchLayout::at<uint32_t>(b, o_f), ScratchLayout::at<uint32_t>(b, o_o), m->cap,
                       ScratchLayout::at<uint32_t>(b, o_t), ScratchLayout::at<char>(b, o_s));
    begin_launch(ctx);
    bm_gather_kernel<<<bm_grid(m->cap), 256, 0, ctx->stream>>>(
        m->keys.as<unsigned long long>(), m->vals.as<uint32_t>(), m->cap, ScratchLayout::at<uint32_t>(b, o_f),
        ScratchLayout::at<uint32_t>(b, o_o), ScratchLayout::at<uint64_t>(b, o_k), ScratchLayout::at<uint32_t>(b, o_v));
    after_launch(ctx, "bm_gather_kernel");
    radix_sort_pairs(ctx, ScratchLayout::at<uint64_t>(b, o_k), ScratchLayout::at<uint32_t>(b, o_v), d_keys_out, d_vals_out,
                     live, 64, ScratchLayout::at<char>(b, o_rt));
    return live;
}

// Grows (and drops tombstones) so that `extra` more entries keep the load at
// or below 3/4 (BlockMap::grow, blockmap.rs:189-197, doubling the capacity).
static void bm_reserve(msbg_blockmap* m, size_t extra) {
    uint64_t live = 0, tomb = 0;
    bm_counts(m, &live, &tomb);
    if (live + tomb + extra <= m->cap * 3 / 4) return;
    uint64_t cap = m->cap;
    while (live + extra > cap * 3 / 4) cap *= 2;
    DevBuf k, v;
    k.reserve(std::max<uint64_t>(live, 1) * 8);
    v.reserve(std::max<uint64_t>(live, 1) * 4);
    const size_t n = bm_pairs(m, k.as<uint64_t>(), v.as<uint32_t>());
    bm_alloc(m, cap);
    if (n) {
        begin_launch(m->ctx);
        bm_insert_kernel<<<bm_grid(n), 256, 0, m->ctx->stream>>>(view(m), k.as<uint64_t>(), v.as<uint32_t>(), n);
        after_launch(m->ctx, "bm_insert_kernel");
    }
    sync(m->ctx);  // k, v die at return
}

static void bm_insert(msbg_blockmap* m, const uint64_t* d_keys, const uint32_t* d_vals, size_t n) {
    msbg_ctx* ctx = m->ctx;
    if (!n) return;
    ScratchLayout L;
    const size_t o_sk = L.add<uint64_t>(n), o_p = L.add<uint32_t>(n), o_f = L.add<uint32_t>(n), o_o = L.add<uint32_t>(n),
                 o_t = L.add<uint32_t>(4), o_uk = L.add<uint64_t>(n), o_uv = L.add<uint32_t>(n),
                 o_rt = L.add<char>(std::max(radix_sort_scratch_bytes(n), scan_scratch_bytes(n))), o_w = L.add<int>(4);
    char* b = scratch(ctx, L);
    require_keys(m, d_keys, n, ScratchLayout::at<int>(b, o_w));
    radix_sort_pairs(ctx, d_keys, nullptr, ScratchLayout::at<uint64_t>(b, o_sk), ScratchLayout::at<uint32_t>(b, o_p), n, 64,
                     ScratchLayout::at<char>(b, o_rt));
    begin_launch(ctx);
    bm_last_of_run_kernel<<<bm_grid(n), 256, 0, ctx->stream>>>(ScratchLayout::at<uint64_t>(b, o_sk), n,
                                                               ScratchLayout::at<uint32_t>(b, o_f));
    after_launch(ctx, "bm_last_of_run_kernel");
    exclusive_scan_u32(ctx, ScratchLayout::at<uint32_t>(b, o_f), ScratchLayout::at<uint32_t>(b, o_o), n,
                       ScratchLayout::at<uint32_t>(b, o_t), ScratchLayout::at<char>(b, o_rt));
    begin_launch(ctx);
    bm_compact_kernel<<<bm_grid(n), 256, 0, ctx->stream>>>(
        ScratchLayout::at<uint64_t>(b, o_sk), ScratchLayout::at<uint32_t>(b, o_p), d_vals, n,
        ScratchLayout::at<uint32_t>(b, o_f), ScratchLayout::at<uint32_t>(b, o_o), ScratchLayout::at<uint64_t>(b, o_uk),
        ScratchLayout::at<uint32_t>(b, o_uv));
    after_launch(ctx, "bm_compact_kernel");
    uint32_t u = 0;
    read_small(ctx, &u, ScratchLayout::at<uint32_t>(b, o_t), 4);
    // growth may reuse the scratch arena: keep the unique batch in a buffer of its own
    DevBuf uk, uv;
    uk.reserve((size_t)u * 8 + 8);
    uv.reserve((size_t)u * 4 + 4);
    CUDA_CHECK(cudaMemcpyAsync(uk.p, ScratchLayout::at<uint64_t>(b, o_uk), (size_t)u * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    CUDA_CHECK(cudaMemcpyAsync(uv.p, ScratchLayout::at<uint32_t>(b, o_uv), (size_t)u * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    bm_reserve(m, u);
    begin_launch(ctx);
    bm_insert_kernel<<<bm_grid(u), 256, 0, ctx->stream>>>(view(m), uk.as<uint64_t>(), uv.as<uint32_t>(), u);
    after_launch(ctx, "bm_insert_kernel");
    sync(ctx);  // uk, uv die at return
}

}  // namespace msbg

using namespace msbg;

extern "C" {

int msbg_blockmap_create(msbg_ctx* ctx, uint64_t capacity, msbg_blockmap** out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && out, "null argument");
    set_device(ctx);
    uint64_t cap = 4;
    while (cap < capacity) cap *= 2;  // with_capacity: max(4).next_power_of_two()
    auto* m = new msbg_blockmap();
    m->ctx = ctx;
    try {
        m->counters.reserve(16);
        bm_alloc(m, cap);
        sync(ctx);
    } catch (...) {
        delete m;
        throw;
    }
    *out = m;
    MSBG_API_END
}

int msbg_blockmap_destroy(msbg_blockmap* m) {
    MSBG_API_BEGIN
    if (m) {
        set_device(m->ctx);
        sync(m->ctx);
        delete m;
    }
    MSBG_API_END
}

int msbg_blockmap_len(msbg_blockmap* m, uint64_t* len_out, uint64_t* capacity_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m, "null argument");
    set_device(m->ctx);
    uint64_t live = 0;
    bm_counts(m, &live, nullptr);
    if (len_out) *len_out = live;
    if (capacity_out) *capacity_out = m->cap;
    MSBG_API_END
}

int msbg_blockmap_insert_device(msbg_blockmap* m, const uint64_t* d_keys, const uint32_t* d_vals, size_t n) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && ((d_keys && d_vals) || !n), "null argument");
    MSBG_REQUIRE(n < (1ULL << 32), "batches hold < 2^32 keys");
    set_device(m->ctx);
    bm_insert(m, d_keys, d_vals, n);
    MSBG_API_END
}

int msbg_blockmap_update_add_device(msbg_blockmap* m, const uint64_t* d_keys, size_t n) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && (d_keys || !n), "null argument");
    set_device(m->ctx);
    if (!n) return MSBG_OK;
    ScratchLayout L;
    const size_t o_w = L.add<int>(4);
    char* b = scratch(m->ctx, L);
    require_keys(m, d_keys, n, ScratchLayout::at<int>(b, o_w));
    bm_reserve(m, n);  // at most n new keys
    begin_launch(m->ctx);
    bm_update_add_kernel<<<bm_grid(n), 256, 0, m->ctx->stream>>>(view(m), d_keys, n);
    after_launch(m->ctx, "bm_update_add_kernel");
    MSBG_API_END
}

int msbg_blockmap_get_device(msbg_blockmap* m, const uint64_t* d_keys, size_t n, uint32_t missing, uint32_t* d_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && ((d_keys && d_out) || !n), "null argument");
    set_device(m->ctx);
    if (!n) return MSBG_OK;
    begin_launch(m->ctx);
    bm_get_kernel<<<bm_grid(n), 256, 0, m->ctx->stream>>>(view(m), d_keys, n, missing, d_out);
    after_launch(m->ctx, "bm_get_kernel");
    MSBG_API_END
}

int msbg_blockmap_remove_device(msbg_blockmap* m, const uint64_t* d_keys, size_t n) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && (d_keys || !n), "null argument");
    set_device(m->ctx);
    if (!n) return MSBG_OK;
    begin_launch(m->ctx);
    bm_remove_kernel<<<bm_grid(n), 256, 0, m->ctx->stream>>>(view(m), d_keys, n);
    after_launch(m->ctx, "bm_remove_kernel");
    MSBG_API_END
}

int msbg_blockmap_sorted_pairs_device(msbg_blockmap* m, uint64_t* d_keys_out, uint32_t* d_vals_out, size_t cap,
                                      size_t* n_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(m && n_out, "null argument");
    set_device(m->ctx);
    uint64_t live = 0;
    bm_counts(m, &live, nullptr);
    *n_out = live;
    if (!d_keys_out) return MSBG_OK;
    MSBG_REQUIRE(d_vals_out && cap >= live, "output arrays smaller than the map");
    bm_pairs(m, d_keys_out, d_vals_out);
    sync(m->ctx);
    MSBG_API_END
}

}  // extern "C"
