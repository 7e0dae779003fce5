// grid.cu -- context, device sparse grid, block transfer and halo gather.
#include <algorithm>
#include <cstring>

#include "grid.cuh"
#include "sort.cuh"
#include "sweep.cuh"

namespace msbg {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

void raise_device_status(msbg_ctx* ctx, int word) {
    if (!word) return;
    CUDA_CHECK(cudaMemsetAsync(ctx->status.p, 0, 4, ctx->stream));
    std::string what;
    if (word & 1) what += "an mbarrier wait inside a tensor-core kernel";
    if (word & 2) what += std::string(what.empty() ? "" : " and ") + "a radix-sort look-back";
    if (word & 4) what += std::string(what.empty() ? "" : " and ") + "a P2G tile-order wait";
    if (word & 8) what += std::string(what.empty() ? "" : " and ") + "a sweep's wait for its neighbours";
    MSBG_THROW(MSBG_ERR_TIMEOUT, what + " waited past its time limit and gave up");
}

void check_device_status(msbg_ctx* ctx) {
    int h = 0;
    read_small(ctx, &h, ctx->status.p, 4);
    raise_device_status(ctx, h);
}

__global__ void readback_kernel(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, size_t n) {
    if ((((uintptr_t)src | (uintptr_t)dst | n) & 3) == 0) {
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n / 4; i += (size_t)gridDim.x * blockDim.x)
            reinterpret_cast<uint32_t*>(dst)[i] = reinterpret_cast<const uint32_t*>(src)[i];
    } else {
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
            dst[i] = src[i];
    }
}

void SmallReads::add(void* host_dst, const void* dev_src, size_t bytes) {
    if (!bytes) return;
    const size_t off = (used_ + 15) & ~size_t(15);
    if (ctx_->rb_dev && off + bytes <= ctx_->rb_cap) {
        begin_launch(ctx_);
        readback_kernel<<<(unsigned)std::min<size_t>(div_up(bytes, 1024), 64), 256, 0, ctx_->stream>>>(
            (const uint8_t*)dev_src, (uint8_t*)ctx_->rb_dev + off, bytes);
        after_launch(ctx_, "readback_kernel");
        items_.push_back({host_dst, off, bytes, true});
        used_ = off + bytes;
    } else {
        CUDA_CHECK(cudaMemcpyAsync(host_dst, dev_src, bytes, cudaMemcpyDeviceToHost, ctx_->stream));
        items_.push_back({host_dst, 0, bytes, false});
    }
}

void SmallReads::wait() {
    sync(ctx_);
    for (const Item& it : items_)
        if (it.staged) std::memcpy(it.dst, (const char*)ctx_->rb_host + it.off, it.bytes);
    items_.clear();
    used_ = 0;
}

char* scratch(msbg_ctx* ctx, const ScratchLayout& L) {
    if (L.size > ctx->scratch.bytes) {
        // Grow preserving contents: a multi-phase pipeline extends its layout
        // after the first phase and keeps the first phase's offsets.
        size_t grow = std::max(L.size, ctx->scratch.bytes + ctx->scratch.bytes / 2);
        void* p = nullptr;
        CUDA_CHECK(cudaMalloc(&p, grow));
        if (ctx->scratch.p)
            CUDA_CHECK(cudaMemcpyAsync(p, ctx->scratch.p, ctx->scratch.bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
        ctx->scratch.release();
        ctx->scratch.p = p;
        ctx->scratch.bytes = grow;
    }
    return ctx->scratch.as<char>();
}

void resolve_timing(msbg_ctx* ctx) {
    if (ctx->pending.empty()) return;
    CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    for (auto& p : ctx->pending) {
        float ms = 0.0f;
        CUDA_CHECK(cudaEventElapsedTime(&ms, p.a, p.b));
        auto& t = ctx->totals[p.name];
        t.first += 1;
        t.second += ms;
        ctx->pool.push_back(p.a);
        ctx->pool.push_back(p.b);
    }
    ctx->pending.clear();
}

float quantize_roundtrip(int dtype, float v) {
    if (dtype == MSBG_U16) {
        float r = roundf(v * 65535.0f);
        r = r > 0.0f ? r : 0.0f;
        r = r < 65535.0f ? r : 65535.0f;
        return (float)(uint16_t)r * (1.0f / 65535.0f);
    }
    if (dtype == MSBG_BF16) {
        uint32_t u;
        memcpy(&u, &v, 4);
        if ((u & 0x7fffffffu) > 0x7f800000u) return v;
        u += 0x7fffu + ((u >> 16) & 1u);
        u &= 0xffff0000u;
        float f;
        memcpy(&f, &u, 4);
        return f;
    }
    if (dtype == MSBG_U8) {
        float r = roundf(v * 255.0f);
        r = r > 0.0f ? r : 0.0f;
        r = r < 255.0f ? r : 255.0f;
        return (float)(uint8_t)r * (1.0f / 255.0f);
    }
    if (dtype == MSBG_F16) return __half2float(__float2half_rn(v));
    return v;
}

void HostHash::build(const std::unordered_map<uint64_t, int32_t>& m) {
    size_t cap = 16;
    while (cap < 2 * m.size() + 16) cap <<= 1;
    keys.assign(cap, kHashEmpty);
    vals.assign(cap, kCodeEmpty);
    mask = (uint32_t)(cap - 1);
    shift = 64 - ilog2i(cap);
    for (const auto& kv : m) {
        uint32_t i = hash_slot(kv.first, shift);
        while (keys[i] != kHashEmpty) i = (i + 1) & mask;
        keys[i] = kv.first;
        vals[i] = kv.second;
    }
}

DevHash device_hash(msbg_grid* g) {
    if (g->hash_dirty) {
        HostHash h;
        h.build(g->map);
        g->hkeys.reserve(h.keys.size() * 8);
        g->hvals.reserve(h.vals.size() * 4);
        CUDA_CHECK(cudaMemcpyAsync(g->hkeys.p, h.keys.data(), h.keys.size() * 8, cudaMemcpyHostToDevice, g->ctx->stream));
        CUDA_CHECK(cudaMemcpyAsync(g->hvals.p, h.vals.data(), h.vals.size() * 4, cudaMemcpyHostToDevice, g->ctx->stream));
        // The host vectors die at return: make the copies complete first.
        sync(g->ctx);
        g->hmask = h.mask;
        g->hshift = h.shift;
        g->hash_dirty = false;
    }
    return DevHash{g->hkeys.as<uint64_t>(), g->hvals.as<int32_t>(), g->hmask, g->hshift};
}

const int32_t* device_dense(msbg_grid* g) {
    if (g->n_blocks > kDenseMaxBlocks) return nullptr;
    if (g->dense_dirty || g->hash_dirty) {
        std::vector<int32_t> t(g->n_blocks, kCodeEmpty);
        for (const auto& kv : g->map) t[kv.first] = kv.second;
        g->dense.reserve(t.size() * 4);
        CUDA_CHECK(cudaMemcpyAsync(g->dense.p, t.data(), t.size() * 4, cudaMemcpyHostToDevice, g->ctx->stream));
        sync(g->ctx);
        g->dense_dirty = false;
    }
    return g->dense.as<int32_t>();
}

int32_t grid_code(const msbg_grid* g, uint64_t bid) {
    auto it = g->map.find(bid);
    return it == g->map.end() ? kCodeEmpty : it->second;
}

void block_coords(const msbg_grid* g, uint64_t bid, int64_t* bx, int64_t* by, int64_t* bz) {
    *bx = (int64_t)(bid % g->nx);
    *by = (int64_t)((bid / g->nx) % g->ny);
    *bz = (int64_t)(bid / g->nxy);
}

void grid_reserve(msbg_grid* g, size_t need) {
    if (need <= g->cap_slots) return;
    size_t cap = std::max<size_t>(need, g->cap_slots + g->cap_slots / 2);
    cap = std::max<size_t>(cap, 8);
    void* p = nullptr;
    CUDA_CHECK(cudaMalloc(&p, cap * g->block_elems * g->esize));
    // Callers list the new slots before reserving them, so only the old
    // capacity holds data to keep.
    const size_t keep = std::min(g->n_slots(), g->cap_slots);
    if (g->payload.p && keep)
        CUDA_CHECK(cudaMemcpyAsync(p, g->payload.p, keep * g->block_elems * g->esize, cudaMemcpyDeviceToDevice,
                                   g->ctx->stream));
    sync(g->ctx);
    g->payload.release();
    g->payload.p = p;
    g->payload.bytes = cap * g->block_elems * g->esize;
    g->cap_slots = cap;
}

template <class E>
__global__ void fill_slots_kernel(typename E::T* payload, const int32_t* slots, size_t count,
                                  size_t block_elems, float value) {
    typename E::T v = E::store(value);
    for (size_t k = blockIdx.x; k < count; k += gridDim.x) {
        int32_t s = slots[k];
        if (s < 0) continue;
        typename E::T* dst = payload + (size_t)s * block_elems;
        for (size_t i = threadIdx.x; i < block_elems; i += blockDim.x) dst[i] = v;
    }
}

void grid_fill_slots(msbg_grid* g, const int32_t* d_slots, size_t count, float value) {
    if (!count) return;
    unsigned grid = (unsigned)std::min<size_t>(count, 65535);
    begin_launch(g->ctx);
    if (g->dtype == MSBG_F32)
        fill_slots_kernel<ElemF32><<<grid, 256, 0, g->ctx->stream>>>((float*)g->payload.p, d_slots, count, g->block_elems, value);
    else if (g->dtype == MSBG_U16)
        fill_slots_kernel<ElemU16><<<grid, 256, 0, g->ctx->stream>>>((uint16_t*)g->payload.p, d_slots, count, g->block_elems, value);
    else if (g->dtype == MSBG_U8)
        fill_slots_kernel<ElemU8><<<grid, 256, 0, g->ctx->stream>>>((uint8_t*)g->payload.p, d_slots, count, g->block_elems, value);
    else if (g->dtype == MSBG_F16)
        fill_slots_kernel<ElemF16><<<grid, 256, 0, g->ctx->stream>>>((uint16_t*)g->payload.p, d_slots, count, g->block_elems, value);
    else
        fill_slots_kernel<ElemBF16><<<grid, 256, 0, g->ctx->stream>>>((uint16_t*)g->payload.p, d_slots, count, g->block_elems, value);
    after_launch(g->ctx, "fill_slots_kernel");
}

void grid_ensure(msbg_grid* g, const uint64_t* bids, size_t n, int32_t* slots) {
    std::vector<int32_t> fresh;
    size_t first_new = g->n_slots();
    for (size_t k = 0; k < n; ++k) {
        uint64_t bid = bids[k];
        if (bid >= g->n_blocks) MSBG_THROW(MSBG_ERR_ARG, "block id out of range");
        auto it = g->map.find(bid);
        int32_t s;
        if (it != g->map.end() && it->second >= 0) {
            s = it->second;
        } else {
            s = (int32_t)g->slot_bid.size();
            g->slot_bid.push_back(bid);
            g->map[bid] = s;
            fresh.push_back(s);
        }
        if (slots) slots[k] = s;
    }
    if (!fresh.empty()) {
        g->version++;
        g->hash_dirty = true;
        g->dense_dirty = true;
        grid_reserve(g, g->n_slots());
        // A private buffer, not the context arena: pipelines call this while
        // their own temporaries live in the arena.
        DevBuf tmp;
        tmp.reserve(fresh.size() * 4);
        int32_t* d = tmp.as<int32_t>();
        CUDA_CHECK(cudaMemcpyAsync(d, fresh.data(), fresh.size() * 4, cudaMemcpyHostToDevice, g->ctx->stream));
        grid_fill_slots(g, d, fresh.size(), g->empty_value);
        sync(g->ctx);
        (void)first_new;
    }
}

// ---------------------------------------------------------------------------
// Block materialisation from a device list (ensure_blocks_parallel,
// sparse_grid.rs:326-355): the table lookups, the deduplication and the
// table updates run on the device; only the ids of the blocks that are new
// come back to the host (to keep its mirror of the table), so a block set
// that changes every step costs one small read instead of a rebuild and
// upload of the whole table.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int32_t dev_code(const int32_t* dense, const DevHash& h, uint64_t bid) {
    return dense ? dense[bid] : hash_find(h, bid);
}

// flags[i] = 1 for the first of each run of equal (sorted) ids whose block is
// not a value block yet; bad = an id out of range.
__global__ void ens_new_kernel(const uint64_t* __restrict__ sorted, size_t n, uint64_t n_blocks, const int32_t* dense,
                               DevHash h, uint32_t* __restrict__ flags, int* __restrict__ bad) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t b = sorted[i];
        if (b >= n_blocks) {
            atomicExch(bad, 1);
            flags[i] = 0;
            continue;
        }
        flags[i] = (i == 0 || sorted[i - 1] != b) && dev_code(dense, h, b) < 0 ? 1u : 0u;
    }
}

__global__ void ens_compact_kernel(const uint64_t* __restrict__ sorted, size_t n, const uint32_t* __restrict__ flags,
                                   const uint32_t* __restrict__ off, uint64_t* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (flags[i]) out[off[i]] = sorted[i];
}

// New blocks get slots first_slot + rank: written into the dense table, or
// inserted into the hash (linear probing from hash_slot; a full dummy's entry
// takes the slot), and listed for the fill.
__global__ void ens_insert_kernel(const uint64_t* __restrict__ fresh, size_t n, int32_t first_slot, int32_t* dense,
                                  unsigned long long* hkeys, int32_t* hvals, uint32_t hmask, int hshift,
                                  int32_t* __restrict__ fresh_slots) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long b = fresh[i];
        const int32_t s = first_slot + (int32_t)i;
        fresh_slots[i] = s;
        if (dense) dense[b] = s;
        if (hkeys) {
            uint32_t j = hash_slot(b, hshift);
            for (uint32_t probe = 0; probe <= hmask; ++probe) {
                const unsigned long long k = atomicCAS(hkeys + j, (unsigned long long)kHashEmpty, b);
                if (k == kHashEmpty || k == b) {
                    hvals[j] = s;
                    break;
                }
                j = (j + 1) & hmask;
            }
        }
    }
}

__global__ void ens_slots_kernel(const uint64_t* __restrict__ bids, size_t n, const int32_t* dense, DevHash h,
                                 int32_t* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = dev_code(dense, h, bids[i]);
}

void grid_ensure_device(msbg_grid* g, const uint64_t* d_bids, size_t n, int32_t* d_slots_out) {
    msbg_ctx* ctx = g->ctx;
    if (!n) return;
    MSBG_REQUIRE(n < (1ULL << 32), "at most 2^32 - 1 block ids per call");
    const int32_t* dense = device_dense(g);
    DevHash h = device_hash(g);
    DevBuf tmp;  // private: callers may hold the context arena
    const size_t b_sorted = (n * 8 + 255) & ~size_t(255), b_perm = (n * 4 + 255) & ~size_t(255);
    const size_t b_flags = b_perm, b_off = b_perm, b_fresh = b_sorted;
    const size_t b_rs = (std::max(radix_sort_scratch_bytes(n), scan_scratch_bytes(n)) + 255) & ~size_t(255);
    tmp.reserve(b_sorted + b_perm + b_flags + b_off + b_fresh + b_rs + 256);
    char* p = (char*)tmp.p;
    uint64_t* sorted = (uint64_t*)p; p += b_sorted;
    uint32_t* perm = (uint32_t*)p;   p += b_perm;
    uint32_t* flags = (uint32_t*)p;  p += b_flags;
    uint32_t* off = (uint32_t*)p;    p += b_off;
    uint64_t* fresh = (uint64_t*)p;  p += b_fresh;
    char* rs = p;                    p += b_rs;
    int* words = (int*)p;            // [0] bad, [1..] scan total
    CUDA_CHECK(cudaMemsetAsync(words, 0, 16, ctx->stream));
    radix_sort_pairs(ctx, d_bids, nullptr, sorted, perm, n, ilog2i(g->n_blocks + 1) + 1, rs);
    const unsigned grid = (unsigned)std::min<size_t>(std::max<size_t>(div_up(n, 256), 1), 148 * 16);
    begin_launch(ctx);
    ens_new_kernel<<<grid, 256, 0, ctx->stream>>>(sorted, n, g->n_blocks, dense, h, flags, words);
    after_launch(ctx, "ens_new_kernel");
    exclusive_scan_u32(ctx, flags, off, n, (uint32_t*)(words + 1), rs);
    begin_launch(ctx);
    ens_compact_kernel<<<grid, 256, 0, ctx->stream>>>(sorted, n, flags, off, fresh);
    after_launch(ctx, "ens_compact_kernel");
    int hw[2] = {0, 0};
    read_small(ctx, hw, words, 8);
    MSBG_REQUIRE(!hw[0], "block id out of range");
    const size_t nf = (size_t)(uint32_t)hw[1];
    if (nf) {
        std::vector<uint64_t> fresh_h(nf);
        read_small(ctx, fresh_h.data(), fresh, nf * 8);
        const int32_t first = (int32_t)g->slot_bid.size();
        for (size_t i = 0; i < nf; ++i) {
            g->slot_bid.push_back(fresh_h[i]);
            g->map[fresh_h[i]] = first + (int32_t)i;
        }
        g->version++;
        grid_reserve(g, g->n_slots());
        // the hash stays below half load: insert in place, else rebuild it on next use
        const bool hash_in_place = !g->hash_dirty && g->map.size() * 2 <= (size_t)g->hmask + 1;
        if (!hash_in_place) g->hash_dirty = true;
        int32_t* fresh_slots = (int32_t*)perm;  // the permutation is no longer needed
        begin_launch(ctx);
        ens_insert_kernel<<<(unsigned)std::min<size_t>(div_up(nf, 256), 148 * 16), 256, 0, ctx->stream>>>(
            fresh, nf, first, dense && !g->dense_dirty ? const_cast<int32_t*>(dense) : nullptr,
            hash_in_place ? g->hkeys.as<unsigned long long>() : nullptr, g->hvals.as<int32_t>(), g->hmask, g->hshift,
            fresh_slots);
        after_launch(ctx, "ens_insert_kernel");
        grid_fill_slots(g, fresh_slots, nf, g->empty_value);
    }
    if (d_slots_out) {
        const int32_t* dense2 = device_dense(g);
        DevHash h2 = device_hash(g);
        begin_launch(ctx);
        ens_slots_kernel<<<grid, 256, 0, ctx->stream>>>(d_bids, n, dense2, h2, d_slots_out);
        after_launch(ctx, "ens_slots_kernel");
    }
    sync(ctx);  // tmp dies at return
}

// ---------------------------------------------------------------------------
// Block transfer kernels
// ---------------------------------------------------------------------------
template <class T>
__global__ void scatter_blocks_kernel(T* payload, const int32_t* slots, const T* src, size_t n, size_t be) {
    for (size_t k = blockIdx.x; k < n; k += gridDim.x) {
        T* dst = payload + (size_t)slots[k] * be;
        const T* s = src + k * be;
        for (size_t i = threadIdx.x; i < be; i += blockDim.x) dst[i] = s[i];
    }
}

// codes[k]: slot >= 0 copies the block, kCodeFull the full value, else empty.
template <class T>
__global__ void gather_blocks_kernel(const T* payload, const int32_t* codes, T* dst, size_t n, size_t be,
                                     T empty_v, T full_v) {
    for (size_t k = blockIdx.x; k < n; k += gridDim.x) {
        int32_t c = codes[k];
        T* d = dst + k * be;
        if (c >= 0) {
            const T* s = payload + (size_t)c * be;
            for (size_t i = threadIdx.x; i < be; i += blockDim.x) d[i] = s[i];
        } else {
            T v = c == kCodeFull ? full_v : empty_v;
            for (size_t i = threadIdx.x; i < be; i += blockDim.x) d[i] = v;
        }
    }
}

// The stored bit pattern of a float constant (f32 bits, or the quantised
// u16 / bf16 element).
template <class T> static T host_store(int dtype, float v) {
    if constexpr (sizeof(T) == 4) {
        T t;
        memcpy(&t, &v, 4);
        return t;
    } else {
        float q = quantize_roundtrip(dtype, v);
        if (dtype == MSBG_U16) return (T)lrintf(q * 65535.0f);
        if (dtype == MSBG_U8) return (T)lrintf(q * 255.0f);
        if (dtype == MSBG_F16) return (T)__half_as_ushort(__float2half_rn(q));
        uint32_t u;
        memcpy(&u, &q, 4);
        return (T)(u >> 16);
    }
}

static void write_blocks(msbg_grid* g, const uint64_t* bids, size_t n, const void* payload, bool device_src) {
    if (!n) return;
    std::vector<int32_t> slots(n);
    grid_ensure(g, bids, n, slots.data());
    size_t bytes = n * g->block_elems * g->esize;
    ScratchLayout L;
    size_t os = L.add<int32_t>(n);
    size_t ob = device_src ? 0 : L.add<char>(bytes);
    char* base = scratch(g->ctx, L);
    int32_t* d_slots = ScratchLayout::at<int32_t>(base, os);
    const void* src = payload;
    CUDA_CHECK(cudaMemcpyAsync(d_slots, slots.data(), n * 4, cudaMemcpyHostToDevice, g->ctx->stream));
    if (!device_src) {
        void* d = ScratchLayout::at<char>(base, ob);
        CUDA_CHECK(cudaMemcpyAsync(d, payload, bytes, cudaMemcpyHostToDevice, g->ctx->stream));
        src = d;
    }
    unsigned grid = (unsigned)std::min<size_t>(n, 65535);
    begin_launch(g->ctx);
    if (g->esize == 4)
        scatter_blocks_kernel<uint32_t><<<grid, 256, 0, g->ctx->stream>>>((uint32_t*)g->payload.p, d_slots, (const uint32_t*)src, n, g->block_elems);
    else if (g->esize == 1)
        scatter_blocks_kernel<uint8_t><<<grid, 256, 0, g->ctx->stream>>>((uint8_t*)g->payload.p, d_slots, (const uint8_t*)src, n, g->block_elems);
    else
        scatter_blocks_kernel<uint16_t><<<grid, 256, 0, g->ctx->stream>>>((uint16_t*)g->payload.p, d_slots, (const uint16_t*)src, n, g->block_elems);
    after_launch(g->ctx, "scatter_blocks_kernel");
    sync(g->ctx);  // host vectors go out of scope
}

static void read_blocks(msbg_grid* g, const uint64_t* bids, size_t n, void* out, bool device_dst) {
    if (!n) return;
    std::vector<int32_t> codes(n);
    for (size_t k = 0; k < n; ++k) {
        if (bids[k] >= g->n_blocks) MSBG_THROW(MSBG_ERR_ARG, "block id out of range");
        codes[k] = grid_code(g, bids[k]);
    }
    size_t bytes = n * g->block_elems * g->esize;
    ScratchLayout L;
    size_t oc = L.add<int32_t>(n);
    size_t ob = device_dst ? 0 : L.add<char>(bytes);
    char* base = scratch(g->ctx, L);
    int32_t* d_codes = ScratchLayout::at<int32_t>(base, oc);
    void* dst = device_dst ? out : (void*)ScratchLayout::at<char>(base, ob);
    CUDA_CHECK(cudaMemcpyAsync(d_codes, codes.data(), n * 4, cudaMemcpyHostToDevice, g->ctx->stream));
    unsigned grid = (unsigned)std::min<size_t>(n, 65535);
    begin_launch(g->ctx);
    if (g->esize == 4)
        gather_blocks_kernel<uint32_t><<<grid, 256, 0, g->ctx->stream>>>(
            (const uint32_t*)g->payload.p, d_codes, (uint32_t*)dst, n, g->block_elems,
            host_store<uint32_t>(g->dtype, g->empty_value), host_store<uint32_t>(g->dtype, g->full_value));
    else if (g->esize == 1)
        gather_blocks_kernel<uint8_t><<<grid, 256, 0, g->ctx->stream>>>(
            (const uint8_t*)g->payload.p, d_codes, (uint8_t*)dst, n, g->block_elems,
            host_store<uint8_t>(g->dtype, g->empty_value), host_store<uint8_t>(g->dtype, g->full_value));
    else
        gather_blocks_kernel<uint16_t><<<grid, 256, 0, g->ctx->stream>>>(
            (const uint16_t*)g->payload.p, d_codes, (uint16_t*)dst, n, g->block_elems,
            host_store<uint16_t>(g->dtype, g->empty_value), host_store<uint16_t>(g->dtype, g->full_value));
    after_launch(g->ctx, "gather_blocks_kernel");
    if (!device_dst) CUDA_CHECK(cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToHost, g->ctx->stream));
    sync(g->ctx);
}

// ---------------------------------------------------------------------------
// Halo gather (multires/halo.rs:31-170), one CTA per requested block.
// ---------------------------------------------------------------------------
struct HaloArgs {
    const void* payload;
    DevHash hash;
    int64_t nx, ny, nz;
    int32_t sx, sy, sz;
    float empty, full;
};

template <class E, int BSX, int HALO>
__global__ void halo_gather_kernel(HaloArgs a, const uint64_t* bids, size_t n, int full_mode, int bc, float* out) {
    constexpr int HSX = BSX + 2 * HALO;
    constexpr int LG = BSX == 1 ? 0 : BSX == 2 ? 1 : BSX == 4 ? 2 : BSX == 8 ? 3 : BSX == 16 ? 4 : 5;
    __shared__ int32_t nb[27];
    __shared__ int8_t ok[3][HSX], dd[3][HSX];
    __shared__ int8_t ll[3][HSX];
    const typename E::T* payload = (const typename E::T*)a.payload;
    for (size_t k = blockIdx.x; k < n; k += gridDim.x) {
        uint64_t bid = bids[k];
        int64_t b0[3] = {(int64_t)(bid % a.nx), (int64_t)((bid / a.nx) % a.ny), (int64_t)(bid / (a.nx * a.ny))};
        __syncthreads();
        if (threadIdx.x < 27) {
            int dx = threadIdx.x % 3 - 1, dy = (threadIdx.x / 3) % 3 - 1, dz = threadIdx.x / 9 - 1;
            int64_t X = b0[0] + dx, Y = b0[1] + dy, Z = b0[2] + dz;
            int32_t c = kCodeEmpty;
            if (X >= 0 && Y >= 0 && Z >= 0 && X < a.nx && Y < a.ny && Z < a.nz)
                c = hash_find(a.hash, (uint64_t)X + (uint64_t)Y * a.nx + (uint64_t)Z * a.nx * a.ny);
            nb[threadIdx.x] = c;
        }
        if (threadIdx.x >= 32 && threadIdx.x < 32 + 3 * HSX) {
            int ax = (threadIdx.x - 32) / HSX, h = (threadIdx.x - 32) % HSX;
            int32_t smax = ax == 0 ? a.sx : ax == 1 ? a.sy : a.sz;
            int32_t g = (int32_t)(b0[ax] * BSX) + h - HALO, r;
            bool o = resolve_axis(g, smax - 1, bc, &r);
            ok[ax][h] = o;
            dd[ax][h] = o ? (int8_t)((r >> LG) - (int32_t)b0[ax] + 1) : 0;
            ll[ax][h] = o ? (int8_t)(r & (BSX - 1)) : 0;
        }
        __syncthreads();
        float* dst = out + k * (size_t)HSX * HSX * HSX;
        for (int i = threadIdx.x; i < HSX * HSX * HSX; i += blockDim.x) {
            int hx = i % HSX, hy = (i / HSX) % HSX, hz = i / (HSX * HSX);
            bool midx = hx >= HALO && hx < HALO + BSX, midy = hy >= HALO && hy < HALO + BSX,
                 midz = hz >= HALO && hz < HALO + BSX;
            float v = 0.0f;
            // full == 0 writes the middle segment of every row and the x-halo
            // columns of the centre rows only (halo.rs:150-152).
            if (full_mode || midx || (midy && midz)) {
                if (ok[0][hx] && ok[1][hy] && ok[2][hz]) {
                    int c = nb[dd[0][hx] + 3 * dd[1][hy] + 9 * dd[2][hz]];
                    if (c >= 0)
                        v = E::load(payload[(size_t)c * (BSX * BSX * BSX) + (ll[0][hx] | (ll[1][hy] << LG) | (ll[2][hz] << (2 * LG)))]);
                    else
                        v = c == kCodeFull ? a.full : a.empty;
                } else {
                    v = a.empty;
                }
            }
            dst[i] = v;
        }
    }
}

template <class E, int BSX>
static void launch_halo_gather_bsx(msbg_grid* g, const HaloArgs& a, const uint64_t* d_bids, size_t n, int halo,
                                   int full, int bc, float* d_out) {
    unsigned grid = (unsigned)std::min<size_t>(n, 65535);
    begin_launch(g->ctx);
    if (halo == 1)
        halo_gather_kernel<E, BSX, 1><<<grid, 256, 0, g->ctx->stream>>>(a, d_bids, n, full, bc, d_out);
    else
        halo_gather_kernel<E, BSX, 2><<<grid, 256, 0, g->ctx->stream>>>(a, d_bids, n, full, bc, d_out);
    after_launch(g->ctx, "halo_gather_kernel");
}

template <class E>
static void launch_halo_gather(msbg_grid* g, const HaloArgs& a, const uint64_t* d_bids, size_t n, int halo,
                               int full, int bc, float* d_out) {
    switch (g->bsx) {
        case 1: launch_halo_gather_bsx<E, 1>(g, a, d_bids, n, halo, full, bc, d_out); break;
        case 2: launch_halo_gather_bsx<E, 2>(g, a, d_bids, n, halo, full, bc, d_out); break;
        case 4: launch_halo_gather_bsx<E, 4>(g, a, d_bids, n, halo, full, bc, d_out); break;
        case 8: launch_halo_gather_bsx<E, 8>(g, a, d_bids, n, halo, full, bc, d_out); break;
        case 16: launch_halo_gather_bsx<E, 16>(g, a, d_bids, n, halo, full, bc, d_out); break;
        default: launch_halo_gather_bsx<E, 32>(g, a, d_bids, n, halo, full, bc, d_out); break;
    }
}

static void halo_gather(msbg_grid* g, const uint64_t* d_bids, size_t n, int halo, int full, int bc, float* d_out) {
    MSBG_REQUIRE(halo == 1 || halo == 2, "halo must be 1 or 2");
    MSBG_REQUIRE(bc >= 0 && bc <= 2, "bad boundary condition");
    MSBG_REQUIRE(halo <= g->bsx, "halo wider than a block");
    if (!n) return;
    HaloArgs a;
    a.payload = g->payload.p;
    a.hash = device_hash(g);
    a.nx = (int64_t)g->nx; a.ny = (int64_t)g->ny; a.nz = (int64_t)g->nz;
    a.sx = (int32_t)g->sx; a.sy = (int32_t)g->sy; a.sz = (int32_t)g->sz;
    a.empty = quantize_roundtrip(g->dtype, g->empty_value);
    a.full = quantize_roundtrip(g->dtype, g->full_value);
    if (g->dtype == MSBG_F32) launch_halo_gather<ElemF32>(g, a, d_bids, n, halo, full, bc, d_out);
    else if (g->dtype == MSBG_U16) launch_halo_gather<ElemU16>(g, a, d_bids, n, halo, full, bc, d_out);
    else if (g->dtype == MSBG_U8) launch_halo_gather<ElemU8>(g, a, d_bids, n, halo, full, bc, d_out);
    else if (g->dtype == MSBG_F16) launch_halo_gather<ElemF16>(g, a, d_bids, n, halo, full, bc, d_out);
    else launch_halo_gather<ElemBF16>(g, a, d_bids, n, halo, full, bc, d_out);
}

}  // namespace msbg

using namespace msbg;

msbg_grid::~msbg_grid() { delete plan; }

extern "C" {

const char* msbg_status_string(int s) {
    switch (s) {
        case MSBG_OK: return "ok";
        case MSBG_ERR_ARG: return "invalid argument";
        case MSBG_ERR_OOM: return "out of memory";
        case MSBG_ERR_TIMEOUT: return "device wait timed out";
        case MSBG_ERR_CUDA: return "CUDA error";
        case MSBG_ERR_STATE: return "invalid state";
        case MSBG_ERR_NUMERIC: return "numerical breakdown";
        default: return "unknown status";
    }
}

const char* msbg_last_error(void) { return g_last_error.c_str(); }


int msbg_ctx_create(int device, msbg_ctx** out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(out, "null output");
    int n = 0;
    CUDA_CHECK(cudaGetDeviceCount(&n));
    MSBG_REQUIRE(device >= 0 && device < n, "no such CUDA device");
    auto* c = new msbg_ctx;
    c->device = device;
    try {
        CUDA_CHECK(cudaSetDevice(device));
        CUDA_CHECK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->status.reserve(64);
        CUDA_CHECK(cudaMemsetAsync(c->status.p, 0, 64, c->stream));
        c->rb_cap = (size_t)1 << 20;
        CUDA_CHECK(cudaHostAlloc(&c->rb_host, c->rb_cap, cudaHostAllocMapped));
        CUDA_CHECK(cudaHostGetDevicePointer(&c->rb_dev, c->rb_host, 0));
        CUDA_CHECK(cudaStreamSynchronize(c->stream));
    } catch (...) {
        if (c->rb_host) cudaFreeHost(c->rb_host);
        delete c;
        throw;
    }
    *out = c;
    MSBG_API_END
}

int msbg_ctx_destroy(msbg_ctx* ctx) {
    MSBG_API_BEGIN
    if (!ctx) return MSBG_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& p : ctx->pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    for (auto e : ctx->pool) cudaEventDestroy(e);
    if (ctx->open) cudaEventDestroy(ctx->open);
    ctx->scratch.release();
    ctx->status.release();
    if (ctx->rb_host) cudaFreeHost(ctx->rb_host);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    MSBG_API_END
}

int msbg_ctx_synchronize(msbg_ctx* ctx) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx, "null context");
    sync(ctx);
    MSBG_API_END
}

int msbg_ctx_stream(msbg_ctx* ctx, void** s) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && s, "null argument");
    *s = (void*)ctx->stream;
    MSBG_API_END
}

int msbg_ctx_kernel_launches(msbg_ctx* ctx, uint64_t* out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && out, "null argument");
    *out = ctx->launches;
    MSBG_API_END
}

int msbg_ctx_set_timing(msbg_ctx* ctx, int enable) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx, "null context");
    set_device(ctx);
    resolve_timing(ctx);
    ctx->timing = enable != 0;
    MSBG_API_END
}

int msbg_ctx_timing_report(msbg_ctx* ctx, int reset, char* buf, size_t cap, size_t* len_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && len_out, "null argument");
    set_device(ctx);
    resolve_timing(ctx);
    std::vector<std::pair<std::string, std::pair<uint64_t, double>>> rows(ctx->totals.begin(), ctx->totals.end());
    std::sort(rows.begin(), rows.end());
    std::string text;
    char line[256];
    for (auto& r : rows) {
        snprintf(line, sizeof line, "%s %llu %.6f\n", r.first.c_str(), (unsigned long long)r.second.first, r.second.second);
        text += line;
    }
    *len_out = text.size();
    if (buf && cap) {
        size_t n = std::min(cap - 1, text.size());
        memcpy(buf, text.data(), n);
        buf[n] = 0;
    }
    if (reset) ctx->totals.clear();
    MSBG_API_END
}

int msbg_ctx_scratch_bytes(msbg_ctx* ctx, uint64_t* out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && out, "null argument");
    *out = ctx->scratch.bytes;
    MSBG_API_END
}

int msbg_grid_create(msbg_ctx* ctx, uint64_t sx, uint64_t sy, uint64_t sz, int bsx, int dtype,
                     float empty_value, float full_value, msbg_grid** out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && out, "null argument");
    MSBG_REQUIRE(is_pow2((uint64_t)bsx) && bsx <= 32, "bsx must be a power of two <= 32");
    MSBG_REQUIRE(dtype >= MSBG_F32 && dtype <= MSBG_F16, "bad dtype");
    MSBG_REQUIRE(sx > 0 && sy > 0 && sz > 0 && sx < (1ULL << 31) && sy < (1ULL << 31) && sz < (1ULL << 31),
                 "domain extents must be in [1, 2^31)");
    set_device(ctx);
    auto* g = new msbg_grid;
    g->ctx = ctx;
    g->sx = sx; g->sy = sy; g->sz = sz;
    g->bsx = bsx; g->lg = ilog2i((uint64_t)bsx);
    g->nx = (sx + bsx - 1) >> g->lg; g->ny = (sy + bsx - 1) >> g->lg; g->nz = (sz + bsx - 1) >> g->lg;
    g->nxy = g->nx * g->ny;
    g->n_blocks = g->nxy * g->nz;
    g->dtype = dtype;
    g->esize = dtype_size(dtype);
    g->block_elems = (size_t)bsx * bsx * bsx;
    g->empty_value = empty_value;
    g->full_value = full_value;
    *out = g;
    MSBG_API_END
}

int msbg_grid_destroy(msbg_grid* g) {
    MSBG_API_BEGIN
    if (!g) return MSBG_OK;
    cudaSetDevice(g->ctx->device);
    cudaStreamSynchronize(g->ctx->stream);
    delete g;
    MSBG_API_END
}

int msbg_grid_dims(const msbg_grid* g, uint64_t out[8]) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && out, "null argument");
    out[0] = g->sx; out[1] = g->sy; out[2] = g->sz;
    out[3] = g->nx; out[4] = g->ny; out[5] = g->nz;
    out[6] = g->n_blocks; out[7] = g->n_slots();
    MSBG_API_END
}

int msbg_grid_ensure_blocks(msbg_grid* g, const uint64_t* bids, size_t n) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && (bids || !n), "null argument");
    set_device(g->ctx);
    grid_ensure(g, bids, n, nullptr);
    MSBG_API_END
}

int msbg_grid_ensure_blocks_device(msbg_grid* g, const uint64_t* d_bids, size_t n, int32_t* d_slots_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && (d_bids || !n), "null argument");
    set_device(g->ctx);
    grid_ensure_device(g, d_bids, n, d_slots_out);
    MSBG_API_END
}

int msbg_grid_set_full_blocks(msbg_grid* g, const uint64_t* bids, size_t n) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && (bids || !n), "null argument");
    for (size_t k = 0; k < n; ++k) {
        MSBG_REQUIRE(bids[k] < g->n_blocks, "block id out of range");
        MSBG_REQUIRE(grid_code(g, bids[k]) < 0, "set_full_block on a value block");
    }
    for (size_t k = 0; k < n; ++k) g->map[bids[k]] = kCodeFull;
    if (n) { g->hash_dirty = true; g->dense_dirty = true; g->version++; }
    MSBG_API_END
}

int msbg_grid_set_empty_blocks(msbg_grid* g, const uint64_t* bids, size_t n) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && (bids || !n), "null argument");
    for (size_t k = 0; k < n; ++k) {
        MSBG_REQUIRE(bids[k] < g->n_blocks, "block id out of range");
        MSBG_REQUIRE(grid_code(g, bids[k]) < 0, "set_empty_block on a value block");
    }
    for (size_t k = 0; k < n; ++k) g->map.erase(bids[k]);
    if (n) { g->hash_dirty = true; g->dense_dirty = true; g->version++; }
    MSBG_API_END
}

int msbg_grid_set_values(msbg_grid* g, float empty_value, float full_value) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g, "null grid");
    g->empty_value = empty_value;
    g->full_value = full_value;
    g->version++;
    MSBG_API_END
}

int msbg_grid_write_blocks(msbg_grid* g, const uint64_t* bids, size_t n, const void* payload) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && ((bids && payload) || !n), "null argument");
    set_device(g->ctx);
    write_blocks(g, bids, n, payload, false);
    MSBG_API_END
}

int msbg_grid_write_blocks_device(msbg_grid* g, const uint64_t* bids, size_t n, const void* d_payload) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && ((bids && d_payload) || !n), "null argument");
    set_device(g->ctx);
    write_blocks(g, bids, n, d_payload, true);
    MSBG_API_END
}

int msbg_grid_read_blocks(msbg_grid* g, const uint64_t* bids, size_t n, void* payload) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && ((bids && payload) || !n), "null argument");
    set_device(g->ctx);
    read_blocks(g, bids, n, payload, false);
    MSBG_API_END
}

int msbg_grid_read_blocks_device(msbg_grid* g, const uint64_t* bids, size_t n, void* d_payload) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && ((bids && d_payload) || !n), "null argument");
    set_device(g->ctx);
    read_blocks(g, bids, n, d_payload, true);
    MSBG_API_END
}

int msbg_grid_fill_blocks(msbg_grid* g, const uint64_t* bids, size_t n, float value) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && (bids || !n), "null argument");
    set_device(g->ctx);
    std::vector<int32_t> slots;
    for (size_t k = 0; k < n; ++k) {
        MSBG_REQUIRE(bids[k] < g->n_blocks, "block id out of range");
        int32_t c = grid_code(g, bids[k]);
        if (c >= 0) slots.push_back(c);
    }
    if (!slots.empty()) {
        ScratchLayout L;
        size_t o = L.add<int32_t>(slots.size());
        char* base = scratch(g->ctx, L);
        int32_t* d = ScratchLayout::at<int32_t>(base, o);
        CUDA_CHECK(cudaMemcpyAsync(d, slots.data(), slots.size() * 4, cudaMemcpyHostToDevice, g->ctx->stream));
        grid_fill_slots(g, d, slots.size(), value);
        sync(g->ctx);
    }
    MSBG_API_END
}

int msbg_grid_value_block_ids(const msbg_grid* g, uint64_t* out, size_t cap, size_t* n_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && n_out, "null argument");
    std::vector<uint64_t> ids(g->slot_bid);
    std::sort(ids.begin(), ids.end());
    for (size_t k = 0; k < ids.size() && k < cap; ++k) out[k] = ids[k];
    *n_out = ids.size();
    MSBG_API_END
}

int msbg_grid_payload(msbg_grid* g, void** d_payload, uint64_t* n_slots) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g, "null grid");
    if (d_payload) *d_payload = g->payload.p;
    if (n_slots) *n_slots = g->n_slots();
    MSBG_API_END
}

int msbg_grid_slots(const msbg_grid* g, const uint64_t* bids, size_t n, int32_t* slots_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && ((bids && slots_out) || !n), "null argument");
    for (size_t k = 0; k < n; ++k) {
        int32_t c = bids[k] < g->n_blocks ? grid_code(g, bids[k]) : kCodeEmpty;
        slots_out[k] = c >= 0 ? c : -1;
    }
    MSBG_API_END
}

int msbg_halo_gather(msbg_grid* g, const uint64_t* bids, size_t n, int halo, int full, int bc, float* out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && ((bids && out) || !n), "null argument");
    for (size_t k = 0; k < n; ++k) MSBG_REQUIRE(bids[k] < g->n_blocks, "block id out of range");
    if (!n) return MSBG_OK;
    set_device(g->ctx);
    size_t hsx = (size_t)g->bsx + 2 * halo;
    size_t out_elems = n * hsx * hsx * hsx;
    ScratchLayout L;
    size_t ob = L.add<uint64_t>(n), oo = L.add<float>(out_elems);
    char* base = scratch(g->ctx, L);
    uint64_t* d_bids = ScratchLayout::at<uint64_t>(base, ob);
    float* d_out = ScratchLayout::at<float>(base, oo);
    CUDA_CHECK(cudaMemcpyAsync(d_bids, bids, n * 8, cudaMemcpyHostToDevice, g->ctx->stream));
    halo_gather(g, d_bids, n, halo, full, bc, d_out);
    CUDA_CHECK(cudaMemcpyAsync(out, d_out, out_elems * 4, cudaMemcpyDeviceToHost, g->ctx->stream));
    sync(g->ctx);
    MSBG_API_END
}

int msbg_halo_gather_device(msbg_grid* g, const uint64_t* d_bids, size_t n, int halo, int full, int bc, float* d_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && ((d_bids && d_out) || !n), "null argument");
    set_device(g->ctx);
    halo_gather(g, d_bids, n, halo, full, bc, d_out);
    MSBG_API_END
}

}  // extern "C"
