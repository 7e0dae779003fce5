// grid.cuh -- the device-resident sparse grid (sparse_grid.rs:61-435) and the
// device block table (blockmap.rs:35-209).
//
// HBM layout of one grid:
//   payload  [cap_slots][bsx^3] elements of the grid dtype: value blocks only,
//            slot order = order of materialisation (the crate's BlockPool).
//   table    open-addressing hash bid -> code (keys u64, vals i32), power-of-2
//            capacity, linear probing, Fibonacci hash of the bid.  code >= 0 is
//            a payload slot, -2 the full dummy; absent bids are empty.
// The empty and full dummies are not stored: kernels substitute their
// constant values.  A host mirror of the table drives materialisation.
#pragma once

#include "common.cuh"

namespace msbg {

constexpr uint64_t kHashEmpty = ~0ULL;
constexpr int32_t kCodeEmpty = -1;
constexpr int32_t kCodeFull = -2;
// Codes <= kCodeCoarse0 name a coarse-level slot: slot = kCodeCoarse0 - code.
constexpr int32_t kCodeCoarse0 = -3;

struct DevHash {
    const uint64_t* keys;
    const int32_t* vals;
    uint32_t mask;
    int shift;  // 64 - log2(capacity)
};

__host__ __device__ inline uint32_t hash_slot(uint64_t key, int shift) {
    return (uint32_t)((key * 0x9e3779b97f4a7c15ULL) >> shift);
}

// Lookup with a probe bound of the table capacity (the table is never full:
// capacity >= 2 * entries).
__device__ inline int32_t hash_find(const DevHash& h, uint64_t key) {
    uint32_t i = hash_slot(key, h.shift);
    for (uint32_t probe = 0; probe <= h.mask; ++probe) {
        uint64_t k = h.keys[i];
        if (k == key) return h.vals[i];
        if (k == kHashEmpty) return kCodeEmpty;
        i = (i + 1) & h.mask;
    }
    return kCodeEmpty;
}

// Host-built open-addressing table, uploaded as a whole.
struct HostHash {
    std::vector<uint64_t> keys;
    std::vector<int32_t> vals;
    uint32_t mask = 0;
    int shift = 64;
    void build(const std::unordered_map<uint64_t, int32_t>& m);
};

struct SweepPlan;

}  // namespace msbg

struct msbg_grid {
    msbg_ctx* ctx = nullptr;
    uint64_t sx = 0, sy = 0, sz = 0, nx = 0, ny = 0, nz = 0, nxy = 0, n_blocks = 0;
    int bsx = 0, lg = 0, dtype = MSBG_F32;
    size_t esize = 4, block_elems = 0;
    float empty_value = 0.0f, full_value = 0.0f;

    // host mirror of the block table
    std::unordered_map<uint64_t, int32_t> map;  // bid -> slot or kCodeFull
    std::vector<uint64_t> slot_bid;             // slot -> bid
    uint64_t version = 0;                       // bumps when the block set changes

    // device state
    msbg::DevBuf payload;
    size_t cap_slots = 0;
    msbg::DevBuf hkeys, hvals;
    uint32_t hmask = 0;
    int hshift = 64;
    bool hash_dirty = true;
    msbg::DevBuf dense;  // int32 code per block id, for grids of <= kDenseMaxBlocks blocks
    bool dense_dirty = true;

    msbg::SweepPlan* plan = nullptr;  // cached sweep plan

    ~msbg_grid();
    size_t n_slots() const { return slot_bid.size(); }
    void* slot_ptr(size_t s) const { return (char*)payload.p + s * block_elems * esize; }
};

namespace msbg {

// Makes sure the device table mirrors the host map.
DevHash device_hash(msbg_grid* g);
// A dense bid -> code table (null when the grid has more than kDenseMaxBlocks
// blocks): one load instead of a hash probe for small and medium domains.
constexpr uint64_t kDenseMaxBlocks = 1ull << 24;
const int32_t* device_dense(msbg_grid* g);
// Materialises value blocks for `bids` (new ones filled with the empty value);
// returns the slot of each bid in `slots` (may be null).
void grid_ensure(msbg_grid* g, const uint64_t* bids, size_t n, int32_t* slots);
// Grows the payload arena to hold `need` slots, preserving contents.
void grid_reserve(msbg_grid* g, size_t need);
// Fills slots [first, first + count) with a float constant (quantised).
void grid_fill_slots(msbg_grid* g, const int32_t* d_slots, size_t count, float value);
int32_t grid_code(const msbg_grid* g, uint64_t bid);
void block_coords(const msbg_grid* g, uint64_t bid, int64_t* bx, int64_t* by, int64_t* bz);

}  // namespace msbg
