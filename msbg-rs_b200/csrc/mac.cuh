// mac.cuh -- the staggered MAC grid (fluid/mac.rs): six f32 channels that
// always share one block set, so one slot addresses the same block in all six.
#pragma once

#include "grid.cuh"

struct msbg_mac {
    msbg_ctx* ctx = nullptr;
    msbg_grid* ch[6] = {nullptr};  // 0..2 velocity[X..Z], 3..5 mass[X..Z]
    std::vector<uint64_t> active;  // active block set of the last P2G
    ~msbg_mac();
};

namespace msbg {
// Ensures `bids` on all six channels (same slot in each); returns the slots.
void mac_ensure(msbg_mac* m, const uint64_t* bids, size_t n, int32_t* slots);
}  // namespace msbg
