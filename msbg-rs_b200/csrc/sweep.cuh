// sweep.cuh -- the cached plan of an 8-colour in-place sweep (solver.rs:141-267).
#pragma once

#include "grid.cuh"

namespace msbg {

// Everything a sweep needs besides the payload: the blocks of the active list
// that are value blocks, grouped by colour (solver.rs:247-267: colour =
// bx&1 | (by&1)<<1 | (bz&1)<<2, Morton order inside a colour), and for each
// of them the 27 neighbour codes (slot, empty, full or coarse slot) and the
// block coordinates.  Rebuilt when the list, the grid's block set or (for a
// multiresolution sweep) the coarse level changes.
struct SweepPlan {
    uint64_t key = 0;
    size_t n = 0;
    int color_off[9] = {0};
    DevBuf nbr;    // int32 [n][27]
    DevBuf bxyz;   // int32 [n][3]
    DevBuf order;  // int32 [n] plan indices grouped by colour
    // Slots whose x-faces the sweep reads (x-neighbours of active blocks, as
    // faces or edges), for the x-face side buffer (see sweep.cu).
    DevBuf xslots;  // int32 [n_xslots]
    size_t n_xslots = 0;
    DevBuf xface;   // f32 [n_slots][2 xd][bsx^2]: the xd outermost x-planes per side, [z][y]
    size_t xface_slots = 0;  // capacity in slots x xd
    // One-launch sweeps (sweep_wave_kernel): colour and block-layer
    // coordinate of every plan index (host), the (sweep, plan index) items in
    // wavefront order for `wave_iters` sweeps, and the per-slot progress
    // words with the claim counter behind them.
    std::vector<uint8_t> h_col;
    std::vector<int32_t> h_bz;
    DevBuf wave_items;  // int2 [n * wave_iters]
    int wave_iters = -1;
    DevBuf wave_prog;   // int32 [slots], then the counter
    size_t wave_slots = 0;
    // Captured launches of earlier f32 calls on this plan, keyed by the
    // arguments and buffers they bake in.
    struct Graph {
        uint64_t key;
        cudaGraphExec_t exec;
        int kernels;
    };
    std::vector<Graph> graphs;
    SweepPlan() = default;
    SweepPlan(const SweepPlan&) = delete;
    SweepPlan& operator=(const SweepPlan&) = delete;
    ~SweepPlan() {
        for (auto& q : graphs) cudaGraphExecDestroy(q.exec);
    }
};

}  // namespace msbg
