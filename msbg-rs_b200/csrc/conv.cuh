// conv.cuh -- block-sparse 3x3x3 convolutions on the sparse block grid,
// implicit GEMM on the tcgen05 tensor cores.
//
// A feature map of one resolution level lives in HBM as bf16 [cells][C]
// (channels contiguous) with the level's cells in block order: block k holds
// cells k * bs^3 ... (k + 1) * bs^3 - 1 in the payload order x | y<<lg |
// z<<2lg.  Cells of blocks outside the active set read as zero (zero
// padding at the sparse boundary).  A per-level table nbr27[k][27] gives the
// slot of each of the 26 neighbour blocks (-1 when absent; entry 13 is k).
//
// Convolution:  y[c][o] = b[o] + sum_t sum_i w[t][o][i] x[c + d(t)][i],
//   t = (dx+1) + 3 (dy+1) + 9 (dz+1), weights bf16 [27][Cout][Cin].
// Forward and the data gradient (the same convolution with the taps
// mirrored and Cin/Cout swapped) run on 8^3 blocks with Cin, Cout <= 32 as
// conv3_b8_kernel: persistent CTAs copy each block's 10^3 input halo into
// shared memory once (double-buffered) and the weights of all taps once;
// every tap's operand for one z-plane of the block is a strided view of the
// halo, so the MMAs (M = 64 cells of a plane) need no per-tap staging, and
// eight warps issue the eight planes' MMAs side by side.  Other shapes run as
// conv3_fwd_kernel: one CTA computes a tile of 128 output cells x Cout in
// TMEM; per tap its threads gather the shifted input rows (cp.async,
// several taps in flight) into a K-major operand and the weights into a
// K-major operand in shared memory, one thread issues Cin/16 MMAs and
// commits them to the stage's mbarrier.  The weight gradient
//   dw[t][o][i] = sum_c x[c + d(t)][i] dy[c][o]
// runs as conv3_wgrad_kernel: M = the (tap, Cin) pairs in tiles of 128,
// N = Cout, K = cells, operands MN-major (16-byte rows of 8 channels of one
// cell), partial sums per cell range reduced in a fixed order.
#pragma once

#include "common.cuh"

namespace msbg {

struct ConvLevel {
    const int32_t* nbr27;  // [n_blocks][27]
    int lg;                // log2 block size
    int64_t n_blocks;
    __host__ __device__ int64_t cells() const { return n_blocks << (3 * lg); }
};

// y = conv(x) (+ bias) (ReLU): x bf16 [cells][cin], w bf16 [27][cout][cin],
// y bf16 or f32 [cells][cout].  cin, cout in {16, 32, 64}.  mask (bf16
// [cells][cout], optional) zeroes outputs where it is not positive (the ReLU
// derivative of the data gradient).  out_ch (f32 output only, 0 = cout)
// writes the first out_ch channels as rows of out_ch.
void conv3_forward(msbg_ctx* ctx, const ConvLevel& L, int cin, int cout, const uint16_t* x, const uint16_t* w,
                   const float* bias, bool relu, bool out_f32, void* y, const uint16_t* mask = nullptr, int out_ch = 0);

// dw = sum over cells of x[c + d(t)] dy[c]^T as f32 [27][cout][cin]; `acc`
// adds to dw instead of overwriting.
void conv3_wgrad(msbg_ctx* ctx, const ConvLevel& L, int cin, int cout, const uint16_t* x, const uint16_t* dy, float* dw,
                 bool acc);

}  // namespace msbg
