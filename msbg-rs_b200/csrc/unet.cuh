// unet.cuh -- the learned preconditioner of the pressure solve: a
// block-sparse 3D U-Net over the solve's level-0 blocks.
//
// Three resolution levels on the same block set: level 0 has 16^3 cells per
// block, level 1 8^3, level 2 4^3 (the V-cycle's first three levels).  All
// convolutions are 3x3x3 with zero padding outside the active blocks, bf16
// weights and activations, f32 accumulation on the tensor cores (conv.cuh).
//
//   a0 = relu(conv0a(x))            level 0, 1 -> 16   (input padded to 16)
//   a1 = relu(conv1a(pool(a0)))     level 1, 16 -> 32
//   a2 = relu(conv2a(pool(a1)))     level 2, 32 -> 64
//   a3 = relu(conv2b(a2))           level 2, 64 -> 64
//   u1 = relu(up(conv2c(a3)) + a1)  level 2 -> 1, 64 -> 32
//   a4 = relu(conv1c(u1))           level 1, 32 -> 32
//   u0 = relu(up(conv1d(a4)) + a0)  level 1 -> 0, 32 -> 16
//   y  = conv0c(u0)                 level 0, 16 -> 1   (output padded to 16)
//
// pool = mean of the 8 children, up = copy to the 8 children.  Applied as a
// preconditioner: z = s_out * y(x = r / s_in), s_in = rms(r), s_out = s_in *
// out_scale.
#pragma once

#include "common.cuh"

struct msbg_unet;

namespace msbg {

// z = rms(r) * out_scale * N(r / rms(r)) on the level-0 cells (f32 vectors in
// block order); z = 0 when r = 0.
void unet_apply(msbg_unet* net, const float* r, float* z);

// One training pass on the pair (r, e): forward on r / rms(r), loss
// sum((out_scale * y - e / rms(r))^2) / sum((e / rms(r))^2), backward into the
// gradient buffer; with `update` an Adam step follows.  Returns the loss.
double unet_train_step(msbg_unet* net, const float* r, const float* e, float lr, bool update);

int64_t unet_blocks(const msbg_unet* net);
msbg_ctx* unet_ctx(const msbg_unet* net);

}  // namespace msbg
