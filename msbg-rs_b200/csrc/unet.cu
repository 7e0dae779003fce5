// unet.cu -- the learned preconditioner's network: parameters, forward and
// backward passes over the tcgen05 convolutions, Adam, and the C ABI.
#include <algorithm>
#include <cmath>
#include <random>
#include <unordered_map>

#include "conv.cuh"
#include "unet.cuh"

namespace msbg {

// One convolution layer.  Channel counts are the padded ones the kernels run
// (multiples of 16); cin_real / cout_real are the network's.
struct ULayer {
    int level, cin, cout, cin_real, cout_real;
    bool relu;
    size_t w_off, b_off;  // f32 parameter offsets: w [27][cout][cin], b [cout]
    size_t wb_off;        // bf16 offsets (same for the forward and the mirrored copy)
};

enum { L0A, L1A, L2A, L2B, L2C, L1C, L1D, L0C, N_LAYERS };

}  // namespace msbg

struct msbg_unet {
    msbg_ctx* ctx = nullptr;
    int64_t nb = 0;
    int64_t n[3] = {0, 0, 0};  // cells per level
    msbg::DevBuf nbr;          // int32 [nb][27], shared by the three levels
    std::vector<msbg::ULayer> layers;
    size_t n_params = 0, n_wb = 0;
    msbg::DevBuf params, grads, adam_m, adam_v, pmask;  // f32 [n_params]; pmask 1 = trainable
    msbg::DevBuf wb, wt;                                 // bf16 forward / mirrored-transposed weights
    msbg::DevBuf act;                                    // activations and gradients
    msbg::DevBuf red;                                    // reduction partials
    float out_scale = 1.0f;
    int64_t adam_t = 0;
    bool weights_dirty = true;
    // activation pointers (into act)
    uint16_t *x0, *a0, *p1, *a1, *p2, *a2, *a3, *c2, *u1, *a4, *c1, *u0;
    uint16_t* x0c;  // compact 1-channel input (bf16 [n0]) read by the direct first layer
    float* y;
    uint16_t *dyb, *du0m, *dc1, *da4m, *du1m, *dc2, *da3m, *da2m, *da1m, *da0m;
    float *dp2, *dp1;
};

namespace msbg {

static unsigned grid1(int64_t n, int threads = 256) {
    return (unsigned)std::min<int64_t>(std::max<int64_t>((n + threads - 1) / threads, 1), 148 * 32);
}

__device__ __forceinline__ float bf(uint16_t h) { return __uint_as_float((uint32_t)h << 16); }
__device__ __forceinline__ uint16_t tobf(float v) { return ElemBF16::store(v); }

__device__ __forceinline__ void unpack8(uint4 q, float* f) {
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        f[2 * i] = __uint_as_float(w[i] << 16);
        f[2 * i + 1] = __uint_as_float(w[i] & 0xFFFF0000u);
    }
}
__device__ __forceinline__ uint4 pack8(const float* f) {
    uint32_t w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) w[i] = (uint32_t)tobf(f[2 * i]) | ((uint32_t)tobf(f[2 * i + 1]) << 16);
    return make_uint4(w[0], w[1], w[2], w[3]);
}

// x0c[c] = bf16(r[c] * s); with x0 also the same value padded to 16
// channels (the weight gradient of the first layer reads that form).
__global__ void un_input_kernel(int64_t n, const float* __restrict__ r, const double* __restrict__ s_in,
                                uint16_t* __restrict__ x0c, uint16_t* __restrict__ x0) {
    const float s = (float)(1.0 / *s_in);
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const uint16_t h = tobf(r[c] * s);
        x0c[c] = h;
        if (x0) {
            uint4* o = reinterpret_cast<uint4*>(x0 + c * 16);
            o[0] = make_uint4((uint32_t)h, 0u, 0u, 0u);
            o[1] = make_uint4(0u, 0u, 0u, 0u);
        }
    }
}

// Level-0 halo staging: CTA (block k, octant o) covers the 8^3 cells of
// octant o of block k; halo cell h in [0, 10^3) sits at in-block coordinate
// octant origin - 1 + (h % 10, h / 10 % 10, h / 100), in the neighbouring
// block across a face (nbr27) where it leaves the block; -1 where that block
// is not in the set.
__device__ __forceinline__ int64_t l0_halo_cell(const int32_t* __restrict__ nbr27, int64_t nb, int64_t k, int o, int h) {
    const int gx = (o & 1) * 8 - 1 + h % 10, gy = ((o >> 1) & 1) * 8 - 1 + (h / 10) % 10, gz = (o >> 2) * 8 - 1 + h / 100;
    const int ox = gx < 0 ? 0 : (gx > 15 ? 2 : 1), oy = gy < 0 ? 0 : (gy > 15 ? 2 : 1), oz = gz < 0 ? 0 : (gz > 15 ? 2 : 1);
    const int code = ox + 3 * oy + 9 * oz;
    const int32_t kk = code == 13 ? (int32_t)k : nbr27[k * 27 + code];
    if (kk < 0 || kk >= nb) return -1;
    return ((int64_t)kk << 12) + ((gx & 15) | ((gy & 15) << 4) | ((gz & 15) << 8));
}

// First layer on the CUDA cores: a0[c][o] = relu(b[o] + sum_t w[t][o][0] x[c + d(t)]),
// 1 -> 16 channels (weights bf16 [27][16][16], input channel 0 only).  One CTA
// per (block, octant): the octant's 10^3 input halo in shared memory; each
// thread computes cells (x, y, z) and (x, y, z + 4) of the octant, taps in
// order t = 0..26 (fmaf), the tap loop unrolled so every halo offset is a
// constant and each tap's 16 weights are read once for both cells.
__global__ void __launch_bounds__(256) un_conv_in1_kernel(const int32_t* __restrict__ nbr27, int64_t nb,
                                                          const uint16_t* __restrict__ x0c, const uint16_t* __restrict__ w,
                                                          const float* __restrict__ bias, uint16_t* __restrict__ a0) {
    __shared__ float4 ws[27][4];
    __shared__ float bs[16];
    __shared__ float xs[1000];
    const int64_t k = blockIdx.x >> 3;
    const int o = blockIdx.x & 7;
    for (int e = threadIdx.x; e < 27 * 16; e += blockDim.x)
        reinterpret_cast<float*>(ws)[e] = bf(w[(e / 16) * 256 + (e % 16) * 16]);
    if (threadIdx.x < 16) bs[threadIdx.x] = bias[threadIdx.x];
    for (int h = threadIdx.x; h < 1000; h += blockDim.x) {
        const int64_t src = l0_halo_cell(nbr27, nb, k, o, h);
        xs[h] = src >= 0 ? bf(__ldg(x0c + src)) : 0.0f;
    }
    __syncthreads();
    const int c = threadIdx.x;  // cells c and c + 256 of the octant
    const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
    const float* xp = xs + (z * 10 + y) * 10 + x;
    float acc0[16], acc1[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) acc0[q] = acc1[q] = 0.0f;
#pragma unroll
    for (int t = 0; t < 27; ++t) {
        const int off = ((t / 9) * 10 + (t / 3) % 3) * 10 + t % 3;
        const float x0 = xp[off], x1 = xp[off + 400];
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) {
            const float4 wv = ws[t][qq];
            acc0[4 * qq] = fmaf(wv.x, x0, acc0[4 * qq]);
            acc0[4 * qq + 1] = fmaf(wv.y, x0, acc0[4 * qq + 1]);
            acc0[4 * qq + 2] = fmaf(wv.z, x0, acc0[4 * qq + 2]);
            acc0[4 * qq + 3] = fmaf(wv.w, x0, acc0[4 * qq + 3]);
            acc1[4 * qq] = fmaf(wv.x, x1, acc1[4 * qq]);
            acc1[4 * qq + 1] = fmaf(wv.y, x1, acc1[4 * qq + 1]);
            acc1[4 * qq + 2] = fmaf(wv.z, x1, acc1[4 * qq + 2]);
            acc1[4 * qq + 3] = fmaf(wv.w, x1, acc1[4 * qq + 3]);
        }
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        acc0[q] = fmaxf(acc0[q] + bs[q], 0.0f);
        acc1[q] = fmaxf(acc1[q] + bs[q], 0.0f);
    }
    const int64_t gx = (o & 1) * 8 + x, gy = ((o >> 1) & 1) * 8 + y, gz = (o >> 2) * 8 + z;
    const int64_t cell0 = (k << 12) + (gx | (gy << 4) | (gz << 8)), cell1 = cell0 + (4 << 8);
    uint4* out0 = reinterpret_cast<uint4*>(a0 + cell0 * 16);
    out0[0] = pack8(acc0);
    out0[1] = pack8(acc0 + 8);
    uint4* out1 = reinterpret_cast<uint4*>(a0 + cell1 * 16);
    out1[0] = pack8(acc1);
    out1[1] = pack8(acc1 + 8);
}

// Last layer on the CUDA cores: y[c] = b[0] + sum_t sum_i w[t][0][i] u[c + d(t)][i],
// 16 -> 1 channel, f32 output.  One CTA per (block, octant): the octant's
// 10^3 halo of 16-channel rows in shared memory as two planes of 8 channels
// (16-byte rows, conflict-free); each thread computes cells (x, y, z) and
// (x, y, z + 4), taps in order and channels in order within a tap (fmaf),
// the tap loop unrolled so every halo offset is a constant.
__global__ void __launch_bounds__(256) un_conv_out1_kernel(const int32_t* __restrict__ nbr27, int64_t nb,
                                                           const uint16_t* __restrict__ u0, const uint16_t* __restrict__ w,
                                                           const float* __restrict__ bias, float* __restrict__ y) {
    __shared__ float4 ws[27][4];
    __shared__ uint4 us[2][1000];
    const int64_t k = blockIdx.x >> 3;
    const int o = blockIdx.x & 7;
    for (int e = threadIdx.x; e < 27 * 16; e += blockDim.x)
        reinterpret_cast<float*>(ws)[e] = bf(w[(e / 16) * 256 + (e % 16)]);
    for (int e = threadIdx.x; e < 2000; e += blockDim.x) {
        const int h = e >> 1, half = e & 1;
        const int64_t src = l0_halo_cell(nbr27, nb, k, o, h);
        us[half][h] = src >= 0 ? __ldg(reinterpret_cast<const uint4*>(u0 + src * 16) + half) : make_uint4(0u, 0u, 0u, 0u);
    }
    __syncthreads();
    const float b0 = bias[0];
    const int c = threadIdx.x;  // cells c and c + 256 of the octant
    const int x = c & 7, yy = (c >> 3) & 7, z = c >> 6;
    const int h0 = (z * 10 + yy) * 10 + x;
    float acc0 = 0.0f, acc1 = 0.0f;
#pragma unroll
    for (int t = 0; t < 27; ++t) {
        const int h = h0 + ((t / 9) * 10 + (t / 3) % 3) * 10 + t % 3;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            float v0[8], v1[8];
            unpack8(us[half][h], v0);
            unpack8(us[half][h + 400], v1);
            const float4 wa = ws[t][2 * half], wb = ws[t][2 * half + 1];
            const float wv[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                acc0 = fmaf(wv[i], v0[i], acc0);
                acc1 = fmaf(wv[i], v1[i], acc1);
            }
        }
    }
    const int64_t gx = (o & 1) * 8 + x, gy = ((o >> 1) & 1) * 8 + yy, gz = (o >> 2) * 8 + z;
    const int64_t cell0 = (k << 12) + (gx | (gy << 4) | (gz << 8));
    y[cell0] = acc0 + b0;
    y[cell0 + (4 << 8)] = acc1 + b0;
}

// Coarse cell i of level lgc (same block, cells twice the size) from its 8
// children at level lgc+1: p = scale * sum(children), per 8-channel chunk.
__global__ void un_pool_kernel(int64_t nc, int lgc, int C, const uint16_t* __restrict__ a, float scale,
                               uint16_t* __restrict__ p) {
    const int chunks = C / 8, lgf = lgc + 1, mc = (1 << lgc) - 1;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nc * chunks; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / chunks;
        const int j = (int)(e % chunks);
        const int64_t k = i >> (3 * lgc);
        const int v = (int)(i & ((1 << (3 * lgc)) - 1));
        const int cx = v & mc, cy = (v >> lgc) & mc, cz = v >> (2 * lgc);
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            const int fx = 2 * cx + (d & 1), fy = 2 * cy + ((d >> 1) & 1), fz = 2 * cz + (d >> 2);
            const int64_t f = (k << (3 * lgf)) + (fx | (fy << lgf) | (fz << (2 * lgf)));
            float t[8];
            unpack8(__ldg(reinterpret_cast<const uint4*>(a + f * C) + j), t);
#pragma unroll
            for (int q = 0; q < 8; ++q) s[q] += t[q];
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) s[q] *= scale;
        reinterpret_cast<uint4*>(p + i * C)[j] = pack8(s);
    }
}

// u = relu(c[parent] + skip) at level lgf (c at level lgf-1).
__global__ void un_up_add_relu_kernel(int64_t nf, int lgf, int C, const uint16_t* __restrict__ c,
                                      const uint16_t* __restrict__ skip, uint16_t* __restrict__ u) {
    const int chunks = C / 8, lgc = lgf - 1, mf = (1 << lgf) - 1;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nf * chunks; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / chunks;
        const int j = (int)(e % chunks);
        const int64_t k = i >> (3 * lgf);
        const int v = (int)(i & ((1 << (3 * lgf)) - 1));
        const int fx = v & mf, fy = (v >> lgf) & mf, fz = v >> (2 * lgf);
        const int64_t pc = (k << (3 * lgc)) + ((fx >> 1) | ((fy >> 1) << lgc) | ((fz >> 1) << (2 * lgc)));
        float a[8], b[8];
        unpack8(__ldg(reinterpret_cast<const uint4*>(c + pc * C) + j), a);
        unpack8(__ldg(reinterpret_cast<const uint4*>(skip + i * C) + j), b);
#pragma unroll
        for (int q = 0; q < 8; ++q) a[q] = fmaxf(a[q] + b[q], 0.0f);
        reinterpret_cast<uint4*>(u + i * C)[j] = pack8(a);
    }
}

// Gradient reaching a skip-connected activation a = relu(...) at level lgf:
// out = (g_skip + 0.125 * g_pool[parent]) * (a > 0).
__global__ void un_skip_pool_mask_kernel(int64_t nf, int lgf, int C, const uint16_t* __restrict__ gskip,
                                         const float* __restrict__ gpool, const uint16_t* __restrict__ a,
                                         uint16_t* __restrict__ out) {
    const int chunks = C / 8, lgc = lgf - 1, mf = (1 << lgf) - 1;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nf * chunks; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / chunks;
        const int j = (int)(e % chunks);
        const int64_t k = i >> (3 * lgf);
        const int v = (int)(i & ((1 << (3 * lgf)) - 1));
        const int fx = v & mf, fy = (v >> lgf) & mf, fz = v >> (2 * lgf);
        const int64_t pc = (k << (3 * lgc)) + ((fx >> 1) | ((fy >> 1) << lgc) | ((fz >> 1) << (2 * lgc)));
        float g[8], av[8];
        unpack8(__ldg(reinterpret_cast<const uint4*>(gskip + i * C) + j), g);
        unpack8(__ldg(reinterpret_cast<const uint4*>(a + i * C) + j), av);
        const float* gp = gpool + pc * C + j * 8;
#pragma unroll
        for (int q = 0; q < 8; ++q) g[q] = av[q] > 0.0f ? g[q] + 0.125f * gp[q] : 0.0f;
        reinterpret_cast<uint4*>(out + i * C)[j] = pack8(g);
    }
}

// Fixed-order FP64 reductions: stage 1 per CTA, stage 2 in one CTA.
constexpr int RED_T = 256, RED_B = 592;

__device__ __forceinline__ double block_sum(double v, double* sm) {
    sm[threadIdx.x] = v;
    __syncthreads();
    for (int o = RED_T / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
        __syncthreads();
    }
    const double r = sm[0];
    __syncthreads();
    return r;
}

// part[b] = sum r^2 over the CTA's cells
__global__ void __launch_bounds__(RED_T) un_sumsq_kernel(int64_t n, const float* __restrict__ r, double* __restrict__ part) {
    __shared__ double sm[RED_T];
    double s = 0.0;
    for (int64_t c = blockIdx.x * (int64_t)RED_T + threadIdx.x; c < n; c += (int64_t)gridDim.x * RED_T) s += (double)r[c] * r[c];
    s = block_sum(s, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// out[j] = sum of part[b][j] over b (j < width), fixed order; out[width] =
// sqrt(out[0] / count) when rms != 0.
__global__ void __launch_bounds__(RED_T) un_final_kernel(const double* __restrict__ part, int nb, int width, double count,
                                                         int rms, double* __restrict__ out) {
    __shared__ double sm[RED_T];
    for (int j = 0; j < width; ++j) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nb; b += RED_T) s += part[(int64_t)b * width + j];
        s = block_sum(s, sm);
        if (threadIdx.x == 0) out[j] = s;
    }
    if (rms && threadIdx.x == 0) out[width] = out[0] > 0.0 ? sqrt(out[0] / count) : 1.0;
}

// part[b] = (sum ehat^2, sum (S y - ehat)^2), ehat = e / s_in
__global__ void __launch_bounds__(RED_T) un_loss_kernel(int64_t n, const float* __restrict__ y, const float* __restrict__ e,
                                                        const double* __restrict__ s_in, float S, double* __restrict__ part) {
    __shared__ double sm[RED_T];
    const double inv = 1.0 / *s_in;
    double a = 0.0, b = 0.0;
    for (int64_t c = blockIdx.x * (int64_t)RED_T + threadIdx.x; c < n; c += (int64_t)gridDim.x * RED_T) {
        const double eh = (double)e[c] * inv;
        const double d = (double)S * y[c] - eh;
        a += eh * eh;
        b += d * d;
    }
    a = block_sum(a, sm);
    b = block_sum(b, sm);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
    }
}

// dy (bf16, padded to 16 channels) = 2 S (S y - ehat) / sum ehat^2
__global__ void un_dy_kernel(int64_t n, const float* __restrict__ y, const float* __restrict__ e,
                             const double* __restrict__ s_in, const double* __restrict__ sums, float S,
                             uint16_t* __restrict__ dyb) {
    const double inv = 1.0 / *s_in;
    const double coef = sums[0] > 0.0 ? 2.0 * S / sums[0] : 0.0;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const float g = (float)(coef * ((double)S * y[c] - (double)e[c] * inv));
        uint4* o = reinterpret_cast<uint4*>(dyb + c * 16);
        o[0] = make_uint4((uint32_t)tobf(g), 0u, 0u, 0u);
        o[1] = make_uint4(0u, 0u, 0u, 0u);
    }
}

// Bias gradient: part[b][j] = sum over the CTA's cells of g[c][j] (C <= 64).
__global__ void __launch_bounds__(RED_T) un_colsum_kernel(int64_t n, int C, const uint16_t* __restrict__ g,
                                                          double* __restrict__ part) {
    __shared__ double sm[RED_T];
    for (int j = 0; j < C; ++j) {
        double s = 0.0;
        for (int64_t c = blockIdx.x * (int64_t)RED_T + threadIdx.x; c < n; c += (int64_t)gridDim.x * RED_T)
            s += (double)bf(g[c * C + j]);
        s = block_sum(s, sm);
        if (threadIdx.x == 0) part[(int64_t)blockIdx.x * C + j] = s;
    }
}

__global__ void un_store_bias_grad_kernel(int C, const double* __restrict__ sums, float* __restrict__ gb) {
    for (int j = threadIdx.x; j < C; j += blockDim.x) gb[j] = (float)sums[j];
}

// f32 weights [27][cout][cin] -> bf16 forward copy and bf16 mirrored,
// transposed copy wt[t][i][o] = w[26 - t][o][i] (the data gradient's weights).
__global__ void un_cast_weights_kernel(int cin, int cout, const float* __restrict__ w, uint16_t* __restrict__ wb,
                                       uint16_t* __restrict__ wt) {
    const int n = 27 * cin * cout;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int i = e % cin, o = (e / cin) % cout, t = e / (cin * cout);
        const uint16_t h = tobf(w[e]);
        wb[e] = h;
        wt[((26 - t) * cin + i) * cout + o] = h;
    }
}

__global__ void un_adam_kernel(int64_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                               float* __restrict__ v, const float* __restrict__ mask, float lr, float b1, float b2,
                               float eps, float bc1, float bc2) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i] * mask[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= mask[i] * lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    }
}

// ---- host ---------------------------------------------------------------------
static ConvLevel level(const msbg_unet* U, int l) { return ConvLevel{U->nbr.as<int32_t>(), 4 - l, U->nb}; }

static void cast_weights(msbg_unet* U) {
    for (const ULayer& L : U->layers) {
        begin_launch(U->ctx);
        un_cast_weights_kernel<<<grid1(27 * L.cin * L.cout), 256, 0, U->ctx->stream>>>(
            L.cin, L.cout, U->params.as<float>() + L.w_off, U->wb.as<uint16_t>() + L.wb_off, U->wt.as<uint16_t>() + L.wb_off);
        after_launch(U->ctx, "un_cast_weights_kernel");
    }
    U->weights_dirty = false;
}

static double* red_part(msbg_unet* U) { return U->red.as<double>(); }
static double* red_out(msbg_unet* U) { return U->red.as<double>() + (size_t)RED_B * 64; }

// s_in = rms(r) into red_out[1] (device), returns nothing (stays on device)
static const double* rms_device(msbg_unet* U, const float* r) {
    msbg_ctx* ctx = U->ctx;
    double* part = red_part(U);
    double* out = red_out(U) + 8;
    begin_launch(ctx);
    un_sumsq_kernel<<<RED_B, RED_T, 0, ctx->stream>>>(U->n[0], r, part);
    after_launch(ctx, "un_sumsq_kernel");
    begin_launch(ctx);
    un_final_kernel<<<1, RED_T, 0, ctx->stream>>>(part, RED_B, 1, (double)U->n[0], 1, out);
    after_launch(ctx, "un_final_kernel");
    return out + 1;
}

static void conv_fwd(msbg_unet* U, int li, const uint16_t* x, void* y, bool out_f32 = false, int out_ch = 0) {
    const ULayer& L = U->layers[li];
    conv3_forward(U->ctx, level(U, L.level), L.cin, L.cout, x, U->wb.as<uint16_t>() + L.wb_off,
                  U->params.as<float>() + L.b_off, L.relu, out_f32, y, nullptr, out_ch);
}

// data gradient of layer li: dx = convT(dy) (masked by `mask` when given)
static void conv_dgrad(msbg_unet* U, int li, const uint16_t* dy, void* dx, const uint16_t* mask, bool out_f32) {
    const ULayer& L = U->layers[li];
    conv3_forward(U->ctx, level(U, L.level), L.cout, L.cin, dy, U->wt.as<uint16_t>() + L.wb_off, nullptr, false, out_f32,
                  dx, mask, 0);
}

static void conv_wgrad(msbg_unet* U, int li, const uint16_t* x, const uint16_t* dy) {
    const ULayer& L = U->layers[li];
    conv3_wgrad(U->ctx, level(U, L.level), L.cin, L.cout, x, dy, U->grads.as<float>() + L.w_off, false);
    msbg_ctx* ctx = U->ctx;
    const int64_t n = U->n[L.level];
    begin_launch(ctx);
    un_colsum_kernel<<<RED_B, RED_T, 0, ctx->stream>>>(n, L.cout, dy, red_part(U));
    after_launch(ctx, "un_colsum_kernel");
    begin_launch(ctx);
    un_final_kernel<<<1, RED_T, 0, ctx->stream>>>(red_part(U), RED_B, L.cout, 0.0, 0, red_out(U) + 16);
    after_launch(ctx, "un_final_kernel");
    begin_launch(ctx);
    un_store_bias_grad_kernel<<<1, 64, 0, ctx->stream>>>(L.cout, red_out(U) + 16, U->grads.as<float>() + L.b_off);
    after_launch(ctx, "un_store_bias_grad_kernel");
}

static void pool(msbg_unet* U, int lc, int C, const uint16_t* a, float scale, uint16_t* p) {
    const int64_t nc = U->n[lc];
    begin_launch(U->ctx);
    un_pool_kernel<<<grid1(nc * (C / 8)), 256, 0, U->ctx->stream>>>(nc, 4 - lc, C, a, scale, p);
    after_launch(U->ctx, "un_pool_kernel");
}

static void up_add_relu(msbg_unet* U, int lf, int C, const uint16_t* c, const uint16_t* skip, uint16_t* u) {
    const int64_t nf = U->n[lf];
    begin_launch(U->ctx);
    un_up_add_relu_kernel<<<grid1(nf * (C / 8)), 256, 0, U->ctx->stream>>>(nf, 4 - lf, C, c, skip, u);
    after_launch(U->ctx, "un_up_add_relu_kernel");
}

static void skip_pool_mask(msbg_unet* U, int lf, int C, const uint16_t* gskip, const float* gpool, const uint16_t* a,
                           uint16_t* out) {
    const int64_t nf = U->n[lf];
    begin_launch(U->ctx);
    un_skip_pool_mask_kernel<<<grid1(nf * (C / 8)), 256, 0, U->ctx->stream>>>(nf, 4 - lf, C, gskip, gpool, a, out);
    after_launch(U->ctx, "un_skip_pool_mask_kernel");
}

// Forward from the padded input x0; y (f32 [n0]) = network output.
static void forward(msbg_unet* U) {
    if (U->weights_dirty) cast_weights(U);
    {
        const ULayer& L = U->layers[L0A];
        begin_launch(U->ctx);
        un_conv_in1_kernel<<<(unsigned)(U->nb * 8), 256, 0, U->ctx->stream>>>(
            U->nbr.as<int32_t>(), U->nb, U->x0c, U->wb.as<uint16_t>() + L.wb_off, U->params.as<float>() + L.b_off, U->a0);
        after_launch(U->ctx, "un_conv_in1_kernel");
    }
    pool(U, 1, 16, U->a0, 0.125f, U->p1);
    conv_fwd(U, L1A, U->p1, U->a1);
    pool(U, 2, 32, U->a1, 0.125f, U->p2);
    conv_fwd(U, L2A, U->p2, U->a2);
    conv_fwd(U, L2B, U->a2, U->a3);
    conv_fwd(U, L2C, U->a3, U->c2);
    up_add_relu(U, 1, 32, U->c2, U->a1, U->u1);
    conv_fwd(U, L1C, U->u1, U->a4);
    conv_fwd(U, L1D, U->a4, U->c1);
    up_add_relu(U, 0, 16, U->c1, U->a0, U->u0);
    {
        const ULayer& L = U->layers[L0C];
        begin_launch(U->ctx);
        un_conv_out1_kernel<<<(unsigned)(U->nb * 8), 256, 0, U->ctx->stream>>>(
            U->nbr.as<int32_t>(), U->nb, U->u0, U->wb.as<uint16_t>() + L.wb_off, U->params.as<float>() + L.b_off, U->y);
        after_launch(U->ctx, "un_conv_out1_kernel");
    }
}

// Backward from dyb; fills every parameter gradient.
static void backward(msbg_unet* U) {
    conv_wgrad(U, L0C, U->u0, U->dyb);
    conv_dgrad(U, L0C, U->dyb, U->du0m, U->u0, false);
    pool(U, 1, 16, U->du0m, 1.0f, U->dc1);
    conv_wgrad(U, L1D, U->a4, U->dc1);
    conv_dgrad(U, L1D, U->dc1, U->da4m, U->a4, false);
    conv_wgrad(U, L1C, U->u1, U->da4m);
    conv_dgrad(U, L1C, U->da4m, U->du1m, U->u1, false);
    pool(U, 2, 32, U->du1m, 1.0f, U->dc2);
    conv_wgrad(U, L2C, U->a3, U->dc2);
    conv_dgrad(U, L2C, U->dc2, U->da3m, U->a3, false);
    conv_wgrad(U, L2B, U->a2, U->da3m);
    conv_dgrad(U, L2B, U->da3m, U->da2m, U->a2, false);
    conv_wgrad(U, L2A, U->p2, U->da2m);
    conv_dgrad(U, L2A, U->da2m, U->dp2, nullptr, true);
    skip_pool_mask(U, 1, 32, U->du1m, U->dp2, U->a1, U->da1m);
    conv_wgrad(U, L1A, U->p1, U->da1m);
    conv_dgrad(U, L1A, U->da1m, U->dp1, nullptr, true);
    skip_pool_mask(U, 0, 16, U->du0m, U->dp1, U->a0, U->da0m);
    conv_wgrad(U, L0A, U->x0, U->da0m);
}

static void input(msbg_unet* U, const float* r, const double* s_in, bool training) {
    begin_launch(U->ctx);
    un_input_kernel<<<grid1(U->n[0]), 256, 0, U->ctx->stream>>>(U->n[0], r, s_in, U->x0c, training ? U->x0 : nullptr);
    after_launch(U->ctx, "un_input_kernel");
}

__global__ void un_output_kernel(int64_t n, const float* __restrict__ y, const double* __restrict__ s_in, float S,
                                 float* __restrict__ z) {
    const float s = (float)(*s_in) * S;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
        z[c] = s * y[c];
}

void unet_apply(msbg_unet* U, const float* r, float* z) {
    const double* s_in = rms_device(U, r);
    input(U, r, s_in, false);
    forward(U);
    begin_launch(U->ctx);
    un_output_kernel<<<grid1(U->n[0]), 256, 0, U->ctx->stream>>>(U->n[0], U->y, s_in, U->out_scale, z);
    after_launch(U->ctx, "un_output_kernel");
}

static double loss_and_grads(msbg_unet* U, const float* r, const float* e) {
    msbg_ctx* ctx = U->ctx;
    const double* s_in = rms_device(U, r);
    input(U, r, s_in, true);
    forward(U);
    double* part = red_part(U);
    double* sums = red_out(U) + 100;  // clear of the rms (8, 9) and bias sums (16 .. 79)
    begin_launch(ctx);
    un_loss_kernel<<<RED_B, RED_T, 0, ctx->stream>>>(U->n[0], U->y, e, s_in, U->out_scale, part);
    after_launch(ctx, "un_loss_kernel");
    begin_launch(ctx);
    un_final_kernel<<<1, RED_T, 0, ctx->stream>>>(part, RED_B, 2, 0.0, 0, sums);
    after_launch(ctx, "un_final_kernel");
    begin_launch(ctx);
    un_dy_kernel<<<grid1(U->n[0]), 256, 0, ctx->stream>>>(U->n[0], U->y, e, s_in, sums, U->out_scale, U->dyb);
    after_launch(ctx, "un_dy_kernel");
    backward(U);
    double h[2];
    read_small(ctx, h, sums, 16);
    check_device_status(ctx);
    return h[0] > 0.0 ? h[1] / h[0] : 0.0;
}

static void adam(msbg_unet* U, float lr) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    U->adam_t++;
    const float bc1 = 1.0f - std::pow(b1, (float)U->adam_t), bc2 = 1.0f - std::pow(b2, (float)U->adam_t);
    begin_launch(U->ctx);
    un_adam_kernel<<<grid1((int64_t)U->n_params), 256, 0, U->ctx->stream>>>(
        (int64_t)U->n_params, U->params.as<float>(), U->grads.as<float>(), U->adam_m.as<float>(), U->adam_v.as<float>(),
        U->pmask.as<float>(), lr, b1, b2, eps, bc1, bc2);
    after_launch(U->ctx, "un_adam_kernel");
    U->weights_dirty = true;
}

double unet_train_step(msbg_unet* U, const float* r, const float* e, float lr, bool update) {
    const double loss = loss_and_grads(U, r, e);
    if (update) adam(U, lr);
    return loss;
}

int64_t unet_blocks(const msbg_unet* U) { return U->nb; }
msbg_ctx* unet_ctx(const msbg_unet* U) { return U->ctx; }

static void build(msbg_unet* U, uint64_t sx, uint64_t sy, uint64_t sz, const uint64_t* active, size_t n_active,
                  uint64_t seed) {
    const uint64_t nx = sx / 16, ny = sy / 16, nz = sz / 16;
    MSBG_REQUIRE(sx % 16 == 0 && sy % 16 == 0 && sz % 16 == 0, "network domain extents must be multiples of 16");
    std::vector<uint64_t> a(active, active + n_active);
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
    MSBG_REQUIRE(!a.empty(), "empty active set");
    for (uint64_t b : a) MSBG_REQUIRE(b < nx * ny * nz, "active block id out of range");
    U->nb = (int64_t)a.size();
    U->n[0] = U->nb * 4096;
    U->n[1] = U->nb * 512;
    U->n[2] = U->nb * 64;
    std::unordered_map<uint64_t, int32_t> slot;
    for (size_t i = 0; i < a.size(); ++i) slot[a[i]] = (int32_t)i;
    std::vector<int32_t> nbr(a.size() * 27, -1);
    for (size_t i = 0; i < a.size(); ++i) {
        const int64_t b = (int64_t)a[i], bx = b % nx, by = (b / nx) % ny, bz = b / (nx * ny);
        for (int t = 0; t < 27; ++t) {
            const int64_t X = bx + t % 3 - 1, Y = by + (t / 3) % 3 - 1, Z = bz + t / 9 - 1;
            if (X < 0 || Y < 0 || Z < 0 || X >= (int64_t)nx || Y >= (int64_t)ny || Z >= (int64_t)nz) continue;
            auto it = slot.find((uint64_t)(X + Y * nx + Z * nx * ny));
            if (it != slot.end()) nbr[i * 27 + t] = it->second;
        }
    }
    msbg_ctx* ctx = U->ctx;
    U->nbr.reserve(nbr.size() * 4);
    CUDA_CHECK(cudaMemcpyAsync(U->nbr.p, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    // layers: level, cin, cout (padded), real, relu
    struct Spec { int level, cin, cout, cin_real, cout_real; bool relu; };
    const Spec specs[N_LAYERS] = {{0, 16, 16, 1, 16, true},  {1, 16, 32, 16, 32, true}, {2, 32, 64, 32, 64, true},
                                  {2, 64, 64, 64, 64, true}, {2, 64, 32, 64, 32, false}, {1, 32, 32, 32, 32, true},
                                  {1, 32, 16, 32, 16, false}, {0, 16, 16, 16, 1, false}};
    size_t off = 0, boff = 0;
    for (const Spec& s : specs) {
        ULayer L{s.level, s.cin, s.cout, s.cin_real, s.cout_real, s.relu, 0, 0, 0};
        L.w_off = off;
        off += (size_t)27 * s.cin * s.cout;
        L.b_off = off;
        off += (size_t)s.cout;
        L.wb_off = boff;
        boff += (size_t)27 * s.cin * s.cout;
        U->layers.push_back(L);
    }
    U->n_params = off;
    U->n_wb = boff;
    // He initialisation over the real fan-in; padded entries and the masks are zero
    std::vector<float> p(off, 0.0f), mask(off, 0.0f);
    std::mt19937_64 rng(seed);
    for (const ULayer& L : U->layers) {
        const bool last = &L == &U->layers.back();
        const float stdv = (last ? 0.5f : 1.0f) * std::sqrt(2.0f / (27.0f * L.cin_real));
        std::normal_distribution<float> nd(0.0f, stdv);
        for (int t = 0; t < 27; ++t)
            for (int o = 0; o < L.cout; ++o)
                for (int i = 0; i < L.cin; ++i) {
                    const size_t e = L.w_off + ((size_t)t * L.cout + o) * L.cin + i;
                    if (o < L.cout_real && i < L.cin_real) {
                        p[e] = nd(rng);
                        mask[e] = 1.0f;
                    }
                }
        for (int o = 0; o < L.cout_real; ++o) mask[L.b_off + o] = 1.0f;
    }
    U->params.reserve(off * 4);
    U->grads.reserve(off * 4);
    U->adam_m.reserve(off * 4);
    U->adam_v.reserve(off * 4);
    U->pmask.reserve(off * 4);
    CUDA_CHECK(cudaMemcpyAsync(U->params.p, p.data(), off * 4, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_CHECK(cudaMemcpyAsync(U->pmask.p, mask.data(), off * 4, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_CHECK(cudaMemsetAsync(U->grads.p, 0, off * 4, ctx->stream));
    CUDA_CHECK(cudaMemsetAsync(U->adam_m.p, 0, off * 4, ctx->stream));
    CUDA_CHECK(cudaMemsetAsync(U->adam_v.p, 0, off * 4, ctx->stream));
    U->wb.reserve(boff * 2);
    U->wt.reserve(boff * 2);
    // activations: bf16 channel counts per level
    const int64_t n0 = U->n[0], n1 = U->n[1], n2 = U->n[2];
    struct Slot { uint16_t** ptr; int64_t elems; };
    const Slot slots[] = {{&U->x0, n0 * 16},  {&U->a0, n0 * 16},   {&U->p1, n1 * 16},   {&U->a1, n1 * 32},
                          {&U->p2, n2 * 32},  {&U->a2, n2 * 64},   {&U->a3, n2 * 64},   {&U->c2, n2 * 32},
                          {&U->u1, n1 * 32},  {&U->a4, n1 * 32},   {&U->c1, n1 * 16},   {&U->u0, n0 * 16},
                          {&U->dyb, n0 * 16}, {&U->du0m, n0 * 16}, {&U->dc1, n1 * 16},  {&U->da4m, n1 * 32},
                          {&U->du1m, n1 * 32}, {&U->dc2, n2 * 32}, {&U->da3m, n2 * 64}, {&U->da2m, n2 * 64},
                          {&U->da1m, n1 * 32}, {&U->da0m, n0 * 16}};
    size_t bytes = (((size_t)n0 * 2 + 255) & ~size_t(255));  // x0c
    for (const Slot& s : slots) bytes += ((size_t)s.elems * 2 + 255) & ~size_t(255);
    const size_t f32_bytes = (((size_t)n0 * 4 + 255) & ~size_t(255)) + (((size_t)n2 * 32 * 4 + 255) & ~size_t(255)) +
                             (((size_t)n1 * 16 * 4 + 255) & ~size_t(255));
    U->act.reserve(bytes + f32_bytes + 256);
    char* base = (char*)U->act.p;
    U->x0c = reinterpret_cast<uint16_t*>(base);
    base += ((size_t)n0 * 2 + 255) & ~size_t(255);
    for (const Slot& s : slots) {
        *s.ptr = reinterpret_cast<uint16_t*>(base);
        base += ((size_t)s.elems * 2 + 255) & ~size_t(255);
    }
    U->y = reinterpret_cast<float*>(base);
    base += ((size_t)n0 * 4 + 255) & ~size_t(255);
    U->dp2 = reinterpret_cast<float*>(base);
    base += ((size_t)n2 * 32 * 4 + 255) & ~size_t(255);
    U->dp1 = reinterpret_cast<float*>(base);
    U->red.reserve(((size_t)RED_B * 64 + 128) * 8);
    U->weights_dirty = true;
    sync(ctx);
}

}  // namespace msbg

using namespace msbg;

extern "C" {

int msbg_unet_create(msbg_ctx* ctx, uint64_t sx, uint64_t sy, uint64_t sz, const uint64_t* active, size_t n,
                     uint64_t seed, msbg_unet** out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && out && (active || !n), "null argument");
    set_device(ctx);
    auto* U = new msbg_unet;
    U->ctx = ctx;
    try {
        build(U, sx, sy, sz, active, n, seed);
    } catch (...) {
        delete U;
        throw;
    }
    *out = U;
    MSBG_API_END
}

int msbg_unet_destroy(msbg_unet* U) {
    MSBG_API_BEGIN
    if (!U) return MSBG_OK;
    cudaSetDevice(U->ctx->device);
    cudaStreamSynchronize(U->ctx->stream);
    delete U;
    MSBG_API_END
}

int msbg_unet_num_params(const msbg_unet* U, size_t* out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(U && out, "null argument");
    *out = U->n_params;
    MSBG_API_END
}

// Layer table: per layer (level, cin, cout, cin_real, cout_real, relu, w_off, b_off).
int msbg_unet_layers(const msbg_unet* U, int64_t* out, size_t cap, size_t* n_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(U && n_out, "null argument");
    *n_out = U->layers.size();
    for (size_t i = 0; i < U->layers.size() && (i + 1) * 8 <= cap; ++i) {
        const ULayer& L = U->layers[i];
        const int64_t v[8] = {L.level, L.cin, L.cout, L.cin_real, L.cout_real, L.relu ? 1 : 0, (int64_t)L.w_off,
                              (int64_t)L.b_off};
        std::copy(v, v + 8, out + i * 8);
    }
    MSBG_API_END
}

int msbg_unet_get_params(msbg_unet* U, float* out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(U && out, "null argument");
    set_device(U->ctx);
    CUDA_CHECK(cudaMemcpyAsync(out, U->params.p, U->n_params * 4, cudaMemcpyDeviceToHost, U->ctx->stream));
    sync(U->ctx);
    MSBG_API_END
}

int msbg_unet_set_params(msbg_unet* U, const float* in) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(U && in, "null argument");
    set_device(U->ctx);
    CUDA_CHECK(cudaMemcpyAsync(U->params.p, in, U->n_params * 4, cudaMemcpyHostToDevice, U->ctx->stream));
    sync(U->ctx);
    U->weights_dirty = true;
    MSBG_API_END
}

int msbg_unet_get_grads(msbg_unet* U, float* out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(U && out, "null argument");
    set_device(U->ctx);
    CUDA_CHECK(cudaMemcpyAsync(out, U->grads.p, U->n_params * 4, cudaMemcpyDeviceToHost, U->ctx->stream));
    sync(U->ctx);
    MSBG_API_END
}

int msbg_unet_set_output_scale(msbg_unet* U, float s) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(U && std::isfinite(s), "bad argument");
    U->out_scale = s;
    MSBG_API_END
}

int msbg_unet_apply_device(msbg_unet* U, const float* d_r, float* d_z) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(U && d_r && d_z, "null argument");
    set_device(U->ctx);
    unet_apply(U, d_r, d_z);
    MSBG_API_END
}

// Forward output y (f32 [n0]) for the input x = r / rms(r), for tests.
int msbg_unet_forward_raw_device(msbg_unet* U, const float* d_r, float* d_y) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(U && d_r && d_y, "null argument");
    set_device(U->ctx);
    const double* s_in = rms_device(U, d_r);
    input(U, d_r, s_in, false);
    forward(U);
    CUDA_CHECK(cudaMemcpyAsync(d_y, U->y, U->n[0] * 4, cudaMemcpyDeviceToDevice, U->ctx->stream));
    sync(U->ctx);
    check_device_status(U->ctx);
    MSBG_API_END
}

int msbg_unet_train_step_device(msbg_unet* U, const float* d_r, const float* d_e, float lr, int update, double* loss_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(U && d_r && d_e && lr >= 0.0f, "bad argument");
    set_device(U->ctx);
    const double l = unet_train_step(U, d_r, d_e, lr, update != 0);
    if (loss_out) *loss_out = l;
    MSBG_API_END
}

}  // extern "C"
