// conv.cu -- block-sparse 3x3x3 convolutions on tcgen05 (see conv.cuh).
#include <algorithm>

#include "conv.cuh"
#include "tc.cuh"

namespace msbg {

constexpr int kConvStages = 3;
constexpr int kWgCells = 64;  // cells (K) per weight-gradient stage

__device__ __forceinline__ uint16_t bf16_rne(float v) { return ElemBF16::store(v); }

// Source row of cell `cell` shifted by tap t, or null when it falls outside
// the active blocks (zero padding).
template <int C>
__device__ __forceinline__ const uint4* tap_row(const ConvLevel& L, const uint16_t* __restrict__ x, int64_t cell, int t) {
    const int lg = L.lg, m = (1 << lg) - 1;
    const int64_t k = cell >> (3 * lg);
    const int v = (int)(cell & ((1 << (3 * lg)) - 1));
    const int gx = (v & m) + t % 3 - 1, gy = ((v >> lg) & m) + (t / 3) % 3 - 1, gz = (v >> (2 * lg)) + t / 9 - 1;
    const int ox = gx < 0 ? 0 : (gx > m ? 2 : 1), oy = gy < 0 ? 0 : (gy > m ? 2 : 1), oz = gz < 0 ? 0 : (gz > m ? 2 : 1);
    const int code = ox + 3 * oy + 9 * oz;
    const int32_t kk = code == 13 ? (int32_t)k : L.nbr27[k * 27 + code];
    if (kk < 0 || kk >= L.n_blocks) return nullptr;  // absent (or a corrupt table entry: read as zero)
    const int64_t c2 = ((int64_t)kk << (3 * lg)) + ((gx & m) | ((gy & m) << lg) | ((gz & m) << (2 * lg)));
    return reinterpret_cast<const uint4*>(x + c2 * C);
}

// Stages of the forward pipeline: four while they fit in 64 KB, else three.
template <int CIN, int COUT>
constexpr int fwd_stages() { return 4 * (128 * CIN * 2 + COUT * CIN * 2) <= 65536 ? 4 : 3; }

template <int CIN, int COUT>
struct FwdSmem {
    static constexpr int STAGES = fwd_stages<CIN, COUT>();
    static constexpr int A_BYTES = 128 * CIN * 2;
    static constexpr int B_BYTES = COUT * CIN * 2;
    static constexpr int OFF_B = STAGES * A_BYTES;
    static constexpr int OFF_BAR = OFF_B + STAGES * B_BYTES;
    static constexpr int BYTES = OFF_BAR + 64;
    // At least 32 KB per CTA: at most 7 CTAs share an SM, so their TMEM
    // columns (<= 64 each) never exceed the 512 an SM has.
    static constexpr int ALLOC = BYTES < 32768 ? 32768 : BYTES;
};

// 16-byte asynchronous copy global -> shared; `present` false writes zeros
// (source size 0: nothing is read from `src`).
__device__ __forceinline__ void cp16_zfill(void* dst, const void* src, bool present) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(tc::smem_u32(dst)), "l"(src),
                 "r"(present ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Epilogue of one output cell: 16 accumulator columns c0 .. c0 + 15, plus
// bias, ReLU, the optional ReLU-derivative mask; bf16 or f32 rows.
template <int COUT>
__device__ __forceinline__ void store16(float* acc, int64_t cell, int c0, const float* __restrict__ bias, int relu,
                                        const uint16_t* __restrict__ mask, int out_f32, int out_ch,
                                        void* __restrict__ y) {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        float v = acc[i] + (bias ? __ldg(bias + c0 + i) : 0.0f);
        acc[i] = relu ? fmaxf(v, 0.0f) : v;
    }
    if (mask) {  // ReLU backward: zero where the layer's stored activation is not positive
        const uint4* mk = reinterpret_cast<const uint4*>(mask + cell * COUT + c0);
        uint32_t mw[8];
        *reinterpret_cast<uint4*>(mw) = __ldg(mk);
        *reinterpret_cast<uint4*>(mw + 4) = __ldg(mk + 1);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const uint32_t h = (mw[i >> 1] >> (16 * (i & 1))) & 0xFFFFu;
            if (!(h != 0u && !(h & 0x8000u))) acc[i] = 0.0f;  // bf16 > 0: nonzero, sign clear
        }
    }
    if (out_f32 && out_ch < COUT) {
        float* yo = static_cast<float*>(y) + cell * out_ch + c0;
#pragma unroll
        for (int i = 0; i < 16; ++i)
            if (c0 + i < out_ch) yo[i] = acc[i];
    } else if (out_f32) {
        float4* yo = reinterpret_cast<float4*>(static_cast<float*>(y) + cell * COUT + c0);
#pragma unroll
        for (int i = 0; i < 4; ++i) yo[i] = make_float4(acc[4 * i], acc[4 * i + 1], acc[4 * i + 2], acc[4 * i + 3]);
    } else {
        uint32_t pk[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) pk[i] = (uint32_t)bf16_rne(acc[2 * i]) | ((uint32_t)bf16_rne(acc[2 * i + 1]) << 16);
        uint4* yo = reinterpret_cast<uint4*>(static_cast<uint16_t*>(y) + cell * COUT + c0);
        yo[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        yo[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    }
}

// Taps flow through STAGES shared-memory stages: the copies of taps t + 1 ..
// t + STAGES - 2 are in flight (cp.async, zero-filled outside the active
// blocks) while the MMAs of tap t run, and a stage is refilled once the MMAs
// that read it (two taps back) have arrived on its mbarrier.
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) conv3_fwd_kernel(ConvLevel L, const uint16_t* __restrict__ x,
                                                        const uint16_t* __restrict__ w, const float* __restrict__ bias,
                                                        int relu, const uint16_t* __restrict__ mask, int out_f32,
                                                        int out_ch, void* __restrict__ y, int* __restrict__ status) {
    using S = FwdSmem<CIN, COUT>;
    constexpr int ST = S::STAGES;
    constexpr int TCOLS = COUT < 32 ? 32 : COUT;
    constexpr int KCH = CIN / 8;
    constexpr uint32_t SBO = KCH * 128;
    constexpr uint32_t IDESC = tc::idesc_bf16(128, COUT, 0, 0);
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S::OFF_BAR);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + ST);
    const int tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) tc::tmem_alloc(tslot, TCOLS);
    if (tid == 0) {
        for (int s = 0; s < ST; ++s) tc::mbar_init(&bars[s], 1);
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;

    const int64_t cell = (int64_t)blockIdx.x * 128 + tid;
    const bool valid = cell < L.cells();
    auto issue = [&](int t) {
        const int s = t % ST;
        const uint4* src = valid ? tap_row<CIN>(L, x, cell, t) : nullptr;
        const uint4* from = src ? src : reinterpret_cast<const uint4*>(x);
        uint8_t* arow = smem + s * S::A_BYTES + (tid >> 3) * SBO + (tid & 7) * 16;
#pragma unroll
        for (int j = 0; j < KCH; ++j) cp16_zfill(arow + j * 128, src ? from + j : from, src != nullptr);
        uint8_t* bst = smem + S::OFF_B + s * S::B_BYTES;
        const uint4* wt = reinterpret_cast<const uint4*>(w + (int64_t)t * COUT * CIN);
#pragma unroll
        for (int q = tid; q < COUT * KCH; q += 128) {
            const int n = q / KCH, j = q % KCH;
            cp16_zfill(bst + (n >> 3) * SBO + j * 128 + (n & 7) * 16, wt + q, true);
        }
    };
    constexpr int D = ST - 2;  // prefetch distance in taps
    bool ok = true;
#pragma unroll 1
    for (int t = 0; t < D; ++t) {
        issue(t);
        cp_commit();
    }
#pragma unroll 1
    for (int t = 0; t < 27; ++t) {
        const int s = t % ST;
        cp_wait<D - 1>();  // this thread's copies of tap t have landed
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t a0 = tc::smem_u32(smem + s * S::A_BYTES), b0 = tc::smem_u32(smem + S::OFF_B + s * S::B_BYTES);
#pragma unroll
            for (int kk = 0; kk < CIN / 16; ++kk)
                tc::mma_bf16(tmem, tc::sdesc(a0 + kk * 256, 128, SBO), tc::sdesc(b0 + kk * 256, 128, SBO), IDESC,
                             (t | kk) != 0);
            tc::mma_commit(&bars[s]);
        }
        const int tn = t + D;  // refills the stage of tap tn - ST = t - 2
        if (tn < 27) {
            if (tn >= ST) ok &= tc::mbar_wait(&bars[tn % ST], ((tn - ST) / ST) & 1);
            issue(tn);
        }
        cp_commit();
    }
    ok &= tc::mbar_wait(&bars[26 % ST], (26 / ST) & 1);
    tc::fence_after_sync();
    float acc[16];
#pragma unroll
    for (int c0 = 0; c0 < COUT; c0 += 16) {
        tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, acc);
        if (valid && c0 < out_ch) store16<COUT>(acc, cell, c0, bias, relu, mask, out_f32, out_ch, y);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, TCOLS);
    if (!ok && tid == 0) atomicOr(status, 1);
}

// 8^3 blocks (lg = 3), Cin and Cout <= 32: persistent CTAs, one per SM,
// over the blocks.  The weights of all 27 taps are copied into shared memory
// once; per block, its input halo (10^3 rows, each 8-channel chunk of it a
// slab of 16-byte rows in x | y | z order) is copied into one of two halo
// buffers.  Each tap's operand for one z-plane of the block is then a view of
// the halo: 8 groups (y) of 8 rows (x), the groups 160 bytes apart, so one
// lane of warp z issues every MMA of plane z (M = the 64 cells of the plane,
// N = Cout, K = Cin per tap) back to back with no per-tap staging.  Plane z
// of a block accumulates in TMEM columns z * Cout .. of one of two
// accumulators, in the M = 64 data-path layout (row m of the plane in lane
// (m % 16) + 32 (m / 16)).
// While the tensor core works on block i, the threads copy the halo of block
// i + 1 and write out block i - 1.
constexpr int kB8Threads = 512;

template <int CIN, int COUT>
struct B8Smem {
    static constexpr int KCH = CIN / 8;
    static constexpr int SLAB = 1000 * 16;  // one 8-channel chunk of a halo
    static constexpr int HALO = KCH * SLAB;
    static constexpr int B_BYTES = COUT * CIN * 2;
    static constexpr int OFF_W = 2 * HALO;
    static constexpr int OFF_BAR = OFF_W + 27 * B_BYTES;
    static constexpr int BYTES = OFF_BAR + 64;
    static constexpr int ACC_COLS = 8 * COUT;
    static constexpr int TCOLS = 2 * ACC_COLS;
    // More than half of the SM's shared memory: one CTA per SM, so the
    // TMEM columns (up to all 512) are never contended.
    static constexpr int ALLOC = BYTES < 116 * 1024 ? 116 * 1024 : BYTES;
    static constexpr bool FITS = CIN <= 32 && COUT <= 32 && ALLOC <= 227 * 1024;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(kB8Threads) conv3_b8_kernel(ConvLevel L, const uint16_t* __restrict__ x,
                                                              const uint16_t* __restrict__ w,
                                                              const float* __restrict__ bias, int relu,
                                                              const uint16_t* __restrict__ mask, int out_f32, int out_ch,
                                                              void* __restrict__ y, int* __restrict__ status) {
    using S = B8Smem<CIN, COUT>;
    constexpr int KCH = S::KCH;
    constexpr uint32_t SBO_W = KCH * 128;
    constexpr uint32_t IDESC = tc::idesc_bf16(64, COUT, 0, 0);
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S::OFF_BAR);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // halo of block k into buffer `buf` (zero rows outside the active blocks)
    auto load_halo = [&](int64_t k, int buf) {
        uint8_t* hb = smem + buf * S::HALO;
#pragma unroll 4
        for (int e = tid; e < 1000 * KCH; e += kB8Threads) {
            const int h = e / KCH, j = e % KCH;
            const int gx = h % 10 - 1, gy = (h / 10) % 10 - 1, gz = h / 100 - 1;
            const int ox = gx < 0 ? 0 : (gx > 7 ? 2 : 1), oy = gy < 0 ? 0 : (gy > 7 ? 2 : 1),
                      oz = gz < 0 ? 0 : (gz > 7 ? 2 : 1);
            const int code = ox + 3 * oy + 9 * oz;
            const int32_t kk = code == 13 ? (int32_t)k : __ldg(L.nbr27 + k * 27 + code);
            const bool present = kk >= 0 && kk < L.n_blocks;
            const int64_t c2 = present ? ((int64_t)kk << 9) + ((gx & 7) | ((gy & 7) << 3) | ((gz & 7) << 6)) : 0;
            cp16_zfill(hb + j * S::SLAB + h * 16, reinterpret_cast<const uint4*>(x + c2 * CIN) + j, present);
        }
    };
    for (int e = tid; e < 27 * COUT * KCH; e += kB8Threads) {
        const int t = e / (COUT * KCH), q = e % (COUT * KCH), n = q / KCH, j = q % KCH;
        cp16_zfill(smem + S::OFF_W + t * S::B_BYTES + (n >> 3) * SBO_W + j * 128 + (n & 7) * 16,
                   reinterpret_cast<const uint4*>(w) + e, true);
    }
    const int64_t k0 = blockIdx.x;
    if (k0 < L.n_blocks) load_halo(k0, 0);
    cp_commit();
    if (warp == 0) tc::tmem_alloc(tslot, S::TCOLS);
    if (tid == 0) {
        tc::mbar_init(&bars[0], 8);  // one commit per issuing warp
        tc::mbar_init(&bars[1], 8);
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;

    // warps 4g .. 4g + 3 write planes 2g and 2g + 1; lanes 0-15 of warp w
    // hold rows 16 (w % 4) + lane of a plane
    auto epilogue = [&](int64_t k, int buf) {
        __syncwarp();  // tcgen05.ld is warp-wide
        const int m = 16 * (warp & 3) + (lane & 15);
        float acc[16];
#pragma unroll 1
        for (int zz = 0; zz < 2; ++zz) {
            const int z = 2 * (warp >> 2) + zz;
            const int64_t cell = (k << 9) + ((m & 7) | ((m >> 3) << 3) | (z << 6));
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 16) {
                tc::tmem_ld16(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(buf * S::ACC_COLS + z * COUT + c0),
                              acc);
                if (lane < 16 && c0 < out_ch) store16<COUT>(acc, cell, c0, bias, relu, mask, out_f32, out_ch, y);
            }
        }
    };

    bool ok = true;
    int i = 0;
    int64_t kprev = -1;
#pragma unroll 1
    for (int64_t k = k0; k < L.n_blocks; k += gridDim.x, ++i) {
        const int buf = i & 1;
        cp_wait<0>();  // this thread's copies of block k's halo (and the weights) have landed
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (lane == 0 && warp < 8) {
            // warp w issues the MMAs of plane w (every offset below is a
            // compile-time constant added to the descriptors' address field)
            const int z = warp;
            const uint64_t a0 = tc::sdesc(tc::smem_u32(smem + buf * S::HALO) + (uint32_t)(z * 1600), S::SLAB, 160);
            const uint64_t b0 = tc::sdesc(tc::smem_u32(smem + S::OFF_W), 128, SBO_W);
            const uint32_t d = tmem + (uint32_t)(buf * S::ACC_COLS + z * COUT);
#pragma unroll 1
            for (int dz = 0; dz < 3; ++dz) {
                // dz * 100: one halo plane (1600 bytes) in the 16-byte units of the address field
                const uint64_t az = a0 + (uint64_t)(dz * 100), bz = b0 + (uint64_t)((dz * 9 * S::B_BYTES) >> 4);
#pragma unroll
                for (int r = 0; r < 9; ++r) {
#pragma unroll
                    for (int kk = 0; kk < CIN / 16; ++kk) {
                        const uint32_t ao = ((r / 3) * 10 + r % 3) * 16 + 2 * kk * S::SLAB;
                        const uint32_t bo = r * S::B_BYTES + kk * 256;
                        tc::mma_bf16(d, az + (ao >> 4), bz + (bo >> 4), IDESC, (dz | r | kk) != 0);
                    }
                }
            }
            tc::mma_commit(&bars[buf]);
        }
        if (kprev >= 0) {
            // block kprev's MMAs (the previous use of the other halo buffer) are done
            ok &= tc::mbar_wait(&bars[buf ^ 1], ((i - 1) >> 1) & 1);
            tc::fence_after_sync();
        }
        if (k + gridDim.x < L.n_blocks) load_halo(k + gridDim.x, buf ^ 1);
        cp_commit();
        if (kprev >= 0) epilogue(kprev, buf ^ 1);
        kprev = k;
    }
    if (kprev >= 0) {
        ok &= tc::mbar_wait(&bars[(i - 1) & 1], ((i - 1) >> 1) & 1);
        tc::fence_after_sync();
        epilogue(kprev, (i - 1) & 1);
    }
    cp_wait<0>();
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, S::TCOLS);
    if (!ok && tid == 0) atomicOr(status, 1);
}

template <int CIN, int COUT>
struct WgSmem {
    static constexpr int A_BYTES = 128 * kWgCells * 2;
    static constexpr int B_BYTES = COUT * kWgCells * 2;
    static constexpr int OFF_B = kConvStages * A_BYTES;
    static constexpr int OFF_BAR = OFF_B + kConvStages * B_BYTES;
    static constexpr int BYTES = OFF_BAR + 64;
    static constexpr int ALLOC = BYTES < 32768 ? 32768 : BYTES;
};

// partial[part][q][o], q = tap * CIN + i over tiles of 128 (rows past
// 27 * CIN are zero).
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) conv3_wgrad_kernel(ConvLevel L, const uint16_t* __restrict__ x,
                                                          const uint16_t* __restrict__ dy, int64_t cells_per_part,
                                                          float* __restrict__ partial, int* __restrict__ status) {
    using S = WgSmem<CIN, COUT>;
    constexpr int TCOLS = COUT < 32 ? 32 : COUT;
    constexpr uint32_t SBO = (kWgCells / 8) * 128;
    constexpr uint32_t IDESC = tc::idesc_bf16(128, COUT, 1, 1);
    constexpr int TPT = 128 / CIN;  // taps per M tile
    constexpr int MROWS = ((27 * CIN + 127) / 128) * 128;
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S::OFF_BAR);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + kConvStages);
    const int tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) tc::tmem_alloc(tslot, TCOLS);
    if (tid == 0) {
        for (int s = 0; s < kConvStages; ++s) tc::mbar_init(&bars[s], 1);
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;

    const int mt = blockIdx.x, part = blockIdx.y;
    const int tap0 = mt * TPT;
    const int64_t total = L.cells();
    const int64_t c_begin = (int64_t)part * cells_per_part;
    const int64_t c_end = std::min<int64_t>(total, c_begin + cells_per_part);
    const int nchunks = c_end > c_begin ? (int)((c_end - c_begin + kWgCells - 1) / kWgCells) : 0;
    bool ok = true;
    for (int ch = 0; ch < nchunks; ++ch) {
        const int s = ch % kConvStages;
        if (ch >= kConvStages) ok &= tc::mbar_wait(&bars[s], ((ch / kConvStages) - 1) & 1);
        const int64_t cbase = c_begin + (int64_t)ch * kWgCells;
        uint8_t* ast = smem + s * S::A_BYTES;
#pragma unroll 4
        for (int r = 0; r < (kWgCells * 16) / 128; ++r) {
            const int item = tid + 128 * r;
            const int c = item % kWgCells, mg = item / kWgCells;
            const int64_t cell = cbase + c;
            const int q0 = mg * 8;
            const int tap = tap0 + q0 / CIN, ci0 = q0 % CIN;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (cell < c_end && tap < 27) {
                const uint4* src = tap_row<CIN>(L, x, cell, tap);
                if (src) v = __ldg(src + ci0 / 8);
            }
            *reinterpret_cast<uint4*>(ast + mg * SBO + (c >> 3) * 128 + (c & 7) * 16) = v;
        }
        uint8_t* bst = smem + S::OFF_B + s * S::B_BYTES;
        for (int item = tid; item < kWgCells * (COUT / 8); item += 128) {
            const int c = item % kWgCells, ng = item / kWgCells;
            const int64_t cell = cbase + c;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (cell < c_end) v = __ldg(reinterpret_cast<const uint4*>(dy + cell * COUT) + ng);
            *reinterpret_cast<uint4*>(bst + ng * SBO + (c >> 3) * 128 + (c & 7) * 16) = v;
        }
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t a0 = tc::smem_u32(ast), b0 = tc::smem_u32(bst);
#pragma unroll
            for (int kk = 0; kk < kWgCells / 16; ++kk)
                tc::mma_bf16(tmem, tc::sdesc(a0 + kk * 256, 128, SBO), tc::sdesc(b0 + kk * 256, 128, SBO), IDESC,
                             (ch | kk) != 0);
            tc::mma_commit(&bars[s]);
        }
    }
    if (nchunks > 0) {
        ok &= tc::mbar_wait(&bars[(nchunks - 1) % kConvStages], ((nchunks - 1) / kConvStages) & 1);
        tc::fence_after_sync();
    }
    float acc[16];
    const int q = mt * 128 + tid;
    float* out = partial + ((int64_t)part * MROWS + q) * COUT;
#pragma unroll
    for (int c0 = 0; c0 < COUT; c0 += 16) {
        if (nchunks > 0) {
            tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, acc);
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[i] = 0.0f;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
            reinterpret_cast<float4*>(out + c0)[i] = make_float4(acc[4 * i], acc[4 * i + 1], acc[4 * i + 2], acc[4 * i + 3]);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, TCOLS);
    if (!ok && tid == 0) atomicOr(status, 1);
}

// dw[t][o][i] (+)= sum over parts (in order) of partial[part][t * CIN + i][o]
__global__ void conv3_wgrad_reduce_kernel(const float* __restrict__ partial, int parts, int cin, int cout, int mrows,
                                          float* __restrict__ dw, int acc) {
    const int n = 27 * cin * cout;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int i = e % cin, o = (e / cin) % cout, t = e / (cin * cout);
        const int q = t * cin + i;
        float s = 0.0f;
        for (int p = 0; p < parts; ++p) s += partial[((int64_t)p * mrows + q) * cout + o];
        dw[e] = acc ? dw[e] + s : s;
    }
}

template <int CIN, int COUT>
static void launch_fwd(msbg_ctx* ctx, const ConvLevel& L, const uint16_t* x, const uint16_t* w, const float* bias, bool relu,
                       const uint16_t* mask, bool out_f32, int out_ch, void* y) {
    using S = FwdSmem<CIN, COUT>;
    static bool attr = false;
    if (!attr) {
        CUDA_CHECK(cudaFuncSetAttribute(conv3_fwd_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::ALLOC));
        attr = true;
    }
    const int64_t cells = L.cells();
    if (!cells) return;
    if constexpr (B8Smem<CIN, COUT>::FITS) {
        if (L.lg == 3) {
            using S8 = B8Smem<CIN, COUT>;
            static bool attr8 = false;
            if (!attr8) {
                CUDA_CHECK(cudaFuncSetAttribute(conv3_b8_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                S8::ALLOC));
                attr8 = true;
            }
            static int sms = 0;
            if (!sms) CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
            begin_launch(ctx);
            const unsigned grid = (unsigned)std::min<int64_t>(L.n_blocks, sms);
            conv3_b8_kernel<CIN, COUT><<<grid, kB8Threads, S8::ALLOC, ctx->stream>>>(
                L, x, w, bias, relu ? 1 : 0, mask, out_f32 ? 1 : 0, out_ch > 0 ? out_ch : COUT, y, ctx->status.as<int>());
            after_launch(ctx, "conv3_b8_kernel");
            return;
        }
    }
    begin_launch(ctx);
    conv3_fwd_kernel<CIN, COUT><<<(unsigned)((cells + 127) / 128), 128, S::ALLOC, ctx->stream>>>(
        L, x, w, bias, relu ? 1 : 0, mask, out_f32 ? 1 : 0, out_ch > 0 ? out_ch : COUT, y, ctx->status.as<int>());
    after_launch(ctx, "conv3_fwd_kernel");
}

template <int CIN, int COUT>
static void launch_wgrad(msbg_ctx* ctx, const ConvLevel& L, const uint16_t* x, const uint16_t* dy, float* dw, bool acc) {
    using S = WgSmem<CIN, COUT>;
    static bool attr = false;
    if (!attr) {
        CUDA_CHECK(cudaFuncSetAttribute(conv3_wgrad_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::ALLOC));
        attr = true;
    }
    constexpr int MT = (27 * CIN + 127) / 128;
    constexpr int MROWS = MT * 128;
    const int64_t cells = L.cells();
    // about 4 CTAs per SM in total, each over a contiguous range of whole 64-cell chunks
    const int64_t chunks = std::max<int64_t>(1, (cells + kWgCells - 1) / kWgCells);
    const int parts = (int)std::min<int64_t>(chunks, std::max<int64_t>(1, 592 / MT));
    const int64_t cells_per_part = ((chunks + parts - 1) / parts) * kWgCells;
    ScratchLayout SL;
    const size_t op = SL.add<float>((size_t)parts * MROWS * COUT);
    float* partial = ScratchLayout::at<float>(scratch(ctx, SL), op);
    begin_launch(ctx);
    conv3_wgrad_kernel<CIN, COUT><<<dim3(MT, parts), 128, S::ALLOC, ctx->stream>>>(L, x, dy, cells_per_part, partial,
                                                                                  ctx->status.as<int>());
    after_launch(ctx, "conv3_wgrad_kernel");
    begin_launch(ctx);
    conv3_wgrad_reduce_kernel<<<(27 * CIN * COUT + 255) / 256, 256, 0, ctx->stream>>>(partial, parts, CIN, COUT, MROWS, dw,
                                                                                       acc ? 1 : 0);
    after_launch(ctx, "conv3_wgrad_reduce_kernel");
}

#define MSBG_CONV_PAIRS(X) X(16, 32) X(32, 16) X(32, 32) X(32, 64) X(64, 32) X(64, 64) X(16, 16) X(64, 16) X(16, 64)

void conv3_forward(msbg_ctx* ctx, const ConvLevel& L, int cin, int cout, const uint16_t* x, const uint16_t* w,
                   const float* bias, bool relu, bool out_f32, void* y, const uint16_t* mask, int out_ch) {
    MSBG_REQUIRE(out_ch >= 0 && out_ch <= cout && (out_f32 || out_ch == 0 || out_ch == cout), "conv3: bad output width");
#define MSBG_FWD_CASE(A, B) \
    if (cin == A && cout == B) return launch_fwd<A, B>(ctx, L, x, w, bias, relu, mask, out_f32, out_ch, y);
    MSBG_CONV_PAIRS(MSBG_FWD_CASE)
#undef MSBG_FWD_CASE
    MSBG_THROW(MSBG_ERR_ARG, "conv3: channel counts must be 16, 32 or 64");
}

void conv3_wgrad(msbg_ctx* ctx, const ConvLevel& L, int cin, int cout, const uint16_t* x, const uint16_t* dy, float* dw,
                 bool acc) {
#define MSBG_WG_CASE(A, B) \
    if (cin == A && cout == B) return launch_wgrad<A, B>(ctx, L, x, dy, dw, acc);
    MSBG_CONV_PAIRS(MSBG_WG_CASE)
#undef MSBG_WG_CASE
    MSBG_THROW(MSBG_ERR_ARG, "conv3: channel counts must be 16, 32 or 64");
}

}  // namespace msbg

using namespace msbg;

extern "C" {

int msbg_conv3_forward_device(msbg_ctx* ctx, const int32_t* d_nbr27, int64_t n_blocks, int lg, int cin, int cout,
                              const uint16_t* d_x, const uint16_t* d_w, const float* d_bias, int relu, int out_f32,
                              void* d_y) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && d_nbr27 && d_x && d_w && d_y && n_blocks >= 0 && lg >= 1 && lg <= 5, "bad argument");
    set_device(ctx);
    conv3_forward(ctx, ConvLevel{d_nbr27, lg, n_blocks}, cin, cout, d_x, d_w, d_bias, relu != 0, out_f32 != 0, d_y);
    check_device_status(ctx);
    MSBG_API_END
}

int msbg_conv3_wgrad_device(msbg_ctx* ctx, const int32_t* d_nbr27, int64_t n_blocks, int lg, int cin, int cout,
                            const uint16_t* d_x, const uint16_t* d_dy, float* d_dw) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && d_nbr27 && d_x && d_dy && d_dw && n_blocks >= 0 && lg >= 1 && lg <= 5, "bad argument");
    set_device(ctx);
    conv3_wgrad(ctx, ConvLevel{d_nbr27, lg, n_blocks}, cin, cout, d_x, d_dy, d_dw, false);
    check_device_status(ctx);
    MSBG_API_END
}

}  // extern "C"
