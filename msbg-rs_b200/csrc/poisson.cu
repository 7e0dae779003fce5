// poisson.cu -- matrix-free Poisson solve on the sparse block grid: the 7-point
// operator, weighted Jacobi, a geometric V-cycle over the multiresolution
// hierarchy, and MG-preconditioned CG with FP64 dot products.
//
// The crate has no pressure solver (docs/roadmap.md:608-702 lists the
// operator and the multigrid as not started); the operator follows the
// formulas stated there: matvec y = D x - sum_nb x, relaxation
// y = w (b + sum_nb x) D^-1 + (1 - w) x, with D = 6 (unit spacing) and zero
// Dirichlet values outside the active blocks.
//
// Hierarchy (level l+1 has cells twice the size of level l): while the block
// size is >= 4 the block grid is kept and the block size halves; from block
// size 2 on the block grid halves.  A coarse cell is active when any of its 8
// children is, so every level covers the cells of level 0 (while its cells
// are no wider than a level-0 block).  The level-l operator is the 7-point
// stencil rediscretised on cells of width 2^l in the units of the level-0
// equation, s_l ((6 - g_l m) x - sum of active neighbours), s_l = 0.25^l,
// with m the missing face neighbours of the cell and g_l = 1 - 1/d,
// d = 1/2 + 2^(-l-1): the ghost value that puts the zero Dirichlet value
// where level 0 has it, half a level-0 cell outside the boundary face.
// Prolongation is cell-centred trilinear (3/4 from the parent cell, 1/4 from
// its neighbour on the child's side, per axis), restriction R = P^T / 8, so
// the V-cycle with nu1 = nu2 is symmetric.  Coarsening stops at <= 1024
// cells, solved with a dense FP64 inverse computed at set-up (Cholesky on
// the host; inactive cells have identity rows).  Measured on shells of
// 16^3 and 8^3 blocks, one V(2,2)-cycle with w = 2/3 Jacobi reduces the
// residual by about 0.38, close to the smoothing factor of w-Jacobi in 3D
// (7/9 per sweep).
//
// Layout in HBM: one f32 array per level and vector, [n_blocks][bs^3] in
// ascending block-id order (the block payload layout of the sparse grid).
// Vectors and smoothing are FP32; dot products and norms accumulate in FP64
// with a fixed two-stage reduction order (deterministic).
#include <algorithm>
#include <cmath>
#include <random>

#include "common.cuh"
#include "unet.cuh"

namespace msbg {

constexpr int64_t kPoissonDirect = 1024;

struct PLevelDev {
    int bs, lg;
    int64_t nx, ny, nz;
    std::vector<uint64_t> bids;
    float scale;
    DevBuf nbr;      // int32 [n][6]
    DevBuf coords;   // int32 [n][3] block coordinates
    DevBuf parent;   // int32 [n] parent slot at level l+1 (the last level: unused)
    DevBuf pnb;      // int32 [n][27] level-(l+1) slots of the blocks around the parent block (prolongation)
    DevBuf rnb;      // int32 [n][64] level-(l-1) slots of the 4^3 fine blocks from fb0 (restriction), l >= 1
    DevBuf diag;     // f32 [cells] s_l (6 - g_l m), 0 for inactive cells; l >= 1 (level 0: 6, all active)
    DevBuf x, b, r, t;  // f32 [cells]
    int cfg_jac = 0, cfg_res = 0;  // launch shapes of the level's Jacobi and residual kernels (autotuned)
    int slab = 1;                  // tile of the 16^3 kernels: 1 quad tile, else slab z-planes (autotuned)
    int64_t n() const { return (int64_t)bids.size(); }
    int64_t cells() const { return n() * bs * bs * bs; }
};

}  // namespace msbg

struct msbg_poisson {
    msbg_ctx* ctx = nullptr;
    std::vector<msbg::PLevelDev> lv;
    msbg::DevBuf ainv;   // f64 [nc][nc] column-major inverse of the coarsest operator
    int64_t nc = 0;
    int nu1 = 2, nu2 = 2;
    float omega = 2.0f / 3.0f;
    msbg::DevBuf work;   // PCG vectors + dot partials
    msbg::DevBuf io;     // device copies of host x and b (msbg_poisson_solve), kept between calls
    msbg_unet* net = nullptr;  // learned preconditioner (not owned)
    // PCG statistics of the last solve: preconditioner applications of each
    // kind and whether the learned preconditioner fell back to multigrid
    int n_net = 0, n_vcycle = 0, fell_back = 0, fallback_iter = -1;
    int net_lead = 1;       // method 5: preconditioner applications that use the network
    int net_lead_post = 1;  // method 5: those applications end with the post-smoothing V-cycle
    // Batched solves: independent problems stacked in one hierarchy (see
    // batch_build); each owns a contiguous range of level-0 blocks.
    int np = 0;
    std::vector<int64_t> prob_blocks;  // [np + 1] level-0 block offsets
    msbg::DevBuf d_prob_blocks;        // int64 [np + 1]
    msbg::DevBuf d_blk_prob;           // int32 [level-0 blocks] problem of each block
    msbg::DevBuf bpart;                // f64 [level-0 blocks] per-block dot partials
    msbg::DevBuf scal;                 // f64 [np][16] per-problem scalars
    // Captured V-cycles of the single-problem solve, one per (x, b) pair: a
    // V-cycle is some 40 small launches, which one graph launch replaces.
    struct VGraph {
        float* x;
        const float* b;
        cudaGraphExec_t exec;
        int kernels;
    };
    std::vector<VGraph> vgraphs;
    // Captured solve loops of methods 0 and 1 (iterations in a device-side
    // while loop, no host read between them), one per (method, b, x64).
    struct SGraph {
        int method;
        const float* b;
        const double* x64;
        cudaGraphExec_t exec;
        int kernels_first, kernels_body;  // launches before the loop and per loop iteration
    };
    std::vector<SGraph> sgraphs;
    msbg::DevBuf sctl;   // SolveCtl of the captured loops
    msbg::DevBuf shist;  // f64 [capacity] relative residual per iteration
    ~msbg_poisson() {
        for (auto& g : vgraphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        for (auto& g : sgraphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
    }
};

namespace msbg {

// ---- kernels -----------------------------------------------------------------
struct LevelArgs {
    const int32_t* nbr;
    int lg;
    int64_t cells;
    float scale;
    const float* diag;  // per-cell diagonal (0: inactive cell), or null: 6 s, every cell active
};

// Sum of the 6 face neighbours of cell i (zero outside the active blocks),
// the value at cell index j given by get(j).
template <typename T, typename G>
__device__ __forceinline__ T nb_sum_of(const LevelArgs& L, int64_t i, G get) {
    const int bs = 1 << L.lg, m = bs - 1;
    const int64_t k = i >> (3 * L.lg);
    const int v = (int)(i & ((1 << (3 * L.lg)) - 1));
    const int cx = v & m, cy = (v >> L.lg) & m, cz = v >> (2 * L.lg);
    const int32_t* nb = L.nbr + k * 6;
    T s;
    {
        const int32_t kk = cx > 0 ? (int32_t)k : nb[0];
        s = kk >= 0 ? get(((int64_t)kk << (3 * L.lg)) + (v & ~m) + ((cx - 1) & m)) : T(0);
    }
    {
        const int32_t kk = cx < m ? (int32_t)k : nb[1];
        s += kk >= 0 ? get(((int64_t)kk << (3 * L.lg)) + (v & ~m) + ((cx + 1) & m)) : T(0);
    }
    {
        const int32_t kk = cy > 0 ? (int32_t)k : nb[2];
        s += kk >= 0 ? get(((int64_t)kk << (3 * L.lg)) + cx + (((cy - 1) & m) << L.lg) + (cz << (2 * L.lg))) : T(0);
    }
    {
        const int32_t kk = cy < m ? (int32_t)k : nb[3];
        s += kk >= 0 ? get(((int64_t)kk << (3 * L.lg)) + cx + (((cy + 1) & m) << L.lg) + (cz << (2 * L.lg))) : T(0);
    }
    {
        const int32_t kk = cz > 0 ? (int32_t)k : nb[4];
        s += kk >= 0 ? get(((int64_t)kk << (3 * L.lg)) + cx + (cy << L.lg) + (((cz - 1) & m) << (2 * L.lg))) : T(0);
    }
    {
        const int32_t kk = cz < m ? (int32_t)k : nb[5];
        s += kk >= 0 ? get(((int64_t)kk << (3 * L.lg)) + cx + (cy << L.lg) + (((cz + 1) & m) << (2 * L.lg))) : T(0);
    }
    return s;
}
template <typename T>
__device__ __forceinline__ T nb_sum(const LevelArgs& L, const T* __restrict__ x, int64_t i) {
    return nb_sum_of<T>(L, i, [x](int64_t j) { return x[j]; });
}

// y = A x
__global__ void pk_matvec(LevelArgs L, const float* __restrict__ x, float* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L.cells; i += (int64_t)gridDim.x * blockDim.x) {
        if (!L.diag) y[i] = L.scale * (6.0f * x[i] - nb_sum(L, x, i));
        else {
            const float d = L.diag[i];
            y[i] = d > 0.0f ? d * x[i] - L.scale * nb_sum(L, x, i) : 0.0f;
        }
    }
}

// r = b - A x (0 at inactive cells)
__global__ void pk_residual(LevelArgs L, const float* __restrict__ x, const float* __restrict__ b, float* __restrict__ r) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L.cells; i += (int64_t)gridDim.x * blockDim.x) {
        if (!L.diag) r[i] = b[i] - L.scale * (6.0f * x[i] - nb_sum(L, x, i));
        else {
            const float d = L.diag[i];
            r[i] = d > 0.0f ? b[i] - (d * x[i] - L.scale * nb_sum(L, x, i)) : 0.0f;
        }
    }
}

// r = b - A x with x in FP64 and the operator applied in FP64; r rounded to
// f32.  The solution of a solve accumulates in FP64: with an f32 solution the
// rounding of x alone leaves a relative residual of order 6 eps / lambda_min,
// about 1e-5 on thin shells, above the 1e-6 target.
__global__ void pk_residual64(LevelArgs L, const double* __restrict__ x, const float* __restrict__ b,
                              float* __restrict__ r) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L.cells; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = (float)((double)b[i] - (double)L.scale * (6.0 * x[i] - nb_sum(L, x, i)));
}

// x += a * d (x FP64, d f32)
__global__ void pk_add64(int64_t n, double a, const float* __restrict__ d, double* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] += a * (double)d[i];
}

__global__ void pk_widen(int64_t n, const float* __restrict__ s, double* __restrict__ d) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = (double)s[i];
}

__global__ void pk_narrow(int64_t n, const double* __restrict__ s, float* __restrict__ d) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = (float)s[i];
}

// One weighted Jacobi sweep: xn = w (b + s sum_nb x) / (6 s) + (1 - w) x.
// x == null means x = 0.
__global__ void pk_jacobi(LevelArgs L, const float* __restrict__ x, const float* __restrict__ b, float* __restrict__ xn,
                          float omega) {
    const float inv_d = 1.0f / (6.0f * L.scale);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L.cells; i += (int64_t)gridDim.x * blockDim.x) {
        if (!L.diag) {
            if (x) xn[i] = omega * (b[i] + L.scale * nb_sum(L, x, i)) * inv_d + (1.0f - omega) * x[i];
            else xn[i] = omega * b[i] * inv_d;
        } else {
            // inactive cells stay zero, so neighbour sums need no mask
            const float d = L.diag[i];
            if (!(d > 0.0f)) xn[i] = 0.0f;
            else if (x) xn[i] = omega * (b[i] + L.scale * nb_sum(L, x, i)) / d + (1.0f - omega) * x[i];
            else xn[i] = omega * b[i] / d;
        }
    }
}

// The first two weighted Jacobi sweeps from x = 0 in one pass: the first
// sweep's x1 = w b / (6 s) (w b / d with a diagonal; 0 at inactive cells) is
// formed where the second sweep reads it, with pk_jacobi's operations, so the
// result is the two sweeps' bits (x1's products rounded on their own, as
// when x1 is stored, not fused into the neighbour sum).
__global__ void pk_jacobi_zero2(LevelArgs L, const float* __restrict__ b, float* __restrict__ xn, float omega) {
    const float inv_d = 1.0f / (6.0f * L.scale);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L.cells; i += (int64_t)gridDim.x * blockDim.x) {
        if (!L.diag) {
            auto x1 = [&](int64_t j) { return __fmul_rn(__fmul_rn(omega, b[j]), inv_d); };
            xn[i] = omega * (b[i] + L.scale * nb_sum_of<float>(L, i, x1)) * inv_d + (1.0f - omega) * x1(i);
        } else {
            const float d = L.diag[i];
            auto x1 = [&](int64_t j) {
                const float dj = L.diag[j];
                return !(dj > 0.0f) ? 0.0f : __fdiv_rn(__fmul_rn(omega, b[j]), dj);
            };
            if (!(d > 0.0f)) xn[i] = 0.0f;
            else xn[i] = omega * (b[i] + L.scale * nb_sum_of<float>(L, i, x1)) / d + (1.0f - omega) * x1(i);
        }
    }
}

// The 7-point kernels on 16^3 blocks.  Both tile kernels add the neighbours
// x-1, x+1, y-1, y+1, z-1, z+1 in that order (zeros outside the active
// blocks, as nb_sum) and round every operation as written (no contraction),
// so every tile choice gives the same bits:
// OP 0: weighted Jacobi xn = w (b + s nb) / (6 s) + (1 - w) x (x null: the
// first sweep from zero); 1: residual r = b - s (6 x - nb); 2: y = s (6 x - nb);
// 3: OP 0 on x1 = w b / (6 s), the first sweep from zero formed from b where
// it is read (x is b): the first two sweeps from zero in one pass, bit for bit.
template <int OP>
__device__ __forceinline__ float op7(float sn, float cur, float bz, float scale, float omega, float inv_d) {
    if (OP == 0 || OP == 3)
        return __fadd_rn(__fmul_rn(__fmul_rn(omega, __fadd_rn(bz, __fmul_rn(scale, sn))), inv_d),
                         __fmul_rn(__fsub_rn(1.0f, omega), cur));
    if (OP == 1) return __fsub_rn(bz, __fmul_rn(scale, __fsub_rn(__fmul_rn(6.0f, cur), sn)));
    return __fmul_rn(scale, __fsub_rn(__fmul_rn(6.0f, cur), sn));
}
__device__ __forceinline__ float nb6(float xm, float xp, float ym, float yp, float zm, float zp) {
    float sn = xm;
    sn = __fadd_rn(sn, xp);
    sn = __fadd_rn(sn, ym);
    sn = __fadd_rn(sn, yp);
    sn = __fadd_rn(sn, zm);
    return __fadd_rn(sn, zp);
}

// Slab tile: one 256-thread CTA per slab of SLAB z-planes of a block (2, 4,
// 8 or 16: shorter dependent chains and more CTAs against more re-read slab
// boundaries).  Thread (x, y) walks its z-column with the planes below and
// above in registers (the next one prefetched), the current plane and its
// x/y halo from the face neighbours in shared memory.
template <int OP, int SLAB>
__global__ void __launch_bounds__(256) pk_block16(LevelArgs L, const float* __restrict__ x, const float* __restrict__ b,
                                                  float* __restrict__ out, float omega) {
    __shared__ float pl[18][18];
    __shared__ int32_t nb[6];
    const int64_t k = blockIdx.x / (16 / SLAB);
    const int z0 = (int)(blockIdx.x % (16 / SLAB)) * SLAB;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int col = tx + (ty << 4);
    const int64_t base = k << 12;
    const float inv_d = 1.0f / (6.0f * L.scale);
    if (OP == 0 && !x) {
        for (int z = z0; z < z0 + SLAB; ++z)
            out[base + col + (z << 8)] = __fmul_rn(__fmul_rn(omega, b[base + col + (z << 8)]), inv_d);
        return;
    }
    if (threadIdx.x < 6) nb[threadIdx.x] = L.nbr[k * 6 + threadIdx.x];
    __syncthreads();
    const int32_t nxm = nb[0], nxp = nb[1], nym = nb[2], nyp = nb[3], nzm = nb[4], nzp = nb[5];
    // the value the sweep reads at x[j]: x1 = w b inv_d for OP 3
    auto xv = [&](int64_t j) -> float { return OP == 3 ? __fmul_rn(__fmul_rn(omega, x[j]), inv_d) : x[j]; };
    auto plane = [&](int z) -> float {  // this column's value at plane z in [-1, 16]
        if (z < 0) return nzm >= 0 ? xv(((int64_t)nzm << 12) + col + (15 << 8)) : 0.0f;
        if (z > 15) return nzp >= 0 ? xv(((int64_t)nzp << 12) + col) : 0.0f;
        return xv(base + col + (z << 8));
    };
    float down = plane(z0 - 1), cur = plane(z0), up = plane(z0 + 1);
    for (int z = z0; z < z0 + SLAB; ++z) {
        const float upn = z + 2 <= 16 ? plane(z + 2) : 0.0f;
        const float bz = OP == 2 ? 0.0f : b[base + col + (z << 8)];
        pl[ty + 1][tx + 1] = cur;
        if (tx == 0) pl[ty + 1][0] = nxm >= 0 ? xv(((int64_t)nxm << 12) + 15 + (ty << 4) + (z << 8)) : 0.0f;
        if (tx == 15) pl[ty + 1][17] = nxp >= 0 ? xv(((int64_t)nxp << 12) + (ty << 4) + (z << 8)) : 0.0f;
        if (ty == 0) pl[0][tx + 1] = nym >= 0 ? xv(((int64_t)nym << 12) + tx + (15 << 4) + (z << 8)) : 0.0f;
        if (ty == 15) pl[17][tx + 1] = nyp >= 0 ? xv(((int64_t)nyp << 12) + tx + (z << 8)) : 0.0f;
        __syncthreads();
        const float sn = nb6(pl[ty + 1][tx], pl[ty + 1][tx + 2], pl[ty][tx + 1], pl[ty + 2][tx + 1], down, up);
        out[base + col + (z << 8)] = op7<OP>(sn, cur, bz, L.scale, omega, inv_d);
        __syncthreads();
        down = cur;
        cur = up;
        up = upn;
    }
}

// Quad tile: one 64-thread CTA per block; thread (q, y) owns the four
// x-consecutive cells 4q..4q+3 of row y and walks all 16 z-planes with the
// planes below and above in registers as float4 (plane z+2 loaded one step
// ahead), so each thread keeps two 16-byte loads in flight per plane.  The x
// neighbours come from the adjacent lanes of the row (shuffles) and, at the
// block's x faces, from the neighbour blocks; the y neighbours from a
// double-buffered shared plane whose halo rows the first and last row load
// from the y neighbour blocks.
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float comp(const float4& v, int e) { return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w; }

template <int OP>
__global__ void __launch_bounds__(64) pk_quad16(LevelArgs L, const float* __restrict__ x, const float* __restrict__ b,
                                                float* __restrict__ out, float omega) {
    __shared__ float4 pl[2][18][4];  // rows y = -1..16 of a plane, four quads each
    const int64_t k = blockIdx.x;
    const int q = threadIdx.x & 3, y = threadIdx.x >> 2;
    const int64_t base = k << 12;
    const int off = (y << 4) + (q << 2);
    const float inv_d = 1.0f / (6.0f * L.scale);
    if (OP == 0 && !x) {
        for (int z = 0; z < 16; ++z) {
            const float4 bv = ld4(b + base + off + (z << 8));
            *reinterpret_cast<float4*>(out + base + off + (z << 8)) =
                make_float4(__fmul_rn(__fmul_rn(omega, bv.x), inv_d), __fmul_rn(__fmul_rn(omega, bv.y), inv_d),
                            __fmul_rn(__fmul_rn(omega, bv.z), inv_d), __fmul_rn(__fmul_rn(omega, bv.w), inv_d));
        }
        return;
    }
    const int32_t* nbr = L.nbr + k * 6;
    const int32_t nxm = __ldg(nbr), nxp = __ldg(nbr + 1), nym = __ldg(nbr + 2), nyp = __ldg(nbr + 3), nzm = __ldg(nbr + 4),
                  nzp = __ldg(nbr + 5);
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    // the values the sweep reads: x1 = w b inv_d for OP 3
    auto tr = [&](float v) -> float { return OP == 3 ? __fmul_rn(__fmul_rn(omega, v), inv_d) : v; };
    auto xv4 = [&](const float* p) -> float4 {
        const float4 v = ld4(p);
        return make_float4(tr(v.x), tr(v.y), tr(v.z), tr(v.w));
    };
    auto plane = [&](int z) -> float4 {  // this thread's quad at plane z in [-1, 16]
        if (z < 0) return nzm >= 0 ? xv4(x + ((int64_t)nzm << 12) + off + (15 << 8)) : zero;
        if (z > 15) return nzp >= 0 ? xv4(x + ((int64_t)nzp << 12) + off) : zero;
        return xv4(x + base + off + (z << 8));
    };
    float4 down = plane(-1), cur = plane(0), up = plane(1);
    for (int z = 0; z < 16; ++z) {
        const int buf = z & 1;
        const float4 upn = z + 2 <= 16 ? plane(z + 2) : zero;
        const float4 bz = OP == 2 ? zero : ld4(b + base + off + (z << 8));
        const float xl = q == 0 && nxm >= 0 ? tr(x[((int64_t)nxm << 12) + 15 + (y << 4) + (z << 8)]) : 0.0f;
        const float xr = q == 3 && nxp >= 0 ? tr(x[((int64_t)nxp << 12) + (y << 4) + (z << 8)]) : 0.0f;
        pl[buf][y + 1][q] = cur;
        if (y == 0) pl[buf][0][q] = nym >= 0 ? xv4(x + ((int64_t)nym << 12) + (15 << 4) + (q << 2) + (z << 8)) : zero;
        if (y == 15) pl[buf][17][q] = nyp >= 0 ? xv4(x + ((int64_t)nyp << 12) + (q << 2) + (z << 8)) : zero;
        float lw = __shfl_up_sync(0xffffffffu, cur.w, 1);
        float rx = __shfl_down_sync(0xffffffffu, cur.x, 1);
        if (q == 0) lw = xl;
        if (q == 3) rx = xr;
        __syncthreads();  // one barrier per plane: the two buffers alternate
        const float4 ym = pl[buf][y][q], yp = pl[buf][y + 2][q];
        float r[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float xm = e == 0 ? lw : comp(cur, e - 1), xp = e == 3 ? rx : comp(cur, e + 1);
            const float sn = nb6(xm, xp, comp(ym, e), comp(yp, e), comp(down, e), comp(up, e));
            r[e] = op7<OP>(sn, comp(cur, e), comp(bz, e), L.scale, omega, inv_d);
        }
        *reinterpret_cast<float4*>(out + base + off + (z << 8)) = make_float4(r[0], r[1], r[2], r[3]);
        down = cur;
        cur = up;
        up = upn;
    }
}

// Cell-centred trilinear transfer weights along one axis: a fine cell takes
// 3/4 of its parent cell and 1/4 of the parent's neighbour on its side.
// Restriction is the transpose / 8: coarse cell q gathers fine cells
// 2q-1, 2q, 2q+1, 2q+2 with weights 1/4, 3/4, 3/4, 1/4 per axis.
struct TransferArgs {
    const int32_t* coords;  // [n][3] block coordinates of the level the kernel runs over
    const int32_t* nb;      // prolongation: [nf][27] coarse slots around the parent; restriction: [nc][64] fine slots
    const int32_t* pcoords; // prolongation: coarse block coordinates; restriction: unused
    const int32_t* parent;  // prolongation: [nf] parent slot
    const float* diag;      // the written level's diagonal (0: inactive cell) or null (all active)
    int lgf, lgc;
    int64_t cells;          // cells of the level the kernel runs over
};

__global__ void pk_restrict(TransferArgs T, const float* __restrict__ r, float* __restrict__ bc) {
    const int bsc = 1 << T.lgc, mc = bsc - 1, mf = (1 << T.lgf) - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < T.cells; i += (int64_t)gridDim.x * blockDim.x) {
        if (T.diag && !(T.diag[i] > 0.0f)) {
            bc[i] = 0.0f;
            continue;
        }
        const int64_t k = i >> (3 * T.lgc);
        const int v = (int)(i & ((1 << (3 * T.lgc)) - 1));
        const int q[3] = {T.coords[3 * k] * bsc + (v & mc), T.coords[3 * k + 1] * bsc + ((v >> T.lgc) & mc),
                          T.coords[3 * k + 2] * bsc + (v >> (2 * T.lgc))};
        int fb0[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) fb0[a] = ((2 * T.coords[3 * k + a] * bsc) >> T.lgf) - 1;
        const int32_t* nb = T.nb + k * 64;
        const float w1[4] = {0.25f, 0.75f, 0.75f, 0.25f};
        float s = 0.0f;
#pragma unroll
        for (int tz = 0; tz < 4; ++tz) {
            const int gz = 2 * q[2] - 1 + tz, bz = (gz >> T.lgf) - fb0[2];
#pragma unroll
            for (int ty = 0; ty < 4; ++ty) {
                const int gy = 2 * q[1] - 1 + ty, by = (gy >> T.lgf) - fb0[1];
                float row = 0.0f;
#pragma unroll
                for (int tx = 0; tx < 4; ++tx) {
                    const int gx = 2 * q[0] - 1 + tx, bx = (gx >> T.lgf) - fb0[0];
                    const int32_t sl = nb[bx + 4 * by + 16 * bz];
                    const float val = sl >= 0 ? r[((int64_t)sl << (3 * T.lgf)) + ((gx & mf) | ((gy & mf) << T.lgf) |
                                                                                   ((gz & mf) << (2 * T.lgf)))]
                                              : 0.0f;
                    row += w1[tx] * val;
                }
                s += (w1[ty] * w1[tz]) * row;
            }
        }
        bc[i] = s * 0.125f;
    }
}

// x_f += P x_c at the active fine cells.
__global__ void pk_prolong(TransferArgs T, const float* __restrict__ xc, float* __restrict__ xf) {
    const int bsf = 1 << T.lgf, mf = bsf - 1, mc = (1 << T.lgc) - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < T.cells; i += (int64_t)gridDim.x * blockDim.x) {
        if (T.diag && !(T.diag[i] > 0.0f)) continue;
        const int64_t k = i >> (3 * T.lgf);
        const int v = (int)(i & ((1 << (3 * T.lgf)) - 1));
        const int g[3] = {T.coords[3 * k] * bsf + (v & mf), T.coords[3 * k + 1] * bsf + ((v >> T.lgf) & mf),
                          T.coords[3 * k + 2] * bsf + (v >> (2 * T.lgf))};
        const int32_t pk = T.parent[k];
        int near[3], far[3], bn[3], bf[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            near[a] = g[a] >> 1;
            far[a] = near[a] + ((g[a] & 1) ? 1 : -1);
            const int pc = T.pcoords[3 * pk + a];
            bn[a] = (near[a] >> T.lgc) - pc + 1;
            bf[a] = (far[a] >> T.lgc) - pc + 1;
        }
        const int32_t* nb = T.nb + k * 27;
        float s = 0.0f;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int cx = (c & 1) ? far[0] : near[0], cy = (c & 2) ? far[1] : near[1], cz = (c & 4) ? far[2] : near[2];
            const int ix = (c & 1) ? bf[0] : bn[0], iy = (c & 2) ? bf[1] : bn[1], iz = (c & 4) ? bf[2] : bn[2];
            const int32_t sl = nb[ix + 3 * iy + 9 * iz];
            const float w = ((c & 1) ? 0.25f : 0.75f) * ((c & 2) ? 0.25f : 0.75f) * ((c & 4) ? 0.25f : 0.75f);
            if (sl >= 0) s += w * xc[((int64_t)sl << (3 * T.lgc)) + ((cx & mc) | ((cy & mc) << T.lgc) | ((cz & mc) << (2 * T.lgc)))];
        }
        xf[i] += s;
    }
}

// The transfers between two levels on one block grid (the fine block size
// twice the coarse one, coarse block k the parent of fine block k), one CTA
// per block: the block and a one-cell halo from its neighbours (zeros where
// a neighbour is absent) staged in shared memory, then pk_restrict's and
// pk_prolong's sums in the same order.
// NT threads a CTA; the staging loops are unrolled so that a thread's loads
// are in flight together.
template <int LGF, int NT>
__global__ void __launch_bounds__(NT) pk_restrict_tile(TransferArgs T, const float* __restrict__ r, float* __restrict__ bc) {
    constexpr int BF = 1 << LGF, BC = BF / 2, LGC = LGF - 1, W = BF + 2, NC = BC * BC * BC;
    __shared__ float f[W * W * W];  // fine cells -1 .. BF of the fine block under coarse block k
    __shared__ int32_t fs[27];
    const int64_t k = blockIdx.x;
    if (threadIdx.x < 27) {
        // fine block at offset (t % 3, t / 3 % 3, t / 9) - 1; the restriction table starts at offset -1
        const int t = threadIdx.x;
        fs[t] = T.nb[k * 64 + (t % 3) + 4 * ((t / 3) % 3) + 16 * (t / 9)];
    }
    __syncthreads();
#pragma unroll
    for (int e0 = 0; e0 < W * W * W; e0 += NT) {
        const int e = e0 + (int)threadIdx.x;
        if (e >= W * W * W) break;
        const int lx = e % W - 1, ly = (e / W) % W - 1, lz = e / (W * W) - 1;
        const int ox = lx < 0 ? 0 : lx >= BF ? 2 : 1, oy = ly < 0 ? 0 : ly >= BF ? 2 : 1, oz = lz < 0 ? 0 : lz >= BF ? 2 : 1;
        const int32_t sl = fs[ox + 3 * oy + 9 * oz];
        f[e] = sl >= 0 ? r[((int64_t)sl << (3 * LGF)) + ((lx & (BF - 1)) | ((ly & (BF - 1)) << LGF) | ((lz & (BF - 1)) << (2 * LGF)))]
                       : 0.0f;
    }
    __syncthreads();
    const float w1[4] = {0.25f, 0.75f, 0.75f, 0.25f};
    for (int v = threadIdx.x; v < NC; v += NT) {
        const int64_t i = (k << (3 * LGC)) + v;
        if (T.diag && !(T.diag[i] > 0.0f)) {
            bc[i] = 0.0f;
            continue;
        }
        const int qx = v & (BC - 1), qy = (v >> LGC) & (BC - 1), qz = v >> (2 * LGC);
        const float* fb = f + 2 * qx + W * (2 * qy + W * 2 * qz);  // fine cell 2q - 1 + t sits at window index 2q + t
        float s = 0.0f;
#pragma unroll
        for (int tz = 0; tz < 4; ++tz) {
#pragma unroll
            for (int ty = 0; ty < 4; ++ty) {
                float row = 0.0f;
#pragma unroll
                for (int tx = 0; tx < 4; ++tx) row += w1[tx] * fb[tx + W * (ty + W * tz)];
                s += (w1[ty] * w1[tz]) * row;
            }
        }
        bc[i] = s * 0.125f;
    }
}

template <int LGF, int NT>
__global__ void __launch_bounds__(NT) pk_prolong_tile(TransferArgs T, const float* __restrict__ xc, float* __restrict__ xf) {
    constexpr int BF = 1 << LGF, BC = BF / 2, LGC = LGF - 1, W = BC + 2, NF = BF * BF * BF;
    __shared__ float c[W * W * W];  // coarse cells -1 .. BC of fine block k's parent
    __shared__ int32_t cs[27];
    const int64_t k = blockIdx.x;
    if (threadIdx.x < 27) cs[threadIdx.x] = T.nb[k * 27 + threadIdx.x];
    __syncthreads();
#pragma unroll
    for (int e0 = 0; e0 < W * W * W; e0 += NT) {
        const int e = e0 + (int)threadIdx.x;
        if (e >= W * W * W) break;
        const int lx = e % W - 1, ly = (e / W) % W - 1, lz = e / (W * W) - 1;
        const int ox = lx < 0 ? 0 : lx >= BC ? 2 : 1, oy = ly < 0 ? 0 : ly >= BC ? 2 : 1, oz = lz < 0 ? 0 : lz >= BC ? 2 : 1;
        const int32_t sl = cs[ox + 3 * oy + 9 * oz];
        c[e] = sl >= 0 ? xc[((int64_t)sl << (3 * LGC)) + ((lx & (BC - 1)) | ((ly & (BC - 1)) << LGC) | ((lz & (BC - 1)) << (2 * LGC)))]
                       : 0.0f;
    }
    __syncthreads();
#pragma unroll 4
    for (int v = threadIdx.x; v < NF; v += NT) {
        const int64_t i = (k << (3 * LGF)) + v;
        if (T.diag && !(T.diag[i] > 0.0f)) continue;
        const int g[3] = {v & (BF - 1), (v >> LGF) & (BF - 1), v >> (2 * LGF)};
        int near[3], far[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            near[a] = g[a] >> 1;
            far[a] = near[a] + ((g[a] & 1) ? 1 : -1);
        }
        float s = 0.0f;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int cx = (q & 1) ? far[0] : near[0], cy = (q & 2) ? far[1] : near[1], cz = (q & 4) ? far[2] : near[2];
            const float w = ((q & 1) ? 0.25f : 0.75f) * ((q & 2) ? 0.25f : 0.75f) * ((q & 4) ? 0.25f : 0.75f);
            s += w * c[(cx + 1) + W * ((cy + 1) + W * (cz + 1))];
        }
        xf[i] += s;
    }
}

// x_c = A^-1 b_c with the FP64 inverse, one warp per row.  The inverse of
// the symmetric operator is symmetric, so row i is column i: its n entries
// are contiguous and the warp reads them coalesced.  Lane partial sums are
// combined in a fixed butterfly order (deterministic).
__global__ void pk_dense_solve(const double* __restrict__ ainv, int64_t n, const float* __restrict__ b, float* __restrict__ x) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const double* row = ainv + i * n;
        double s = 0.0;
        for (int64_t j = lane; j < n; j += 32) s += row[j] * (double)b[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) x[i] = (float)s;
    }
}

// FP64 dot product, stage 1: per-CTA partial sums (fixed tree order).
constexpr int DOT_THREADS = 256;
constexpr int DOT_BLOCKS = 1184;  // 8 per SM

__global__ void __launch_bounds__(DOT_THREADS) pk_dot_partial(const float* __restrict__ a, const float* __restrict__ b,
                                                               int64_t n, double* __restrict__ partial) {
    __shared__ double sm[DOT_THREADS];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)DOT_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * DOT_THREADS)
        s += (double)a[i] * (double)b[i];
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int o = DOT_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

__global__ void __launch_bounds__(DOT_THREADS) pk_dot_final(const double* __restrict__ partial, int np, double* __restrict__ out) {
    __shared__ double sm[DOT_THREADS];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += DOT_THREADS) s += partial[i];
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int o = DOT_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sm[0];
}

// y = a*x + b*y (f32 vectors, scalars from FP64)
__global__ void pk_axpby(int64_t n, float a, const float* __restrict__ x, float b, float* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = a * x[i] + b * y[i];
}

// CG scalars kept on the device between kernels (one host read per iteration):
// sc[SC_RZ] = r.z, sc[SC_PQ] = p.Ap, sc[SC_ALPHA], sc[SC_RR] = r.r,
// sc[SC_RZ2] = the new r.z, sc[SC_ZR] = z.r_old (flexible CG), sc[SC_BETA],
// sc[SC_BAD] != 0 when p.Ap <= 0 or r.z is not finite (the updates below are
// then skipped and the host restarts or stops).
enum { SC_RZ, SC_PQ, SC_ALPHA, SC_RR, SC_RZ2, SC_ZR, SC_BETA, SC_BAD, SC_COUNT };

// Stage 2 of p.Ap (the same tree as pk_dot_final), then alpha = r.z / p.Ap.
__global__ void __launch_bounds__(DOT_THREADS) pk_dot_final_alpha(const double* __restrict__ partial, int np,
                                                                   double* __restrict__ sc) {
    __shared__ double sm[DOT_THREADS];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += DOT_THREADS) s += partial[i];
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int o = DOT_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double pq = sm[0], rz = sc[SC_RZ];
        const bool bad = !(pq > 0.0) || !isfinite(rz);
        sc[SC_PQ] = pq;
        sc[SC_BAD] = bad ? 1.0 : 0.0;
        sc[SC_ALPHA] = bad ? 0.0 : rz / pq;
    }
}

// x += alpha p (FP64) and r = (-alpha) q + r (f32) as fused multiply-adds,
// skipped on breakdown.
__global__ void pk_cg_update(int64_t n, const double* __restrict__ sc, const float* __restrict__ p,
                             const float* __restrict__ q, double* __restrict__ x, float* __restrict__ r) {
    if (sc[SC_BAD] != 0.0) return;
    const double a = sc[SC_ALPHA];
    const float na = (float)-a;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] = fma(a, (double)p[i], x[i]);
        r[i] = fmaf(na, q[i], r[i]);
    }
}

// beta = r.z_new / r.z (or (r.z_new - z.r_old) / r.z for flexible CG); r.z = r.z_new.
__global__ void pk_cg_beta(double* __restrict__ sc, int flexible) {
    const double rz2 = sc[SC_RZ2];
    sc[SC_BETA] = flexible ? (rz2 - sc[SC_ZR]) / sc[SC_RZ] : rz2 / sc[SC_RZ];
    sc[SC_RZ] = rz2;
}

// p = z + beta p (f32; beta from the device; the product rounded, then the sum)
__global__ void pk_cg_direction(int64_t n, const double* __restrict__ sc, const float* __restrict__ z,
                                float* __restrict__ p) {
    const float b = (float)sc[SC_BETA];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = __fadd_rn(z[i], __fmul_rn(b, p[i]));
}

// ---- host side -----------------------------------------------------------------
static unsigned grid_for(int64_t n) { return (unsigned)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 16); }

// Launch shapes the autotuner chooses from for the cell-parallel level kernels
// (grid-stride loops): threads per CTA and the grid cap in CTAs per SM.
struct LaunchShape {
    int threads, ctas_per_sm;
};
constexpr LaunchShape kShapes[] = {{256, 16}, {128, 16}, {512, 4}, {256, 4}, {128, 32}, {1024, 2}, {64, 32}, {256, 8}};
constexpr int kNumShapes = (int)(sizeof(kShapes) / sizeof(kShapes[0]));

static dim3 shape_grid(int cfg, int64_t n) {
    const LaunchShape& S = kShapes[cfg];
    return dim3((unsigned)std::min<int64_t>(std::max<int64_t>((n + S.threads - 1) / S.threads, 1), 148LL * S.ctas_per_sm));
}

static LevelArgs level_args(const PLevelDev& L) {
    return LevelArgs{L.nbr.as<int32_t>(), L.lg, L.cells(), L.scale, L.diag.p ? L.diag.as<float>() : nullptr};
}

// Control block of a captured solve loop: iterations run, the limit, the
// stopping threshold tol |b| and |b|.
struct SolveCtl {
    long long it, max_iter;
    double thr, bn;
};

// The test at the end of a captured solve iteration: counts it, records
// |r| / |b| and keeps the loop running while |r| > tol |b|, the limit is not
// reached and (check_bad) CG saw no breakdown.  One thread.
__global__ void pk_solve_test(cudaGraphConditionalHandle h, const double* __restrict__ sc, SolveCtl* __restrict__ c,
                              double* __restrict__ hist, int check_bad) {
    const long long it = c->it + 1;
    c->it = it;
    const double rn = sqrt(sc[SC_RR]);
    hist[it - 1] = rn / c->bn;
    const bool bad = check_bad && sc[SC_BAD] != 0.0;
    cudaGraphSetConditional(h, (rn > c->thr && it < c->max_iter && !bad) ? 1u : 0u);
}

static void upload(msbg_ctx* ctx, DevBuf& d, const void* h, size_t bytes) {
    d.reserve(std::max<size_t>(bytes, 16));
    if (bytes) CUDA_CHECK(cudaMemcpyAsync(d.p, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
}

static void build(msbg_poisson* P, uint64_t sx, uint64_t sy, uint64_t sz, int bsx, const uint64_t* active, size_t n_active,
                  int max_grid_halvings = 1 << 30) {
    msbg_ctx* ctx = P->ctx;
    const uint64_t nx = (sx + bsx - 1) / bsx, ny = (sy + bsx - 1) / bsx, nz = (sz + bsx - 1) / bsx;
    std::vector<uint64_t> a(active, active + n_active);
    for (uint64_t b : a) MSBG_REQUIRE(b < nx * ny * nz, "active block id out of range");
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
    MSBG_REQUIRE(!a.empty(), "empty active set");
    P->lv.clear();
    P->lv.emplace_back();
    {
        PLevelDev& L = P->lv.back();
        L.bs = bsx; L.lg = ilog2i(bsx); L.nx = nx; L.ny = ny; L.nz = nz; L.scale = 1.0f; L.bids = a;
    }
    int halvings = 0;
    while (P->lv.back().cells() > kPoissonDirect) {
        const PLevelDev& F = P->lv.back();
        if (F.bs < 4 && halvings >= max_grid_halvings) break;
        PLevelDev C;
        C.scale = F.scale * 0.25f;
        if (F.bs >= 4) {
            C.bs = F.bs / 2; C.nx = F.nx; C.ny = F.ny; C.nz = F.nz; C.bids = F.bids;
        } else {
            ++halvings;
            C.bs = F.bs; C.nx = (F.nx + 1) / 2; C.ny = (F.ny + 1) / 2; C.nz = (F.nz + 1) / 2;
            for (uint64_t b : F.bids) {
                uint64_t bx = b % F.nx, by = (b / F.nx) % F.ny, bz = b / (F.nx * F.ny);
                C.bids.push_back((bx >> 1) + (by >> 1) * C.nx + (bz >> 1) * C.nx * C.ny);
            }
            std::sort(C.bids.begin(), C.bids.end());
            C.bids.erase(std::unique(C.bids.begin(), C.bids.end()), C.bids.end());
        }
        C.lg = ilog2i(C.bs);
        P->lv.push_back(std::move(C));
    }
    const size_t nl = P->lv.size();
    std::vector<std::unordered_map<uint64_t, int32_t>> slot(nl);
    std::vector<std::vector<int32_t>> coords(nl), nbr(nl);
    for (size_t l = 0; l < nl; ++l) {
        PLevelDev& L = P->lv[l];
        for (int64_t k = 0; k < L.n(); ++k) slot[l][L.bids[k]] = (int32_t)k;
        nbr[l].assign((size_t)L.n() * 6, -1);
        coords[l].resize((size_t)L.n() * 3);
        for (int64_t k = 0; k < L.n(); ++k) {
            const int64_t b = (int64_t)L.bids[k], bx = b % L.nx, by = (b / L.nx) % L.ny, bz = b / (L.nx * L.ny);
            coords[l][3 * k] = (int32_t)bx; coords[l][3 * k + 1] = (int32_t)by; coords[l][3 * k + 2] = (int32_t)bz;
            const int64_t d[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
            for (int f = 0; f < 6; ++f) {
                const int64_t X2 = bx + d[f][0], Y2 = by + d[f][1], Z2 = bz + d[f][2];
                if (X2 < 0 || Y2 < 0 || Z2 < 0 || X2 >= L.nx || Y2 >= L.ny || Z2 >= L.nz) continue;
                auto it = slot[l].find((uint64_t)(X2 + Y2 * L.nx + Z2 * L.nx * L.ny));
                if (it != slot[l].end()) nbr[l][6 * k + f] = it->second;
            }
        }
        upload(ctx, L.nbr, nbr[l].data(), nbr[l].size() * 4);
        upload(ctx, L.coords, coords[l].data(), coords[l].size() * 4);
        const size_t cb = (size_t)L.cells() * 4;
        L.x.reserve(cb); L.b.reserve(cb); L.r.reserve(cb); L.t.reserve(cb);
    }
    // slot of the level-l block at block coordinates (X, Y, Z), or -1
    auto slot_at = [&](size_t l, int64_t X, int64_t Y, int64_t Z) -> int32_t {
        const PLevelDev& L = P->lv[l];
        if (X < 0 || Y < 0 || Z < 0 || X >= L.nx || Y >= L.ny || Z >= L.nz) return -1;
        auto it = slot[l].find((uint64_t)(X + Y * L.nx + Z * L.nx * L.ny));
        return it == slot[l].end() ? -1 : it->second;
    };
    // cell masks (a coarse cell is active when any of its 8 children is) and
    // diagonals s_l (6 - g_l m)
    std::vector<std::vector<uint8_t>> mask(nl);
    std::vector<std::vector<float>> diag(nl);
    for (size_t l = 0; l < nl; ++l) {
        const PLevelDev& L = P->lv[l];
        const int bs = L.bs, m = bs - 1;
        const int64_t N = (int64_t)bs * bs * bs;
        mask[l].assign((size_t)L.cells(), 1);
        if (l > 0) {
            const PLevelDev& F = P->lv[l - 1];
            const int mf = F.bs - 1;
            const bool same_grid = F.bs == 2 * L.bs;  // same block grid: the children of block k are in fine block k
            for (int64_t k = 0; k < L.n(); ++k)
                for (int64_t v = 0; v < N; ++v) {
                    const int64_t q[3] = {coords[l][3 * k] * (int64_t)bs + (v & m), coords[l][3 * k + 1] * (int64_t)bs + ((v >> L.lg) & m),
                                          coords[l][3 * k + 2] * (int64_t)bs + (v >> (2 * L.lg))};
                    const int32_t fs = same_grid ? (int32_t)k
                                                 : slot_at(l - 1, (2 * q[0]) >> F.lg, (2 * q[1]) >> F.lg, (2 * q[2]) >> F.lg);
                    uint8_t a = 0;
                    if (fs >= 0)
                        for (int c = 0; c < 8; ++c) {
                            const int64_t gx = 2 * q[0] + (c & 1), gy = 2 * q[1] + ((c >> 1) & 1), gz = 2 * q[2] + (c >> 2);
                            a |= mask[l - 1][(size_t)fs * F.bs * F.bs * F.bs + ((gx & mf) | ((gy & mf) << F.lg) | ((gz & mf) << (2 * F.lg)))];
                        }
                    mask[l][(size_t)(k * N + v)] = a;
                }
        }
        if (l == 0) continue;
        const double dd = 0.5 + std::ldexp(1.0, -(int)l - 1);
        const double ghost = 1.0 - 1.0 / dd;
        diag[l].assign((size_t)L.cells(), 0.0f);
        for (int64_t k = 0; k < L.n(); ++k)
            for (int64_t v = 0; v < N; ++v) {
                if (!mask[l][(size_t)(k * N + v)]) continue;
                const int c[3] = {(int)(v & m), (int)((v >> L.lg) & m), (int)(v >> (2 * L.lg))};
                int miss = 0;
                for (int f = 0; f < 6; ++f) {
                    int cc[3] = {c[0], c[1], c[2]};
                    cc[f / 2] += (f & 1) ? 1 : -1;
                    int32_t kk = (int32_t)k;
                    if (cc[f / 2] < 0 || cc[f / 2] > m) {
                        kk = nbr[l][6 * k + f];
                        cc[f / 2] &= m;
                    }
                    if (kk < 0 || !mask[l][(size_t)kk * N + (cc[0] | (cc[1] << L.lg) | (cc[2] << (2 * L.lg)))]) ++miss;
                }
                diag[l][(size_t)(k * N + v)] = (float)((double)L.scale * (6.0 - ghost * miss));
            }
        upload(ctx, P->lv[l].diag, diag[l].data(), diag[l].size() * 4);
    }
    // transfer tables
    for (size_t l = 0; l + 1 < nl; ++l) {
        PLevelDev& L = P->lv[l];
        const PLevelDev& C = P->lv[l + 1];
        std::vector<int32_t> parent(L.n()), pnb((size_t)L.n() * 27);
        for (int64_t k = 0; k < L.n(); ++k) {
            const int64_t bx = coords[l][3 * k], by = coords[l][3 * k + 1], bz = coords[l][3 * k + 2];
            const int64_t cbx = (bx * L.bs / 2) / C.bs, cby = (by * L.bs / 2) / C.bs, cbz = (bz * L.bs / 2) / C.bs;
            parent[k] = slot_at(l + 1, cbx, cby, cbz);
            MSBG_REQUIRE(parent[k] >= 0, "Poisson hierarchy: a block without a parent");
            for (int o = 0; o < 27; ++o) pnb[(size_t)k * 27 + o] = slot_at(l + 1, cbx + o % 3 - 1, cby + (o / 3) % 3 - 1, cbz + o / 9 - 1);
        }
        upload(ctx, L.parent, parent.data(), parent.size() * 4);
        upload(ctx, L.pnb, pnb.data(), pnb.size() * 4);
        std::vector<int32_t> rnb((size_t)C.n() * 64);
        for (int64_t k = 0; k < C.n(); ++k) {
            int64_t fb0[3];
            for (int a = 0; a < 3; ++a) fb0[a] = ((2 * (int64_t)coords[l + 1][3 * k + a] * C.bs) >> L.lg) - 1;
            for (int o = 0; o < 64; ++o) rnb[(size_t)k * 64 + o] = slot_at(l, fb0[0] + (o & 3), fb0[1] + ((o >> 2) & 3), fb0[2] + (o >> 4));
        }
        upload(ctx, P->lv[l + 1].rnb, rnb.data(), rnb.size() * 4);
    }
    sync(ctx);  // host tables die at scope end
    // dense FP64 inverse of the coarsest operator (inactive cells: identity rows)
    const PLevelDev& C = P->lv.back();
    const int64_t n = C.cells();
    MSBG_REQUIRE(n <= 4 * kPoissonDirect, "coarsest level too large for the dense solve (too many batched problems)");
    P->nc = n;
    std::vector<double> A((size_t)n * n, 0.0);
    {
        const size_t lc = nl - 1;
        const int bs = C.bs, m = bs - 1;
        const int64_t N = (int64_t)bs * bs * bs;
        for (int64_t k = 0; k < C.n(); ++k)
            for (int64_t v = 0; v < N; ++v) {
                const int64_t i = k * N + v;
                if (!mask[lc][(size_t)i]) {
                    A[(size_t)i * n + i] = 1.0;
                    continue;
                }
                A[(size_t)i * n + i] = lc == 0 ? 6.0 * C.scale : (double)diag[lc][(size_t)i];
                const int c[3] = {(int)(v & m), (int)((v >> C.lg) & m), (int)(v >> (2 * C.lg))};
                for (int f = 0; f < 6; ++f) {
                    int cc[3] = {c[0], c[1], c[2]};
                    cc[f / 2] += (f & 1) ? 1 : -1;
                    int32_t kk = (int32_t)k;
                    if (cc[f / 2] < 0 || cc[f / 2] > m) {
                        kk = nbr[lc][6 * k + f];
                        cc[f / 2] &= m;
                    }
                    if (kk < 0) continue;
                    const int64_t j = (int64_t)kk * N + (cc[0] | (cc[1] << C.lg) | (cc[2] << (2 * C.lg)));
                    if (mask[lc][(size_t)j]) A[(size_t)i * n + j] = -1.0 * C.scale;
                }
            }
    }
    // Cholesky A = L L^T, then the inverse column by column
    for (int64_t j = 0; j < n; ++j) {
        double d = A[(size_t)j * n + j];
        for (int64_t k = 0; k < j; ++k) d -= A[(size_t)j * n + k] * A[(size_t)j * n + k];
        MSBG_REQUIRE(d > 0.0, "coarsest Poisson operator is not positive definite");
        d = std::sqrt(d);
        A[(size_t)j * n + j] = d;
        for (int64_t i = j + 1; i < n; ++i) {
            double s = A[(size_t)i * n + j];
            for (int64_t k = 0; k < j; ++k) s -= A[(size_t)i * n + k] * A[(size_t)j * n + k];
            A[(size_t)i * n + j] = s / d;
        }
    }
    std::vector<double> inv((size_t)n * n), y(n), e(n);
    for (int64_t c = 0; c < n; ++c) {
        for (int64_t i = 0; i < n; ++i) {
            double s = (i == c) ? 1.0 : 0.0;
            for (int64_t k = 0; k < i; ++k) s -= A[(size_t)i * n + k] * y[k];
            y[i] = s / A[(size_t)i * n + i];
        }
        for (int64_t i = n - 1; i >= 0; --i) {
            double s = y[i];
            for (int64_t k = i + 1; k < n; ++k) s -= A[(size_t)k * n + i] * e[k];
            e[i] = s / A[(size_t)i * n + i];
        }
        for (int64_t i = 0; i < n; ++i) inv[(size_t)c * n + i] = e[i];  // column c (symmetric)
    }
    upload(ctx, P->ainv, inv.data(), inv.size() * 8);
    const int64_t n0 = P->lv[0].cells();
    P->work.reserve((size_t)n0 * (7 * 4 + 8) + (DOT_BLOCKS + 16) * 8 + 1024);
    sync(ctx);
}

// tile: 1 = the quad tile (one 64-thread CTA per block), 2, 4, 8, 16 = the
// slab tile with that many z-planes per 256-thread CTA.
template <int OP>
static void launch_block16(msbg_ctx* ctx, const PLevelDev& L, int slab, const float* x, const float* b, float* out,
                           float omega) {
    const LevelArgs a = level_args(L);
    if (slab == 1) {
        pk_quad16<OP><<<(unsigned)L.n(), 64, 0, ctx->stream>>>(a, x, b, out, omega);
        return;
    }
    const unsigned grid = (unsigned)(L.n() * (16 / slab));
    switch (slab) {
        case 2: pk_block16<OP, 2><<<grid, 256, 0, ctx->stream>>>(a, x, b, out, omega); break;
        case 8: pk_block16<OP, 8><<<grid, 256, 0, ctx->stream>>>(a, x, b, out, omega); break;
        case 16: pk_block16<OP, 16><<<grid, 256, 0, ctx->stream>>>(a, x, b, out, omega); break;
        default: pk_block16<OP, 4><<<(unsigned)(L.n() * 4), 256, 0, ctx->stream>>>(a, x, b, out, omega); break;
    }
}
static bool uses_block16(const PLevelDev& L) { return L.lg == 4 && !L.diag.p; }

static void launch_matvec(msbg_poisson* P, int l, const float* x, float* y) {
    const PLevelDev& L = P->lv[l];
    begin_launch(P->ctx);
    if (uses_block16(L)) {
        launch_block16<2>(P->ctx, L, L.slab, x, nullptr, y, 0.0f);
        after_launch(P->ctx, "pk_block16_matvec");
        return;
    }
    pk_matvec<<<grid_for(L.cells()), 256, 0, P->ctx->stream>>>(level_args(L), x, y);
    after_launch(P->ctx, "pk_matvec");
}

static void launch_residual(msbg_poisson* P, int l, const float* x, const float* b, float* r) {
    const PLevelDev& L = P->lv[l];
    begin_launch(P->ctx);
    if (uses_block16(L)) {
        launch_block16<1>(P->ctx, L, L.slab, x, b, r, 0.0f);
        after_launch(P->ctx, "pk_block16_residual");
        return;
    }
    pk_residual<<<shape_grid(L.cfg_res, L.cells()), kShapes[L.cfg_res].threads, 0, P->ctx->stream>>>(level_args(L), x, b, r);
    after_launch(P->ctx, "pk_residual");
}

// `sweeps` Jacobi sweeps on x (in place through the level's t buffer); x_zero
// marks x as all zeros on entry.
static void jacobi(msbg_poisson* P, int l, float* x, const float* b, int sweeps, float omega, bool x_zero) {
    PLevelDev& L = P->lv[l];
    float* t = L.t.as<float>();
    int s = 0;
    if (x_zero && sweeps >= 2) {
        // the first two sweeps from zero in one pass, into x (where the second sweep writes)
        begin_launch(P->ctx);
        if (uses_block16(L)) {
            launch_block16<3>(P->ctx, L, L.slab, b, b, x, omega);
            after_launch(P->ctx, "pk_block16_jacobi0");
        } else {
            pk_jacobi_zero2<<<shape_grid(L.cfg_jac, L.cells()), kShapes[L.cfg_jac].threads, 0, P->ctx->stream>>>(
                level_args(L), b, x, omega);
            after_launch(P->ctx, "pk_jacobi_zero2");
        }
        s = 2;
    }
    for (; s < sweeps; ++s) {
        const float* src = (s % 2 == 0) ? x : t;
        float* dst = (s % 2 == 0) ? t : x;
        begin_launch(P->ctx);
        if (uses_block16(L)) {
            launch_block16<0>(P->ctx, L, L.slab, (s == 0 && x_zero) ? nullptr : src, b, dst, omega);
            after_launch(P->ctx, "pk_block16_jacobi");
            continue;
        }
        pk_jacobi<<<shape_grid(L.cfg_jac, L.cells()), kShapes[L.cfg_jac].threads, 0, P->ctx->stream>>>(
            level_args(L), (s == 0 && x_zero) ? nullptr : src, b, dst, omega);
        after_launch(P->ctx, "pk_jacobi");
    }
    if (sweeps % 2 == 1) CUDA_CHECK(cudaMemcpyAsync(x, t, L.cells() * 4, cudaMemcpyDeviceToDevice, P->ctx->stream));
}

// One V-cycle on level l: x_l improved for A_l x_l = b_l (x_zero: x_l = 0 on entry).
static void vcycle(msbg_poisson* P, int l, float* x, const float* b, bool x_zero) {
    if (l == (int)P->lv.size() - 1) {
        begin_launch(P->ctx);
        pk_dense_solve<<<grid_for(P->nc * 32), 256, 0, P->ctx->stream>>>(P->ainv.as<double>(), P->nc, b, x);
        after_launch(P->ctx, "pk_dense_solve");
        return;
    }
    PLevelDev& F = P->lv[l];
    PLevelDev& C = P->lv[l + 1];
    jacobi(P, l, x, b, P->nu1, P->omega, x_zero);
    launch_residual(P, l, x, b, F.r.as<float>());
    // the fine block size twice the coarse one: coarse block k is fine block k's parent
    const bool same_grid = F.bs == 2 * C.bs && F.lg >= 2 && F.lg <= 4;
    TransferArgs R{C.coords.as<int32_t>(), C.rnb.as<int32_t>(), nullptr, nullptr, C.diag.as<float>(), F.lg, C.lg, C.cells()};
    begin_launch(P->ctx);
    if (same_grid) {
        const unsigned nb = (unsigned)C.n();
        if (F.lg == 4) pk_restrict_tile<4, 256><<<nb, 256, 0, P->ctx->stream>>>(R, F.r.as<float>(), C.b.as<float>());
        else if (F.lg == 3) pk_restrict_tile<3, 128><<<nb, 128, 0, P->ctx->stream>>>(R, F.r.as<float>(), C.b.as<float>());
        else pk_restrict_tile<2, 64><<<nb, 64, 0, P->ctx->stream>>>(R, F.r.as<float>(), C.b.as<float>());
        after_launch(P->ctx, "pk_restrict_tile");
    } else {
        pk_restrict<<<grid_for(C.cells()), 256, 0, P->ctx->stream>>>(R, F.r.as<float>(), C.b.as<float>());
        after_launch(P->ctx, "pk_restrict");
    }
    vcycle(P, l + 1, C.x.as<float>(), C.b.as<float>(), true);
    TransferArgs T{F.coords.as<int32_t>(), F.pnb.as<int32_t>(), C.coords.as<int32_t>(), F.parent.as<int32_t>(),
                   F.diag.p ? F.diag.as<float>() : nullptr, F.lg, C.lg, F.cells()};
    begin_launch(P->ctx);
    if (same_grid) {
        const unsigned nb = (unsigned)F.n();
        if (F.lg == 4) pk_prolong_tile<4, 256><<<nb, 256, 0, P->ctx->stream>>>(T, C.x.as<float>(), x);
        else if (F.lg == 3) pk_prolong_tile<3, 256><<<nb, 256, 0, P->ctx->stream>>>(T, C.x.as<float>(), x);
        else pk_prolong_tile<2, 64><<<nb, 64, 0, P->ctx->stream>>>(T, C.x.as<float>(), x);
        after_launch(P->ctx, "pk_prolong_tile");
    } else {
        pk_prolong<<<grid_for(F.cells()), 256, 0, P->ctx->stream>>>(T, C.x.as<float>(), x);
        after_launch(P->ctx, "pk_prolong");
    }
    jacobi(P, l, x, b, P->nu2, P->omega, false);
}

static double dot(msbg_poisson* P, const float* a, const float* b, int64_t n) {
    double* part = (double*)((char*)P->work.p + P->work.bytes - (DOT_BLOCKS + 16) * 8);
    begin_launch(P->ctx);
    pk_dot_partial<<<DOT_BLOCKS, DOT_THREADS, 0, P->ctx->stream>>>(a, b, n, part);
    after_launch(P->ctx, "pk_dot_partial");
    begin_launch(P->ctx);
    pk_dot_final<<<1, DOT_THREADS, 0, P->ctx->stream>>>(part, DOT_BLOCKS, part + DOT_BLOCKS);
    after_launch(P->ctx, "pk_dot_final");
    double h = 0.0;
    read_small(P->ctx, &h, part + DOT_BLOCKS, 8);
    return h;
}

// The CG scalar block (SC_COUNT doubles after the dot partials and result).
static double* cg_scalars(msbg_poisson* P) {
    return (double*)((char*)P->work.p + P->work.bytes - (DOT_BLOCKS + 16) * 8) + DOT_BLOCKS + 2;
}

// a.b into sc[slot] on the device (no host read); SC_PQ also sets alpha.
static void dot_dev(msbg_poisson* P, const float* a, const float* b, int64_t n, int slot) {
    double* part = (double*)((char*)P->work.p + P->work.bytes - (DOT_BLOCKS + 16) * 8);
    double* sc = cg_scalars(P);
    begin_launch(P->ctx);
    pk_dot_partial<<<DOT_BLOCKS, DOT_THREADS, 0, P->ctx->stream>>>(a, b, n, part);
    after_launch(P->ctx, "pk_dot_partial");
    begin_launch(P->ctx);
    if (slot == SC_PQ) {
        pk_dot_final_alpha<<<1, DOT_THREADS, 0, P->ctx->stream>>>(part, DOT_BLOCKS, sc);
        after_launch(P->ctx, "pk_dot_final_alpha");
    } else {
        pk_dot_final<<<1, DOT_THREADS, 0, P->ctx->stream>>>(part, DOT_BLOCKS, sc + slot);
        after_launch(P->ctx, "pk_dot_final");
    }
}

// Host copy of the CG scalar block (waits for the stream).
static void read_scalars(msbg_poisson* P, double* h) { read_small(P->ctx, h, cg_scalars(P), SC_COUNT * 8); }

static void axpby(msbg_poisson* P, int64_t n, double a, const float* x, double b, float* y) {
    begin_launch(P->ctx);
    pk_axpby<<<grid_for(n), 256, 0, P->ctx->stream>>>(n, (float)a, x, (float)b, y);
    after_launch(P->ctx, "pk_axpby");
}

static void launch_residual64(msbg_poisson* P, const double* x, const float* b, float* r) {
    const PLevelDev& L = P->lv[0];
    begin_launch(P->ctx);
    pk_residual64<<<grid_for(L.cells()), 256, 0, P->ctx->stream>>>(level_args(L), x, b, r);
    after_launch(P->ctx, "pk_residual64");
}

static void add64(msbg_poisson* P, int64_t n, double a, const float* d, double* x) {
    begin_launch(P->ctx);
    pk_add64<<<grid_for(n), 256, 0, P->ctx->stream>>>(n, a, d, x);
    after_launch(P->ctx, "pk_add64");
}

// A V-cycle from level 0 with x = 0 on entry, launched as a captured graph
// (captured on the first use of each (x, b) pair).  With per-kernel timing
// on, the launches go to the stream one by one so that each is timed.
static void vcycle_top(msbg_poisson* P, float* x, const float* b) {
    msbg_ctx* ctx = P->ctx;
    if (ctx->timing) {
        vcycle(P, 0, x, b, true);
        return;
    }
    msbg_poisson::VGraph* g = nullptr;
    for (auto& v : P->vgraphs)
        if (v.x == x && v.b == b) g = &v;
    if (!g) {
        const uint64_t l0 = ctx->launches;
        cudaGraph_t graph = nullptr;
        CUDA_CHECK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        try {
            vcycle(P, 0, x, b, true);
        } catch (...) {
            cudaStreamEndCapture(ctx->stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            ctx->launches = l0;
            throw;
        }
        CUDA_CHECK(cudaStreamEndCapture(ctx->stream, &graph));
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) MSBG_THROW(MSBG_ERR_CUDA, std::string("V-cycle graph: ") + cudaGetErrorString(e));
        P->vgraphs.push_back({x, b, exec, (int)(ctx->launches - l0)});
        ctx->launches = l0;
        g = &P->vgraphs.back();
    }
    CUDA_CHECK(cudaGraphLaunch(g->exec, ctx->stream));
    ctx->launches += (uint64_t)g->kernels;
}

// Releases the captured V-cycles and solve loops: they bake in the smoother
// parameters, the launch shapes and the buffers.
static void drop_graphs(msbg_poisson* P) {
    if (P->vgraphs.empty() && P->sgraphs.empty()) return;
    sync(P->ctx);
    for (auto& g : P->vgraphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto& g : P->sgraphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    P->vgraphs.clear();
    P->sgraphs.clear();
}

// Iterations of method 0 (z = V r, x += z, r = b - A x) or of method 1 (MG-
// PCG from a restart: z = V r, p = z, then CG steps) in one graph launch: a
// device-side while loop whose test (pk_solve_test) ends every iteration, so
// the host waits once instead of once per iteration.  The kernels and their
// order are those of the host loop in solve().  Captured on the first use of
// each (method, b, x64).  Returns the iterations the launch ran; sc_out gets
// the CG scalar block after it.
static int solve_loop(msbg_poisson* P, int method, const float* b, double* x64, float* r, float* z, float* p, float* q,
                      long long it0, long long max_iter, double thr, double bn, double* sc_out) {
    msbg_ctx* ctx = P->ctx;
    const int64_t n = P->lv[0].cells();
    if (P->shist.bytes < (size_t)max_iter * 8) {
        drop_graphs(P);  // the graphs bake in the history buffer
        P->shist.reserve((size_t)max_iter * 8);
    }
    if (!P->sctl.p) P->sctl.reserve(sizeof(SolveCtl));
    double* sc = cg_scalars(P);
    SolveCtl* ctl = P->sctl.as<SolveCtl>();
    double* hist = P->shist.as<double>();
    msbg_poisson::SGraph* g = nullptr;
    for (auto& v : P->sgraphs)
        if (v.method == method && v.b == b && v.x64 == x64) g = &v;
    if (!g) {
        auto cg_step = [&](cudaGraphConditionalHandle h) {  // q = A p, alpha, x += alpha p, r -= alpha q, r.r, test
            launch_matvec(P, 0, p, q);
            dot_dev(P, p, q, n, SC_PQ);
            begin_launch(ctx);
            pk_cg_update<<<grid_for(n), 256, 0, ctx->stream>>>(n, sc, p, q, x64, r);
            after_launch(ctx, "pk_cg_update");
            dot_dev(P, r, r, n, SC_RR);
            begin_launch(ctx);
            pk_solve_test<<<1, 1, 0, ctx->stream>>>(h, sc, ctl, hist, 1);
            after_launch(ctx, "pk_solve_test");
        };
        cudaGraph_t G = nullptr;
        CUDA_CHECK(cudaGraphCreate(&G, 0));
        const uint64_t l0 = ctx->launches;
        bool capturing = false;
        int k_first = 0, k_body = 0;
        cudaGraphExec_t exec = nullptr;
        try {
            // method 0 enters the loop at once (the host has tested |r|);
            // method 1 runs the restart and its first CG step before the loop
            cudaGraphConditionalHandle h;
            CUDA_CHECK(cudaGraphConditionalHandleCreate(&h, G, method == 0 ? 1u : 0u,
                                                        method == 0 ? cudaGraphCondAssignDefault : 0u));
            cudaGraphNode_t tail = nullptr;
            if (method == 1) {
                CUDA_CHECK(cudaStreamBeginCaptureToGraph(ctx->stream, G, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
                capturing = true;
                vcycle(P, 0, z, r, true);
                CUDA_CHECK(cudaMemcpyAsync(p, z, n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
                dot_dev(P, r, z, n, SC_RZ);
                cg_step(h);
                CUDA_CHECK(cudaStreamEndCapture(ctx->stream, &G));
                capturing = false;
                k_first = (int)(ctx->launches - l0);
                // the captured chain's last node
                size_t nn = 0;
                CUDA_CHECK(cudaGraphGetNodes(G, nullptr, &nn));
                std::vector<cudaGraphNode_t> nodes(nn);
                CUDA_CHECK(cudaGraphGetNodes(G, nodes.data(), &nn));
                for (cudaGraphNode_t nd : nodes) {
                    size_t nout = 0;
                    CUDA_CHECK(cudaGraphNodeGetDependentNodes(nd, nullptr, &nout));
                    if (nout == 0) tail = nd;
                }
                MSBG_REQUIRE(tail != nullptr, "captured solve: no last node");
            }
            cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t loop_node;
            CUDA_CHECK(cudaGraphAddNode(&loop_node, G, tail ? &tail : nullptr, tail ? 1 : 0, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            const uint64_t l1 = ctx->launches;
            CUDA_CHECK(cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            capturing = true;
            vcycle(P, 0, z, r, true);
            if (method == 0) {
                add64(P, n, 1.0, z, x64);
                launch_residual64(P, x64, b, r);
                dot_dev(P, r, r, n, SC_RR);
                begin_launch(ctx);
                pk_solve_test<<<1, 1, 0, ctx->stream>>>(h, sc, ctl, hist, 0);
                after_launch(ctx, "pk_solve_test");
            } else {
                dot_dev(P, r, z, n, SC_RZ2);
                begin_launch(ctx);
                pk_cg_beta<<<1, 1, 0, ctx->stream>>>(sc, 0);
                after_launch(ctx, "pk_cg_beta");
                begin_launch(ctx);
                pk_cg_direction<<<grid_for(n), 256, 0, ctx->stream>>>(n, sc, z, p);
                after_launch(ctx, "pk_cg_direction");
                cg_step(h);
            }
            CUDA_CHECK(cudaStreamEndCapture(ctx->stream, &body));
            capturing = false;
            k_body = (int)(ctx->launches - l1);
            CUDA_CHECK(cudaGraphInstantiate(&exec, G, 0));
        } catch (...) {
            if (capturing) {
                cudaGraph_t tmp = nullptr;
                cudaStreamEndCapture(ctx->stream, &tmp);
            }
            cudaGraphDestroy(G);
            ctx->launches = l0;
            throw;
        }
        cudaGraphDestroy(G);
        ctx->launches = l0;
        P->sgraphs.push_back({method, b, x64, exec, k_first, k_body});
        g = &P->sgraphs.back();
    }
    const SolveCtl c0{it0, max_iter, thr, bn};
    CUDA_CHECK(cudaMemcpyAsync(ctl, &c0, sizeof(c0), cudaMemcpyHostToDevice, ctx->stream));
    CUDA_CHECK(cudaGraphLaunch(g->exec, ctx->stream));
    SolveCtl c1;
    {
        SmallReads rd(ctx);
        rd.add(&c1, ctl, sizeof(c1));
        rd.add(sc_out, sc, SC_COUNT * 8);
        rd.wait();
    }
    const int ran = (int)(c1.it - it0);
    // method 1: the first iteration is the part before the loop
    ctx->launches += (uint64_t)g->kernels_first + (uint64_t)(method == 1 ? ran - 1 : ran) * (uint64_t)g->kernels_body;
    return ran;
}

// Relative residuals of iterations [from, to) of the last captured solve loop.
static void loop_history(msbg_poisson* P, double* hist, long long from, long long to) {
    if (hist && to > from) read_small(P->ctx, hist + from, P->shist.as<double>() + from, (size_t)(to - from) * 8);
}

// Preconditioners of the CG solve.
enum { PC_MG = 0, PC_NET = 1, PC_HYBRID = 2 };

// z += V (r - A z).  The network's correction leaves high-frequency error
// that the operator amplifies in the residual; a V-cycle on the residual
// equation removes that.
static void post_smooth(msbg_poisson* P, float* z, const float* r, float* s, float* u) {
    const int64_t n = P->lv[0].cells();
    launch_residual(P, 0, z, r, s);
    vcycle_top(P, u, s);
    axpby(P, n, 1.0, u, 1.0, z);
}

// z = V r, then the network's correction of the remaining error,
// z += N(r - A z), then post_smooth (V-cycle, network, V-cycle).
static void learned_cycle(msbg_poisson* P, float* z, const float* r, float* s, float* u, bool post = true) {
    const int64_t n = P->lv[0].cells();
    vcycle_top(P, z, r);
    launch_residual(P, 0, z, r, s);
    unet_apply(P->net, s, u);
    axpby(P, n, 1.0, u, 1.0, z);
    if (post) post_smooth(P, z, r, s, u);
}

// method 0: V-cycles (x += V(b - A x)); 1: MG-preconditioned CG; 2: flexible
// CG preconditioned by the learned network; 3: flexible CG preconditioned by
// a V-cycle plus the network's correction of the V-cycle's remaining error,
// z = V r + N(r - A V r); 5: method 3's preconditioner for the first
// net_lead applications (where the network removes most error per cost),
// then CG restarted from the current iterate with V-cycles.  Methods 2, 3
// and 5 fall back to the V-cycle
// preconditioner (and restart) when the residual stalls (three iterations in
// a row without a 5 % decrease) or a search direction loses positivity.  The
// solution accumulates in FP64 and convergence is judged on the true
// residual b - A x of that FP64 solution; CG's recursively updated residual
// is replaced by the true one when it reaches the tolerance (and the
// iteration restarts from it if the true residual is still above).  Returns
// iterations.
static int solve(msbg_poisson* P, int method, float* x, const float* b, double tol, int max_iter, double* rel_out,
                 double* hist, double* x64_ext = nullptr) {
    PLevelDev& F = P->lv[0];
    const int64_t n = F.cells();
    float* r = (float*)P->work.p;
    float* z = r + n;
    float* p = z + n;
    float* q = p + n;
    double* x64 = x64_ext ? x64_ext : (double*)(q + n);
    float* r_old = (float*)((double*)(q + n) + n);
    float* sv = r_old + n;
    float* uv = sv + n;
    P->n_net = P->n_vcycle = P->fell_back = 0;
    P->fallback_iter = -1;
    if (method >= 2) MSBG_REQUIRE(P->net != nullptr, "learned preconditioner not set (msbg_poisson_set_preconditioner)");
    if (method == 5 && P->net_lead <= 0) method = 1;
    const double bn = std::sqrt(dot(P, b, b, n));
    if (bn == 0.0) {
        if (x64_ext) CUDA_CHECK(cudaMemsetAsync(x64_ext, 0, n * 8, P->ctx->stream));
        else CUDA_CHECK(cudaMemsetAsync(x, 0, n * 4, P->ctx->stream));
        if (rel_out) *rel_out = 0.0;
        return 0;
    }
    if (!x64_ext) {
        begin_launch(P->ctx);
        pk_widen<<<grid_for(n), 256, 0, P->ctx->stream>>>(n, x, x64);
        after_launch(P->ctx, "pk_widen");
    }
    launch_residual64(P, x64, b, r);
    double rn = std::sqrt(dot(P, r, r, n));
    int it = 0;
    if (method == 0 || method == 4) {
        // stationary iteration x += M r with M = V (method 0) or the hybrid
        // M r = V r + N(r - A V r) (method 4); the learned one falls back to
        // V when an iteration fails to halve the residual
        bool learned = method == 4;
        double rn_prev = rn;
        if (method == 0 && !P->ctx->timing && rn > tol * bn && it < max_iter) {
            double hs[SC_COUNT];
            it = solve_loop(P, 0, b, x64, r, z, nullptr, nullptr, 0, max_iter, tol * bn, bn, hs);
            P->n_vcycle += it;
            loop_history(P, hist, 0, it);
            rn = std::sqrt(hs[SC_RR]);
            if (!std::isfinite(rn)) MSBG_THROW(MSBG_ERR_NUMERIC, "multigrid residual is not finite");
        }
        while (rn > tol * bn && it < max_iter) {
            if (learned) {
                learned_cycle(P, z, r, sv, uv);
                P->n_net++;
                P->n_vcycle++;
            } else {
                vcycle_top(P, z, r);
            }
            P->n_vcycle++;
            add64(P, n, 1.0, z, x64);
            launch_residual64(P, x64, b, r);
            rn = std::sqrt(dot(P, r, r, n));
            if (!std::isfinite(rn)) MSBG_THROW(MSBG_ERR_NUMERIC, "multigrid residual is not finite");
            if (hist) hist[it] = rn / bn;
            ++it;
            if (learned && rn > 0.5 * rn_prev) {
                learned = false;
                P->fell_back = 1;
                P->fallback_iter = it;
            }
            rn_prev = rn;
        }
    } else {
        int pc = method == 1 ? PC_MG : (method == 2 ? PC_NET : PC_HYBRID);
        bool flexible = method >= 2;
        const int lead = method == 5 ? P->net_lead : -1;
        auto precondition = [&](const float* rr, float* zz) {
            if (pc == PC_MG) {
                vcycle_top(P, zz, rr);
                P->n_vcycle++;
            } else if (pc == PC_NET) {
                unet_apply(P->net, rr, zz);
                post_smooth(P, zz, rr, sv, uv);
                P->n_net++;
                P->n_vcycle++;
            } else {
                const bool post = !(lead > 0 && P->net_lead_post == 0);
                learned_cycle(P, zz, rr, sv, uv, post);
                P->n_vcycle += post ? 2 : 1;
                P->n_net++;
            }
        };
        double rz = 0.0;
        double* sc = cg_scalars(P);
        double hs[SC_COUNT];
        auto restart = [&]() {
            precondition(r, z);
            CUDA_CHECK(cudaMemcpyAsync(p, z, n * 4, cudaMemcpyDeviceToDevice, P->ctx->stream));
            dot_dev(P, r, z, n, SC_RZ);
            read_scalars(P, hs);
            rz = hs[SC_RZ];
        };
        int since = 0;  // iterations since the last (re)start
        std::vector<double> rn_hist;
        auto fall_back = [&](int reason) {
            pc = PC_MG;
            P->fell_back = reason;
            P->fallback_iter = it;
            restart();
            since = 0;
        };
        rn_hist.push_back(rn);  // the window below always holds the start
        // MG-PCG from a restart at the current iterate as captured loops: a
        // restart and CG steps until |r| <= tol |b|, the limit or a
        // breakdown; then the host loop's checks
        auto captured_mg_pcg = [&]() {
            while (rn > tol * bn && it < max_iter) {
                const int ran = solve_loop(P, 1, b, x64, r, z, p, q, it, max_iter, tol * bn, bn, hs);
                P->n_vcycle += ran;
                loop_history(P, hist, it, it + ran);
                it += ran;
                if (hs[SC_BAD] != 0.0) MSBG_THROW(MSBG_ERR_NUMERIC, "PCG breakdown (p.Ap <= 0)");
                rn = std::sqrt(hs[SC_RR]);
                if (rn <= tol * bn) {
                    // the true residual decides; above tol the loop restarts from it
                    launch_residual64(P, x64, b, r);
                    rn = std::sqrt(dot(P, r, r, n));
                    if (hist) hist[it - 1] = rn / bn;
                }
            }
        };
        if (method == 1 && !P->ctx->timing) {
            captured_mg_pcg();
        } else {
            restart();
            if (flexible && !(rz > 0.0)) fall_back(3);
            while (rn > tol * bn && it < max_iter) {
                // q = A p, alpha = r.z / p.Ap, x += alpha p, r -= alpha q and r.r
                // run back to back on the device; the host reads the scalars once
                launch_matvec(P, 0, p, q);
                dot_dev(P, p, q, n, SC_PQ);
                if (flexible) CUDA_CHECK(cudaMemcpyAsync(r_old, r, n * 4, cudaMemcpyDeviceToDevice, P->ctx->stream));
                begin_launch(P->ctx);
                pk_cg_update<<<grid_for(n), 256, 0, P->ctx->stream>>>(n, sc, p, q, x64, r);
                after_launch(P->ctx, "pk_cg_update");
                dot_dev(P, r, r, n, SC_RR);
                read_scalars(P, hs);
                if (hs[SC_BAD] != 0.0) {  // p.Ap <= 0: x and r were left as they were
                    if (flexible && pc != PC_MG) {
                        fall_back(2);
                        continue;
                    }
                    MSBG_THROW(MSBG_ERR_NUMERIC, "PCG breakdown (p.Ap <= 0)");
                }
                rn = std::sqrt(hs[SC_RR]);
                ++it;
                if (rn <= tol * bn) {
                    launch_residual64(P, x64, b, r);
                    rn = std::sqrt(dot(P, r, r, n));
                    if (hist) hist[it - 1] = rn / bn;
                    if (rn <= tol * bn) break;
                    restart();
                    since = 0;
                    continue;
                }
                if (hist) hist[it - 1] = rn / bn;
                rn_hist.push_back(rn);
                ++since;
                // stall: the residual norm of CG is not monotone, so the test is
                // over a window: less than a halving in the last 4 iterations
                if (flexible && pc != PC_MG && since >= 4 && rn > 0.5 * rn_hist[rn_hist.size() - 5]) {
                    fall_back(1);
                    continue;
                }
                if (lead > 0 && pc == PC_HYBRID && P->n_net >= lead) {
                    // method 5: the lead is over; CG restarts from the current
                    // iterate with the fixed V-cycle preconditioner
                    pc = PC_MG;
                    flexible = false;
                    if (!P->ctx->timing) {
                        captured_mg_pcg();
                        break;
                    }
                    restart();
                    since = 0;
                    continue;
                }
                precondition(r, z);
                dot_dev(P, r, z, n, SC_RZ2);
                if (flexible) dot_dev(P, z, r_old, n, SC_ZR);
                begin_launch(P->ctx);
                pk_cg_beta<<<1, 1, 0, P->ctx->stream>>>(sc, flexible ? 1 : 0);
                after_launch(P->ctx, "pk_cg_beta");
                if (flexible && pc != PC_MG) {
                    read_scalars(P, hs);
                    if (!(hs[SC_RZ] > 0.0)) {  // the new r.z
                        fall_back(3);
                        continue;
                    }
                }
                begin_launch(P->ctx);
                pk_cg_direction<<<grid_for(n), 256, 0, P->ctx->stream>>>(n, sc, z, p);
                after_launch(P->ctx, "pk_cg_direction");
            }
        }
    }
    if (!x64_ext) {
        begin_launch(P->ctx);
        pk_narrow<<<grid_for(n), 256, 0, P->ctx->stream>>>(n, x64, x);
        after_launch(P->ctx, "pk_narrow");
    }
    if (rel_out) *rel_out = rn / bn;
    return it;
}

// ---- training data: solver-generated (residual, multigrid error) pairs -------
// Right-hand side of the learned-preconditioner workload on the device: the
// divergence of u = sum_i a_i exp(-|x - c_i|^2 / (2 s_i^2)), evaluated at
// level-0 cell centres: b = sum_i -(a_i . (x - c_i)) / s_i^2 g_i(x).
// blobs: [n_blobs][7] = (cx, cy, cz, s, ax, ay, az).
__global__ void pk_blob_rhs(LevelArgs L, const int32_t* __restrict__ coords, const float* __restrict__ blobs, int n_blobs,
                            float* __restrict__ bout) {
    const int bs = 1 << L.lg, m = bs - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L.cells; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i >> (3 * L.lg);
        const int v = (int)(i & ((1 << (3 * L.lg)) - 1));
        const double px = coords[3 * k] * bs + (v & m) + 0.5, py = coords[3 * k + 1] * bs + ((v >> L.lg) & m) + 0.5,
                     pz = coords[3 * k + 2] * bs + (v >> (2 * L.lg)) + 0.5;
        double acc = 0.0;
        for (int j = 0; j < n_blobs; ++j) {
            const float* B = blobs + 7 * j;
            const double dx = px - B[0], dy = py - B[1], dz = pz - B[2], s2 = (double)B[3] * B[3];
            const double g = exp(-(dx * dx + dy * dy + dz * dz) / (2.0 * s2));
            acc += -(B[4] * dx + B[5] * dy + B[6] * dz) / s2 * g;
        }
        bout[i] = (float)acc;
    }
}

// e = xs - x (FP64 in, f32 out)
__global__ void pk_sub64(int64_t n, const double* __restrict__ xs, const double* __restrict__ x, float* __restrict__ e) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        e[i] = (float)(xs[i] - x[i]);
}

// Fills b with the smooth-divergence right-hand side of random seed `seed`.
static void blob_rhs(msbg_poisson* P, uint64_t seed, int n_blobs, float* b, DevBuf& blob_buf) {
    PLevelDev& F = P->lv[0];
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int64_t> pick_block(0, F.n() - 1);
    std::uniform_real_distribution<double> u01(0.0, 1.0);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<float> blobs((size_t)n_blobs * 7);
    for (int j = 0; j < n_blobs; ++j) {
        const uint64_t bid = F.bids[pick_block(rng)];
        const double bx = (double)(bid % F.nx), by = (double)((bid / F.nx) % F.ny), bz = (double)(bid / (F.nx * F.ny));
        blobs[7 * j + 0] = (float)((bx + u01(rng)) * F.bs);
        blobs[7 * j + 1] = (float)((by + u01(rng)) * F.bs);
        blobs[7 * j + 2] = (float)((bz + u01(rng)) * F.bs);
        blobs[7 * j + 3] = (float)(4.0 + 12.0 * u01(rng));
        for (int a = 0; a < 3; ++a) blobs[7 * j + 4 + a] = (float)nd(rng);
    }
    blob_buf.reserve(blobs.size() * 4);
    CUDA_CHECK(cudaMemcpyAsync(blob_buf.p, blobs.data(), blobs.size() * 4, cudaMemcpyHostToDevice, P->ctx->stream));
    begin_launch(P->ctx);
    pk_blob_rhs<<<grid_for(F.cells()), 256, 0, P->ctx->stream>>>(level_args(F), F.coords.as<int32_t>(),
                                                                  blob_buf.as<float>(), n_blobs, b);
    after_launch(P->ctx, "pk_blob_rhs");
    sync(P->ctx);  // the host blob table dies at scope end
}

// Training of the learned preconditioner on pairs the solver generates: for
// each right-hand side, x* from MG-preconditioned CG to 1e-7, then plain
// multigrid from zero; after V-cycle k the pair is (residual r_k, error
// x* - x_k), or with target 1 the pair the hybrid preconditioner needs
// (s_k = r_k - A V r_k, x* - x_k - V r_k).  Pairs go to a pool of `pool`
// slots on the device; after each right-hand side, `steps_per_rhs` Adam
// steps train on pool slots drawn at random.  out_scale is set from the
// first right-hand side's pairs (mean rms(error) / rms(residual)).
struct TrainStats {
    int64_t steps = 0, pairs = 0;
};

static TrainStats train(msbg_poisson* P, int n_rhs, int mg_iters, int steps_per_rhs, int pool, float lr, int target,
                        uint64_t seed, double* loss_hist, int64_t hist_cap, int source = 0) {
    MSBG_REQUIRE(P->net, "learned preconditioner not set");
    PLevelDev& F = P->lv[0];
    const int64_t n = F.cells();
    msbg_ctx* ctx = P->ctx;
    DevBuf bbuf, xs, xk, blobs, pairs;
    bbuf.reserve(n * 4);
    xs.reserve(n * 8);
    xk.reserve(n * 8);
    pairs.reserve((size_t)pool * 2 * n * 4);
    float* b = bbuf.as<float>();
    float* r = (float*)P->work.p;  // solve() scratch, free between solves
    float* z = r + n;
    float* t = z + n;
    std::mt19937_64 rng(seed ^ 0x5eedULL);
    int64_t filled = 0, next = 0;
    TrainStats st;
    double scale_sum = 0.0;
    int scale_cnt = 0;
    for (int i = 0; i < n_rhs; ++i) {
        blob_rhs(P, seed * 1000003ULL + (uint64_t)i, 32, b, blobs);
        // reference solution
        float* xf = (float*)P->work.p + 6 * n;  // uv slot as the f32 solution
        CUDA_CHECK(cudaMemsetAsync(xf, 0, n * 4, ctx->stream));
        solve(P, 1, xf, b, 1e-7, 500, nullptr, nullptr);
        double* x64 = (double*)((float*)P->work.p + 4 * n);
        CUDA_CHECK(cudaMemcpyAsync(xs.p, x64, n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_CHECK(cudaMemsetAsync(xk.p, 0, n * 8, ctx->stream));
        // source 1: the iterates of MG-preconditioned CG (residuals as CG sees
        // them; r is updated recursively, p and q live in the pool's scratch)
        float* pv = t;
        float* qv = t + n;
        double rz = 0.0;
        if (source == 1) {
            launch_residual64(P, xk.as<double>(), b, r);
            vcycle(P, 0, z, r, true);
            CUDA_CHECK(cudaMemcpyAsync(pv, z, n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
            rz = dot(P, r, z, n);
        }
        for (int k = 0; k < mg_iters; ++k) {
            if (source == 0) launch_residual64(P, xk.as<double>(), b, r);
            float* pr = pairs.as<float>() + (size_t)next * 2 * n;
            float* pe = pr + n;
            begin_launch(ctx);
            pk_sub64<<<grid_for(n), 256, 0, ctx->stream>>>(n, xs.as<double>(), xk.as<double>(), pe);
            after_launch(ctx, "pk_sub64");
            vcycle(P, 0, z, r, true);  // z = V r
            if (target == 0) {
                CUDA_CHECK(cudaMemcpyAsync(pr, r, n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
            } else {
                launch_residual(P, 0, z, r, pr);  // s = r - A V r
                axpby(P, n, -1.0, z, 1.0, pe);    // e - V r
            }
            if (i == 0) {
                const double a = dot(P, pe, pe, n), c = dot(P, pr, pr, n);
                if (c > 0.0 && a > 0.0) {
                    scale_sum += std::sqrt(a / c);
                    scale_cnt++;
                }
            }
            if (source == 0) {
                add64(P, n, 1.0, z, xk.as<double>());
            } else {
                launch_matvec(P, 0, pv, qv);
                const double pq = dot(P, pv, qv, n);
                if (pq > 0.0 && rz > 0.0) {
                    const double alpha = rz / pq;
                    add64(P, n, alpha, pv, xk.as<double>());
                    axpby(P, n, -alpha, qv, 1.0, r);
                    vcycle(P, 0, z, r, true);
                    const double rz2 = dot(P, r, z, n);
                    axpby(P, n, 1.0, z, rz2 / rz, pv);
                    rz = rz2;
                }
            }
            next = (next + 1) % pool;
            filled = std::min<int64_t>(filled + 1, pool);
            st.pairs++;
        }
        if (i == 0 && scale_cnt) {
            (void)t;
            MSBG_REQUIRE(std::isfinite(scale_sum / scale_cnt), "non-finite output scale");
            msbg_unet_set_output_scale(P->net, (float)(scale_sum / scale_cnt));
        }
        std::uniform_int_distribution<int64_t> pick(0, std::max<int64_t>(filled - 1, 0));
        for (int s = 0; s < steps_per_rhs && filled > 0; ++s) {
            const int64_t j = pick(rng);
            const float* pr = pairs.as<float>() + (size_t)j * 2 * n;
            const double l = unet_train_step(P->net, pr, pr + n, lr, true);
            if (loss_hist && st.steps < hist_cap) loss_hist[st.steps] = l;
            st.steps++;
        }
    }
    sync(ctx);
    return st;
}

// Mean relative L2 error over fresh pairs (seed `seed`) of: the network
// alone N(r) against e, one V-cycle V r against e, and the hybrid V r +
// N(r - A V r) against e.
static void evaluate(msbg_poisson* P, int n_rhs, int mg_iters, uint64_t seed, double out[3]) {
    PLevelDev& F = P->lv[0];
    const int64_t n = F.cells();
    msbg_ctx* ctx = P->ctx;
    DevBuf bbuf, xs, xk, blobs, ebuf, tmp;
    bbuf.reserve(n * 4);
    xs.reserve(n * 8);
    xk.reserve(n * 8);
    ebuf.reserve(n * 4);
    tmp.reserve(n * 4 * 3);
    float* b = bbuf.as<float>();
    float* e = ebuf.as<float>();
    float* zn = tmp.as<float>();
    float* zv = zn + n;
    float* sres = zv + n;
    double acc[3] = {0, 0, 0};
    int cnt = 0;
    for (int i = 0; i < n_rhs; ++i) {
        blob_rhs(P, seed * 1000003ULL + (uint64_t)i, 32, b, blobs);
        float* xf = (float*)P->work.p + 6 * n;
        CUDA_CHECK(cudaMemsetAsync(xf, 0, n * 4, ctx->stream));
        solve(P, 1, xf, b, 1e-7, 500, nullptr, nullptr);
        CUDA_CHECK(cudaMemcpyAsync(xs.p, (double*)((float*)P->work.p + 4 * n), n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_CHECK(cudaMemsetAsync(xk.p, 0, n * 8, ctx->stream));
        float* r = (float*)P->work.p;
        for (int k = 0; k < mg_iters; ++k) {
            launch_residual64(P, xk.as<double>(), b, r);
            begin_launch(ctx);
            pk_sub64<<<grid_for(n), 256, 0, ctx->stream>>>(n, xs.as<double>(), xk.as<double>(), e);
            after_launch(ctx, "pk_sub64");
            const double en = std::sqrt(dot(P, e, e, n));
            vcycle(P, 0, zv, r, true);
            unet_apply(P->net, r, zn);
            axpby(P, n, -1.0, e, 1.0, zn);  // N r - e
            acc[0] += std::sqrt(dot(P, zn, zn, n)) / en;
            launch_residual(P, 0, zv, r, sres);
            unet_apply(P->net, sres, zn);
            axpby(P, n, 1.0, zv, 1.0, zn);   // V r + N(s)
            axpby(P, n, -1.0, e, 1.0, zn);
            acc[2] += std::sqrt(dot(P, zn, zn, n)) / en;
            axpby(P, n, -1.0, e, 1.0, zv);   // V r - e
            acc[1] += std::sqrt(dot(P, zv, zv, n)) / en;
            // advance the plain multigrid iterate
            vcycle(P, 0, zv, r, true);
            add64(P, n, 1.0, zv, xk.as<double>());
            ++cnt;
        }
    }
    for (int j = 0; j < 3; ++j) out[j] = cnt ? acc[j] / cnt : 0.0;
}

// ---- batched solves ------------------------------------------------------------
// Many independent problems share one hierarchy: problem p's blocks are
// placed at block z offset Z_p of a common virtual domain, with gaps of
// 2^(L+1) blocks (L = the block-grid halvings the hierarchy may make), so no
// two problems touch at any level and every operator is block-diagonal over
// the problems.  Blocks sort by z first, so each problem owns a contiguous
// range of every level's blocks.  CG runs with per-problem scalars kept on
// the device (no host round trip inside an iteration), which lets a whole
// cycle of iterations be captured into one CUDA graph.
enum { S_RZ = 0, S_PQ, S_RZN, S_RR, S_BB, S_ALPHA, S_BETA, S_ACTIVE, S_ITER, S_WIDTH = 16 };

// per-block FP64 partial of a . b (one CTA per block, fixed tree order)
__global__ void __launch_bounds__(256) bk_block_dot(int64_t nblocks, int cells, const float* __restrict__ a,
                                                    const float* __restrict__ b, double* __restrict__ part) {
    __shared__ double sm[256];
    for (int64_t k = blockIdx.x; k < nblocks; k += gridDim.x) {
        double s = 0.0;
        for (int i = threadIdx.x; i < cells; i += 256) s += (double)a[k * cells + i] * (double)b[k * cells + i];
        sm[threadIdx.x] = s;
        __syncthreads();
        for (int o = 128; o > 0; o >>= 1) {
            if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[k] = sm[0];
        __syncthreads();
    }
}

// scal[p][slot] = sum of the partials of problem p's blocks (one warp per problem)
__global__ void bk_seg_sum(int np, const int64_t* __restrict__ pb, const double* __restrict__ part, double* __restrict__ scal,
                           int slot) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < np; p += warps) {
        double s = 0.0;
        for (int64_t k = pb[p] + lane; k < pb[p + 1]; k += 32) s += part[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) scal[(int64_t)p * S_WIDTH + slot] = s;
    }
}

// op 0: alpha = rz / pq; op 1: beta = rz_new / rz, rz = rz_new, one more
// iteration counted; op 2: active = (r.r > tol^2 b.b).  Problems that are not
// active get alpha = beta = 0 and stay where they are.
__global__ void bk_scalars(int np, double* __restrict__ scal, int op, double tol2) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
        double* S = scal + (int64_t)p * S_WIDTH;
        const bool on = S[S_ACTIVE] > 0.0;
        if (op == 0) {
            S[S_ALPHA] = (on && S[S_PQ] > 0.0) ? S[S_RZ] / S[S_PQ] : 0.0;
        } else if (op == 1) {
            S[S_BETA] = (on && S[S_RZ] > 0.0) ? S[S_RZN] / S[S_RZ] : 0.0;
            S[S_RZ] = S[S_RZN];
            if (on) S[S_ITER] += 1.0;
        } else {
            S[S_ACTIVE] = S[S_RR] > tol2 * S[S_BB] ? 1.0 : 0.0;
        }
    }
}

// y += sign * s_p x  (s_p = scal[problem of the cell's block][slot])
__global__ void bk_axpy(int64_t n, int lg3, const int32_t* __restrict__ blk_prob, const double* __restrict__ scal, int slot,
                        float sign, const float* __restrict__ x, float* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] += (float)(sign * scal[(int64_t)blk_prob[i >> lg3] * S_WIDTH + slot]) * x[i];
}

// p = z + beta_p p
__global__ void bk_xpay(int64_t n, int lg3, const int32_t* __restrict__ blk_prob, const double* __restrict__ scal,
                        const float* __restrict__ z, float* __restrict__ p) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + (float)scal[(int64_t)blk_prob[i >> lg3] * S_WIDTH + S_BETA] * p[i];
}

// x64 += alpha_p p
__global__ void bk_add64(int64_t n, int lg3, const int32_t* __restrict__ blk_prob, const double* __restrict__ scal,
                         const float* __restrict__ p, double* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] += scal[(int64_t)blk_prob[i >> lg3] * S_WIDTH + S_ALPHA] * (double)p[i];
}

static void seg_dot(msbg_poisson* P, const float* a, const float* b, int slot) {
    const PLevelDev& F = P->lv[0];
    const int cells = F.bs * F.bs * F.bs;
    begin_launch(P->ctx);
    bk_block_dot<<<(unsigned)std::min<int64_t>(F.n(), 148 * 8), 256, 0, P->ctx->stream>>>(F.n(), cells, a, b,
                                                                                         P->bpart.as<double>());
    after_launch(P->ctx, "bk_block_dot");
    begin_launch(P->ctx);
    bk_seg_sum<<<(unsigned)((P->np * 32 + 255) / 256), 256, 0, P->ctx->stream>>>(
        P->np, P->d_prob_blocks.as<int64_t>(), P->bpart.as<double>(), P->scal.as<double>(), slot);
    after_launch(P->ctx, "bk_seg_sum");
}

static void scalars(msbg_poisson* P, int op, double tol) {
    begin_launch(P->ctx);
    bk_scalars<<<(unsigned)((P->np + 127) / 128), 128, 0, P->ctx->stream>>>(P->np, P->scal.as<double>(), op, tol * tol);
    after_launch(P->ctx, "bk_scalars");
}

// Start of a batched solve (not captured): r = b - A x, b.b, r.r, active flags.
static void batch_start(msbg_poisson* P, double* x64, const float* b, double tol) {
    const int64_t n = P->lv[0].cells();
    float* r = (float*)P->work.p;
    CUDA_CHECK(cudaMemsetAsync(P->scal.p, 0, (size_t)P->np * S_WIDTH * 8, P->ctx->stream));
    launch_residual64(P, x64, b, r);
    seg_dot(P, b, b, S_BB);
    seg_dot(P, r, r, S_RR);
    scalars(P, 2, tol);
    (void)n;
}

// One cycle (capturable): restart CG from the current true residual r, K
// iterations of MG-preconditioned CG with per-problem scalars, then the true
// residual of the FP64 solution replaces r (FP64 residual-based iterative
// refinement) and the active flags are updated.
static void batch_cycle(msbg_poisson* P, double* x64, const float* b, int K, double tol) {
    const PLevelDev& F = P->lv[0];
    const int64_t n = F.cells();
    const int lg3 = 3 * F.lg;
    float* r = (float*)P->work.p;
    float* z = r + n;
    float* p = z + n;
    float* q = p + n;
    const int32_t* bp = P->d_blk_prob.as<int32_t>();
    double* sc = P->scal.as<double>();
    msbg_ctx* ctx = P->ctx;
    vcycle(P, 0, z, r, true);
    CUDA_CHECK(cudaMemcpyAsync(p, z, n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    seg_dot(P, r, z, S_RZ);
    for (int k = 0; k < K; ++k) {
        launch_matvec(P, 0, p, q);
        seg_dot(P, p, q, S_PQ);
        scalars(P, 0, tol);
        begin_launch(ctx);
        bk_add64<<<grid_for(n), 256, 0, ctx->stream>>>(n, lg3, bp, sc, p, x64);
        after_launch(ctx, "bk_add64");
        begin_launch(ctx);
        bk_axpy<<<grid_for(n), 256, 0, ctx->stream>>>(n, lg3, bp, sc, S_ALPHA, -1.0f, q, r);
        after_launch(ctx, "bk_axpy");
        vcycle(P, 0, z, r, true);
        seg_dot(P, r, z, S_RZN);
        scalars(P, 1, tol);
        begin_launch(ctx);
        bk_xpay<<<grid_for(n), 256, 0, ctx->stream>>>(n, lg3, bp, sc, z, p);
        after_launch(ctx, "bk_xpay");
    }
    launch_residual64(P, x64, b, r);
    seg_dot(P, r, r, S_RR);
    scalars(P, 2, tol);
}

// Autotuner: for every level but the coarsest, time each choice on the
// level's own buffers (CUDA events, three launches after one warm-up) and keep
// the fastest: levels of whole 16^3 blocks the tile kernel's slab depth (one
// Jacobi sweep plus one residual per candidate), the others each launch shape
// of the Jacobi and residual kernels.
static void autotune(msbg_poisson* P) {
    msbg_ctx* ctx = P->ctx;
    MSBG_REQUIRE(!ctx->timing, "autotuning needs per-kernel timing off");
    drop_graphs(P);
    cudaEvent_t e0, e1;
    CUDA_CHECK(cudaEventCreate(&e0));
    CUDA_CHECK(cudaEventCreate(&e1));
    for (size_t l = 0; l + 1 < P->lv.size(); ++l) {
        PLevelDev& L = P->lv[l];
        const int64_t cells = L.cells();
        CUDA_CHECK(cudaMemsetAsync(L.x.p, 0, cells * 4, ctx->stream));
        CUDA_CHECK(cudaMemsetAsync(L.b.p, 0, cells * 4, ctx->stream));
        if (uses_block16(L)) {
            float best = 1e30f;
            int best_slab = 4;
            for (int slab : {1, 2, 4, 8, 16}) {
                auto run = [&]() {
                    launch_block16<0>(ctx, L, slab, L.x.as<float>(), L.b.as<float>(), L.t.as<float>(), P->omega);
                    launch_block16<1>(ctx, L, slab, L.x.as<float>(), L.b.as<float>(), L.r.as<float>(), 0.0f);
                };
                run();
                CUDA_CHECK(cudaEventRecord(e0, ctx->stream));
                for (int rep = 0; rep < 3; ++rep) run();
                CUDA_CHECK(cudaEventRecord(e1, ctx->stream));
                CUDA_CHECK(cudaEventSynchronize(e1));
                CUDA_CHECK(cudaGetLastError());
                float ms = 0.0f;
                CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
                ctx->launches += 8;
                if (ms < best) {
                    best = ms;
                    best_slab = slab;
                }
            }
            L.slab = best_slab;
            continue;
        }
        for (int kind = 0; kind < 2; ++kind) {
            float best = 1e30f;
            int best_cfg = 0;
            for (int c = 0; c < kNumShapes; ++c) {
                auto run = [&]() {
                    if (kind == 0)
                        pk_jacobi<<<shape_grid(c, cells), kShapes[c].threads, 0, ctx->stream>>>(
                            level_args(L), L.x.as<float>(), L.b.as<float>(), L.t.as<float>(), P->omega);
                    else
                        pk_residual<<<shape_grid(c, cells), kShapes[c].threads, 0, ctx->stream>>>(
                            level_args(L), L.x.as<float>(), L.b.as<float>(), L.r.as<float>());
                };
                run();
                CUDA_CHECK(cudaEventRecord(e0, ctx->stream));
                for (int rep = 0; rep < 3; ++rep) run();
                CUDA_CHECK(cudaEventRecord(e1, ctx->stream));
                CUDA_CHECK(cudaEventSynchronize(e1));
                CUDA_CHECK(cudaGetLastError());
                float ms = 0.0f;
                CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
                ctx->launches += 4;
                if (ms < best) {
                    best = ms;
                    best_cfg = c;
                }
            }
            if (kind == 0) L.cfg_jac = best_cfg;
            else L.cfg_res = best_cfg;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

}  // namespace msbg

namespace msbg {

// The convergence test of the device-side solve loop: any problem of any
// group still active (S_ACTIVE > 0) and fewer than ctrl[1] cycles run sets
// the loop's condition; `advance` counts the cycle just finished.  One block.
struct GroupScal {
    const double* scal;
    int64_t np;
};
__global__ void bk_loop_ctrl(cudaGraphConditionalHandle h, const GroupScal* __restrict__ gt, int ng,
                             long long* __restrict__ ctrl, int advance) {
    int any = 0;
    for (int g = 0; g < ng; ++g)
        for (int64_t i = threadIdx.x; i < gt[g].np; i += blockDim.x) any |= gt[g].scal[i * S_WIDTH + S_ACTIVE] > 0.0;
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        const long long c = ctrl[0] + advance;
        ctrl[0] = c;
        cudaGraphSetConditional(h, (any && c < ctrl[1]) ? 1u : 0u);
    }
}

}  // namespace msbg

// A batch: problems grouped by block size, each group one stacked hierarchy.
// The solve is one graph: a convergence test, then a device-side while loop
// whose body is one cycle of every group followed by the test again.
struct msbg_batch {
    msbg_ctx* ctx = nullptr;
    std::vector<msbg_poisson*> groups;
    std::vector<int> prob_group, prob_index;  // per problem: group and index inside it
    std::vector<msbg::DevBuf> b, x;           // per group: f32 right-hand sides, FP64 solutions
    msbg::DevBuf gtab;                         // GroupScal per group
    msbg::DevBuf ctrl;                         // long long [2]: cycles run, cycle limit
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_k = 0, graph_kernels = 0;  // CG iterations per cycle, kernels per loop iteration
    double graph_tol = 0.0;
    ~msbg_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (msbg_poisson* P : groups) delete P;
    }
};

namespace msbg {

static void batch_group_build(msbg_poisson* P, int bsx, const std::vector<int>& probs, const uint64_t* dims,
                              const uint64_t* const* active, const size_t* n_active) {
    int64_t NX = 1, NY = 1, nzmax = 1;
    for (int p : probs) {
        NX = std::max<int64_t>(NX, (int64_t)((dims[3 * p] + bsx - 1) / bsx));
        NY = std::max<int64_t>(NY, (int64_t)((dims[3 * p + 1] + bsx - 1) / bsx));
        nzmax = std::max<int64_t>(nzmax, (int64_t)((dims[3 * p + 2] + bsx - 1) / bsx));
    }
    const int L = ilog2i((uint64_t)std::max(NX, std::max(NY, nzmax))) + 1;  // halvings that shrink any problem to one block
    const int64_t G = int64_t(1) << (L + 1);
    std::vector<uint64_t> all;
    std::vector<int64_t> zoff(probs.size());
    int64_t Z = 0;
    for (size_t i = 0; i < probs.size(); ++i) {
        const int p = probs[i];
        const uint64_t nx = (dims[3 * p] + bsx - 1) / bsx, ny = (dims[3 * p + 1] + bsx - 1) / bsx,
                       nz = (dims[3 * p + 2] + bsx - 1) / bsx;
        MSBG_REQUIRE(n_active[p] > 0, "a batched problem has no active blocks");
        zoff[i] = Z;
        for (size_t j = 0; j < n_active[p]; ++j) {
            const uint64_t b = active[p][j];
            MSBG_REQUIRE(b < nx * ny * nz, "active block id out of range");
            const uint64_t bx = b % nx, by = (b / nx) % ny, bz = b / (nx * ny);
            all.push_back(bx + by * (uint64_t)NX + (bz + (uint64_t)Z) * (uint64_t)(NX * NY));
        }
        const int64_t align = int64_t(1) << L;
        Z = ((Z + (int64_t)nz + align - 1) / align) * align + G;
    }
    build(P, (uint64_t)NX * bsx, (uint64_t)NY * bsx, (uint64_t)Z * bsx, bsx, all.data(), all.size(), L);
    // problem ranges of the level-0 blocks (sorted by z, so contiguous)
    const PLevelDev& F = P->lv[0];
    P->np = (int)probs.size();
    P->prob_blocks.assign(P->np + 1, 0);
    std::vector<int32_t> blk_prob(F.n());
    size_t k = 0;
    for (int i = 0; i < P->np; ++i) {
        P->prob_blocks[i] = (int64_t)k;
        const int64_t z_hi = (i + 1 < P->np) ? zoff[i + 1] : INT64_MAX;
        while (k < F.bids.size() && (int64_t)(F.bids[k] / (uint64_t)(NX * NY)) < z_hi) blk_prob[k++] = i;
    }
    P->prob_blocks[P->np] = (int64_t)k;
    MSBG_REQUIRE(k == F.bids.size(), "batched problem layout is inconsistent");
    upload(P->ctx, P->d_prob_blocks, P->prob_blocks.data(), P->prob_blocks.size() * 8);
    upload(P->ctx, P->d_blk_prob, blk_prob.data(), blk_prob.size() * 4);
    P->bpart.reserve((size_t)F.n() * 8 + 64);
    P->scal.reserve((size_t)P->np * S_WIDTH * 8 + 64);
    sync(P->ctx);
}

}  // namespace msbg

using namespace msbg;

extern "C" {

int msbg_poisson_create(msbg_ctx* ctx, uint64_t sx, uint64_t sy, uint64_t sz, int bsx, const uint64_t* active, size_t n,
                        msbg_poisson** out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && out && (active || !n), "null argument");
    MSBG_REQUIRE(is_pow2((uint64_t)bsx) && bsx >= 2 && bsx <= 32, "bsx must be a power of two in [2, 32]");
    set_device(ctx);
    auto* P = new msbg_poisson;
    P->ctx = ctx;
    try {
        build(P, sx, sy, sz, bsx, active, n);
    } catch (...) {
        delete P;
        throw;
    }
    *out = P;
    MSBG_API_END
}

int msbg_poisson_destroy(msbg_poisson* P) {
    MSBG_API_BEGIN
    if (!P) return MSBG_OK;
    cudaSetDevice(P->ctx->device);
    cudaStreamSynchronize(P->ctx->stream);
    delete P;
    MSBG_API_END
}

int msbg_poisson_levels(const msbg_poisson* P, uint64_t* cells_out, size_t cap, size_t* n_levels) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && n_levels, "null argument");
    *n_levels = P->lv.size();
    for (size_t l = 0; l < P->lv.size() && l < cap; ++l) cells_out[l] = (uint64_t)P->lv[l].cells();
    MSBG_API_END
}

int msbg_poisson_set_smoother(msbg_poisson* P, int nu1, int nu2, float omega) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && nu1 >= 0 && nu2 >= 0 && omega > 0.0f && omega < 2.0f, "bad smoother parameters");
    set_device(P->ctx);
    drop_graphs(P);
    P->nu1 = nu1;
    P->nu2 = nu2;
    P->omega = omega;
    MSBG_API_END
}

int msbg_poisson_matvec_device(msbg_poisson* P, const float* d_x, float* d_y) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && d_x && d_y, "null argument");
    set_device(P->ctx);
    launch_matvec(P, 0, d_x, d_y);
    MSBG_API_END
}

int msbg_poisson_jacobi_device(msbg_poisson* P, float* d_x, const float* d_b, float omega, int sweeps) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && d_x && d_b && sweeps >= 0, "bad argument");
    set_device(P->ctx);
    jacobi(P, 0, d_x, d_b, sweeps, omega, false);
    MSBG_API_END
}

int msbg_poisson_residual_device(msbg_poisson* P, const float* d_x, const float* d_b, float* d_r, double* norm_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && d_x && d_b && d_r, "null argument");
    set_device(P->ctx);
    launch_residual(P, 0, d_x, d_b, d_r);
    if (norm_out) *norm_out = std::sqrt(dot(P, d_r, d_r, P->lv[0].cells()));
    MSBG_API_END
}

int msbg_poisson_vcycle_device(msbg_poisson* P, float* d_x, const float* d_b) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && d_x && d_b, "null argument");
    set_device(P->ctx);
    vcycle(P, 0, d_x, d_b, false);
    MSBG_API_END
}

int msbg_poisson_dot_device(msbg_poisson* P, const float* d_a, const float* d_b, double* out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && d_a && d_b && out, "null argument");
    set_device(P->ctx);
    *out = dot(P, d_a, d_b, P->lv[0].cells());
    MSBG_API_END
}

int msbg_poisson_solve_device(msbg_poisson* P, int method, float* d_x, const float* d_b, double tol, int max_iter,
                              int* iters_out, double* rel_res_out, double* history) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && d_x && d_b && method >= 0 && method <= 5 && max_iter >= 0 && tol > 0.0, "bad argument");
    set_device(P->ctx);
    int it = solve(P, method, d_x, d_b, tol, max_iter, rel_res_out, history);
    if (iters_out) *iters_out = it;
    MSBG_API_END
}

int msbg_poisson_solve(msbg_poisson* P, int method, float* x, const float* b, double tol, int max_iter, int* iters_out,
                       double* rel_res_out, double* history) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && x && b && method >= 0 && method <= 5 && max_iter >= 0 && tol > 0.0, "bad argument");
    set_device(P->ctx);
    const int64_t n = P->lv[0].cells();
    DevBuf& io = P->io;
    io.reserve((size_t)n * 8 + 512);
    float* dx = io.as<float>();
    float* db = dx + n;
    CUDA_CHECK(cudaMemcpyAsync(dx, x, n * 4, cudaMemcpyHostToDevice, P->ctx->stream));
    CUDA_CHECK(cudaMemcpyAsync(db, b, n * 4, cudaMemcpyHostToDevice, P->ctx->stream));
    int it = solve(P, method, dx, db, tol, max_iter, rel_res_out, history);
    CUDA_CHECK(cudaMemcpyAsync(x, dx, n * 4, cudaMemcpyDeviceToHost, P->ctx->stream));
    sync(P->ctx);
    if (iters_out) *iters_out = it;
    MSBG_API_END
}

int msbg_poisson_solve_f64_device(msbg_poisson* P, int method, double* d_x, const float* d_b, double tol, int max_iter,
                                  int* iters_out, double* rel_res_out, double* history) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && d_x && d_b && method >= 0 && method <= 5 && max_iter >= 0 && tol > 0.0, "bad argument");
    set_device(P->ctx);
    int it = solve(P, method, nullptr, d_b, tol, max_iter, rel_res_out, history, d_x);
    if (iters_out) *iters_out = it;
    MSBG_API_END
}

int msbg_poisson_set_preconditioner(msbg_poisson* P, msbg_unet* net) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P, "null argument");
    if (net) {
        MSBG_REQUIRE(P->lv[0].bs == 16 && unet_blocks(net) == P->lv[0].n() && unet_ctx(net) == P->ctx,
                     "the network must be built on the solve's level-0 blocks (16^3) and context");
    }
    P->net = net;
    MSBG_API_END
}

int msbg_poisson_set_network_lead(msbg_poisson* P, int k) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P, "null argument");
    P->net_lead = k >= 0 ? k : -k;
    P->net_lead_post = k >= 0 ? 1 : 0;
    MSBG_API_END
}

int msbg_poisson_solve_stats(const msbg_poisson* P, int* out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && out, "null argument");
    out[0] = P->n_vcycle;
    out[1] = P->n_net;
    out[2] = P->fell_back;
    out[3] = P->fallback_iter;
    MSBG_API_END
}

int msbg_poisson_rhs_device(msbg_poisson* P, uint64_t seed, int n_blobs, float* d_b) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && d_b && n_blobs > 0 && n_blobs <= 4096, "bad argument");
    set_device(P->ctx);
    DevBuf blobs;
    blob_rhs(P, seed, n_blobs, d_b, blobs);
    MSBG_API_END
}

int msbg_poisson_train_preconditioner(msbg_poisson* P, int n_rhs, int mg_iters, int steps_per_rhs, int pool, float lr,
                                      int target, uint64_t seed, double* loss_hist, int64_t hist_cap, int64_t* steps_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && n_rhs >= 0 && mg_iters > 0 && steps_per_rhs >= 0 && pool > 0 && lr >= 0.0f &&
                     (target & 1) == target % 2 && target >= 0 && target <= 3,
                 "bad argument");
    set_device(P->ctx);
    // target bit 0: pair kind (0 residual/error, 1 post-V-cycle); bit 1: the
    // iterates of MG-preconditioned CG instead of plain V-cycles
    const TrainStats st = train(P, n_rhs, mg_iters, steps_per_rhs, pool, lr, target & 1, seed, loss_hist, hist_cap,
                                target >> 1);
    if (steps_out) *steps_out = st.steps;
    MSBG_API_END
}

int msbg_poisson_eval_preconditioner(msbg_poisson* P, int n_rhs, int mg_iters, uint64_t seed, double* out3) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && out3 && n_rhs > 0 && mg_iters > 0 && P->net, "bad argument");
    set_device(P->ctx);
    evaluate(P, n_rhs, mg_iters, seed, out3);
    MSBG_API_END
}

int msbg_poisson_autotune(msbg_poisson* P, int* cfg_out, size_t cap, size_t* n_levels) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P, "null argument");
    set_device(P->ctx);
    autotune(P);
    if (n_levels) *n_levels = P->lv.size();
    for (size_t l = 0; l < P->lv.size() && cfg_out && 3 * l + 2 < cap; ++l) {
        cfg_out[3 * l] = P->lv[l].cfg_jac;
        cfg_out[3 * l + 1] = P->lv[l].cfg_res;
        cfg_out[3 * l + 2] = uses_block16(P->lv[l]) ? P->lv[l].slab : 0;
    }
    MSBG_API_END
}

int msbg_poisson_set_tuning(msbg_poisson* P, const int* cfg, size_t n_levels) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && (cfg || !n_levels), "null argument");
    MSBG_REQUIRE(n_levels <= P->lv.size(), "more levels than the hierarchy has");
    for (size_t l = 0; l < n_levels; ++l) {
        const int j = cfg[3 * l], r = cfg[3 * l + 1], t = cfg[3 * l + 2];
        MSBG_REQUIRE(j >= 0 && j < kNumShapes && r >= 0 && r < kNumShapes, "launch shape index out of range");
        MSBG_REQUIRE(uses_block16(P->lv[l]) ? (t == 1 || t == 2 || t == 4 || t == 8 || t == 16) : t == 0,
                     "tile must be 1, 2, 4, 8 or 16 on levels of whole 16^3 blocks and 0 elsewhere");
    }
    set_device(P->ctx);
    drop_graphs(P);
    for (size_t l = 0; l < n_levels; ++l) {
        P->lv[l].cfg_jac = cfg[3 * l];
        P->lv[l].cfg_res = cfg[3 * l + 1];
        if (cfg[3 * l + 2]) P->lv[l].slab = cfg[3 * l + 2];
    }
    MSBG_API_END
}

int msbg_batch_create(msbg_ctx* ctx, int n_problems, const int* bsx, const uint64_t* dims, const uint64_t* const* active,
                      const size_t* n_active, int tune, msbg_batch** out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(ctx && out && n_problems > 0 && bsx && dims && active && n_active, "null argument");
    MSBG_REQUIRE(n_problems <= 256, "at most 256 problems per batch");
    set_device(ctx);
    auto* B = new msbg_batch;
    B->ctx = ctx;
    try {
        B->prob_group.assign(n_problems, -1);
        B->prob_index.assign(n_problems, -1);
        std::vector<int> sizes;
        for (int p = 0; p < n_problems; ++p) {
            MSBG_REQUIRE(is_pow2((uint64_t)bsx[p]) && bsx[p] >= 4 && bsx[p] <= 32, "batched block sizes are powers of two in [4, 32]");
            int g = -1;
            for (size_t i = 0; i < sizes.size(); ++i)
                if (sizes[i] == bsx[p]) g = (int)i;
            if (g < 0) {
                g = (int)sizes.size();
                sizes.push_back(bsx[p]);
            }
            B->prob_group[p] = g;
        }
        for (size_t g = 0; g < sizes.size(); ++g) {
            std::vector<int> probs;
            for (int p = 0; p < n_problems; ++p)
                if (B->prob_group[p] == (int)g) {
                    B->prob_index[p] = (int)probs.size();
                    probs.push_back(p);
                }
            auto* P = new msbg_poisson;
            P->ctx = ctx;
            B->groups.push_back(P);
            batch_group_build(P, sizes[g], probs, dims, active, n_active);
            if (tune) autotune(P);
            const int64_t n = P->lv[0].cells();
            B->b.emplace_back();
            B->x.emplace_back();
            B->b.back().reserve((size_t)n * 4 + 256);
            B->x.back().reserve((size_t)n * 8 + 256);
            CUDA_CHECK(cudaMemsetAsync(B->b.back().p, 0, (size_t)n * 4, ctx->stream));
            CUDA_CHECK(cudaMemsetAsync(B->x.back().p, 0, (size_t)n * 8, ctx->stream));
        }
        sync(ctx);
    } catch (...) {
        delete B;
        throw;
    }
    *out = B;
    MSBG_API_END
}

int msbg_batch_destroy(msbg_batch* B) {
    MSBG_API_BEGIN
    if (!B) return MSBG_OK;
    cudaSetDevice(B->ctx->device);
    cudaStreamSynchronize(B->ctx->stream);
    delete B;
    MSBG_API_END
}

int msbg_batch_problem(const msbg_batch* B, int p, int* group, uint64_t* cell_offset, uint64_t* n_cells) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(B && p >= 0 && p < (int)B->prob_group.size(), "bad argument");
    const int g = B->prob_group[p], i = B->prob_index[p];
    const msbg_poisson* P = B->groups[g];
    const int64_t cb = (int64_t)P->lv[0].bs * P->lv[0].bs * P->lv[0].bs;
    if (group) *group = g;
    if (cell_offset) *cell_offset = (uint64_t)(P->prob_blocks[i] * cb);
    if (n_cells) *n_cells = (uint64_t)((P->prob_blocks[i + 1] - P->prob_blocks[i]) * cb);
    MSBG_API_END
}

int msbg_batch_buffers(msbg_batch* B, int g, float** d_b, double** d_x, uint64_t* n_cells, int* bsx) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(B && g >= 0 && g < (int)B->groups.size(), "bad argument");
    if (d_b) *d_b = B->b[g].as<float>();
    if (d_x) *d_x = B->x[g].as<double>();
    if (n_cells) *n_cells = (uint64_t)B->groups[g]->lv[0].cells();
    if (bsx) *bsx = B->groups[g]->lv[0].bs;
    MSBG_API_END
}

int msbg_batch_set_rhs(msbg_batch* B, int p, const float* b) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(B && b && p >= 0 && p < (int)B->prob_group.size(), "bad argument");
    set_device(B->ctx);
    const int g = B->prob_group[p], i = B->prob_index[p];
    const msbg_poisson* P = B->groups[g];
    const int64_t cb = (int64_t)P->lv[0].bs * P->lv[0].bs * P->lv[0].bs;
    const int64_t off = P->prob_blocks[i] * cb, cnt = (P->prob_blocks[i + 1] - P->prob_blocks[i]) * cb;
    CUDA_CHECK(cudaMemcpyAsync(B->b[g].as<float>() + off, b, (size_t)cnt * 4, cudaMemcpyHostToDevice, B->ctx->stream));
    sync(B->ctx);
    MSBG_API_END
}

int msbg_batch_get_solution(msbg_batch* B, int p, double* x) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(B && x && p >= 0 && p < (int)B->prob_group.size(), "bad argument");
    set_device(B->ctx);
    const int g = B->prob_group[p], i = B->prob_index[p];
    const msbg_poisson* P = B->groups[g];
    const int64_t cb = (int64_t)P->lv[0].bs * P->lv[0].bs * P->lv[0].bs;
    const int64_t off = P->prob_blocks[i] * cb, cnt = (P->prob_blocks[i + 1] - P->prob_blocks[i]) * cb;
    CUDA_CHECK(cudaMemcpyAsync(x, B->x[g].as<double>() + off, (size_t)cnt * 8, cudaMemcpyDeviceToHost, B->ctx->stream));
    sync(B->ctx);
    MSBG_API_END
}

int msbg_batch_groups(const msbg_batch* B, int* n_groups) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(B && n_groups, "null argument");
    *n_groups = (int)B->groups.size();
    MSBG_API_END
}

int msbg_batch_tuning(const msbg_batch* B, int g, int* cfg_out, uint64_t* cells_out, size_t cap, size_t* n_levels) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(B && g >= 0 && g < (int)B->groups.size() && n_levels, "bad argument");
    const msbg_poisson* P = B->groups[g];
    *n_levels = P->lv.size();
    for (size_t l = 0; l < P->lv.size() && l < cap; ++l) {
        if (cfg_out) {
            cfg_out[3 * l] = P->lv[l].cfg_jac;
            cfg_out[3 * l + 1] = P->lv[l].cfg_res;
            cfg_out[3 * l + 2] = uses_block16(P->lv[l]) ? P->lv[l].slab : 0;
        }
        if (cells_out) cells_out[l] = (uint64_t)P->lv[l].cells();
    }
    MSBG_API_END
}

// Solves every problem of the batch to relative residual `tol` (true
// residual of the FP64 solution) from the current solutions (zero_x: from
// zero).  A cycle is iters_per_cycle CG iterations for all problems and the
// FP64 residual replacement; the cycles run in one CUDA graph launch, a
// device-side while loop that stops once no problem is active or after
// max_cycles cycles, so the host waits only once, at the end.
int msbg_batch_solve(msbg_batch* B, double tol, int iters_per_cycle, int max_cycles, int zero_x, int* iters_out,
                     double* rel_out, int* cycles_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(B && tol > 0.0 && iters_per_cycle > 0 && max_cycles >= 0, "bad argument");
    msbg_ctx* ctx = B->ctx;
    MSBG_REQUIRE(!ctx->timing, "per-kernel timing must be off for the captured batch solve");
    set_device(ctx);
    for (size_t g = 0; g < B->groups.size(); ++g) {
        msbg_poisson* P = B->groups[g];
        if (zero_x) CUDA_CHECK(cudaMemsetAsync(B->x[g].p, 0, (size_t)P->lv[0].cells() * 8, ctx->stream));
        batch_start(P, B->x[g].as<double>(), B->b[g].as<float>(), tol);
    }
    if (!B->exec || B->graph_k != iters_per_cycle || B->graph_tol != tol) {
        if (B->exec) cudaGraphExecDestroy(B->exec);
        if (B->graph) cudaGraphDestroy(B->graph);
        B->exec = nullptr;
        B->graph = nullptr;
        const int ng = (int)B->groups.size();
        if (!B->gtab.p) {
            std::vector<GroupScal> gt(ng);
            for (int g = 0; g < ng; ++g) gt[g] = GroupScal{B->groups[g]->scal.as<double>(), (int64_t)B->groups[g]->np};
            B->gtab.reserve(sizeof(GroupScal) * ng);
            B->ctrl.reserve(2 * sizeof(long long));
            CUDA_CHECK(cudaMemcpyAsync(B->gtab.p, gt.data(), sizeof(GroupScal) * ng, cudaMemcpyHostToDevice, ctx->stream));
            sync(ctx);
        }
        const GroupScal* gt = B->gtab.as<GroupScal>();
        long long* ctrl = B->ctrl.as<long long>();
        cudaGraph_t G = nullptr;
        CUDA_CHECK(cudaGraphCreate(&G, 0));
        const uint64_t l0 = ctx->launches;
        bool capturing = false;
        try {
            cudaGraphConditionalHandle h;
            CUDA_CHECK(cudaGraphConditionalHandleCreate(&h, G, 0, 0));
            // the test before the loop, captured into G
            CUDA_CHECK(cudaStreamBeginCaptureToGraph(ctx->stream, G, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            capturing = true;
            bk_loop_ctrl<<<1, 256, 0, ctx->stream>>>(h, gt, ng, ctrl, 0);
            CUDA_CHECK(cudaGetLastError());
            CUDA_CHECK(cudaStreamEndCapture(ctx->stream, &G));
            capturing = false;
            size_t nn = 1;
            cudaGraphNode_t test_node;
            CUDA_CHECK(cudaGraphGetNodes(G, &test_node, &nn));
            // the while node after it
            cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t loop_node;
            CUDA_CHECK(cudaGraphAddNode(&loop_node, G, &test_node, 1, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            // its body: one cycle of every group, then the test
            CUDA_CHECK(cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            capturing = true;
            for (int g = 0; g < ng; ++g)
                batch_cycle(B->groups[g], B->x[g].as<double>(), B->b[g].as<float>(), iters_per_cycle, tol);
            begin_launch(ctx);
            bk_loop_ctrl<<<1, 256, 0, ctx->stream>>>(h, gt, ng, ctrl, 1);
            after_launch(ctx, "bk_loop_ctrl");
            CUDA_CHECK(cudaStreamEndCapture(ctx->stream, &body));
            capturing = false;
            CUDA_CHECK(cudaGraphInstantiate(&B->exec, G, 0));
        } catch (...) {
            if (capturing) {
                cudaGraph_t tmp = nullptr;
                cudaStreamEndCapture(ctx->stream, &tmp);
            }
            cudaGraphDestroy(G);
            ctx->launches = l0;
            throw;
        }
        B->graph = G;
        B->graph_k = iters_per_cycle;
        B->graph_tol = tol;
        B->graph_kernels = (int)(ctx->launches - l0);
        ctx->launches = l0;
    }
    // one launch of the whole solve: the host reads the scalars once, after it
    const long long ctrl_init[2] = {0, (long long)max_cycles};
    CUDA_CHECK(cudaMemcpyAsync(B->ctrl.p, ctrl_init, sizeof(ctrl_init), cudaMemcpyHostToDevice, ctx->stream));
    CUDA_CHECK(cudaGraphLaunch(B->exec, ctx->stream));
    std::vector<std::vector<double>> sc(B->groups.size());
    long long cyc[2] = {0, 0};
    {
        SmallReads rd(ctx);
        for (size_t g = 0; g < B->groups.size(); ++g) {
            const msbg_poisson* P = B->groups[g];
            sc[g].resize((size_t)P->np * S_WIDTH);
            rd.add(sc[g].data(), P->scal.p, sc[g].size() * 8);
        }
        rd.add(cyc, B->ctrl.p, sizeof(cyc));
        rd.wait();
    }
    const int cycles = (int)cyc[0];
    ctx->launches += 1 + (uint64_t)cycles * (uint64_t)B->graph_kernels;
    for (size_t p = 0; p < B->prob_group.size(); ++p) {
        const double* S = sc[B->prob_group[p]].data() + (size_t)B->prob_index[p] * S_WIDTH;
        if (iters_out) iters_out[p] = (int)S[S_ITER];
        if (rel_out) rel_out[p] = S[S_BB] > 0.0 ? std::sqrt(S[S_RR] / S[S_BB]) : 0.0;
    }
    if (cycles_out) *cycles_out = cycles;
    MSBG_API_END
}

}  // extern "C"
