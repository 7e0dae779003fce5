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
// size 2 on the block grid halves (a coarse block is active when any of its 8
// children is).  The level-l operator is s_l (6 x - sum nb), s_l = 0.5^l, the
// Galerkin product R A P for averaging restriction and piecewise-constant
// prolongation.  Coarsening stops at <= 1024 cells, solved with a dense FP64
// inverse computed at set-up (Cholesky on the host).
//
// Layout in HBM: one f32 array per level and vector, [n_blocks][bs^3] in
// ascending block-id order (the block payload layout of the sparse grid).
// Vectors and smoothing are FP32; dot products and norms accumulate in FP64
// with a fixed two-stage reduction order (deterministic).
#include <algorithm>
#include <cmath>

#include "common.cuh"

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
    DevBuf x, b, r, t;  // f32 [cells]
    int64_t n() const { return (int64_t)bids.size(); }
    int64_t cells() const { return n() * bs * bs * bs; }
};

// Child table of a level: for each of its cells, the slot of the finer
// level's block holding the cell's 8 children and the cell index of the
// (0,0,0) child, or slot -1.
struct ChildTable {
    DevBuf slot, v0;
};

}  // namespace msbg

struct msbg_poisson {
    msbg_ctx* ctx = nullptr;
    std::vector<msbg::PLevelDev> lv;
    std::vector<msbg::ChildTable> children;  // children[l]: level-l cells -> level l-1
    msbg::DevBuf ainv;   // f64 [nc][nc] column-major inverse of the coarsest operator
    int64_t nc = 0;
    int nu1 = 2, nu2 = 2;
    float omega = 2.0f / 3.0f;
    msbg::DevBuf work;   // PCG vectors + dot partials
};

namespace msbg {

// ---- kernels -----------------------------------------------------------------
struct LevelArgs {
    const int32_t* nbr;
    int lg;
    int64_t cells;
    float scale;
};

// Sum of the 6 face neighbours of cell i (zero outside the active blocks).
template <typename T>
__device__ __forceinline__ T nb_sum(const LevelArgs& L, const T* __restrict__ x, int64_t i) {
    const int bs = 1 << L.lg, m = bs - 1;
    const int64_t k = i >> (3 * L.lg);
    const int v = (int)(i & ((1 << (3 * L.lg)) - 1));
    const int cx = v & m, cy = (v >> L.lg) & m, cz = v >> (2 * L.lg);
    const int32_t* nb = L.nbr + k * 6;
    T s;
    {
        const int32_t kk = cx > 0 ? (int32_t)k : nb[0];
        s = kk >= 0 ? x[((int64_t)kk << (3 * L.lg)) + (v & ~m) + ((cx - 1) & m)] : T(0);
    }
    {
        const int32_t kk = cx < m ? (int32_t)k : nb[1];
        s += kk >= 0 ? x[((int64_t)kk << (3 * L.lg)) + (v & ~m) + ((cx + 1) & m)] : T(0);
    }
    {
        const int32_t kk = cy > 0 ? (int32_t)k : nb[2];
        s += kk >= 0 ? x[((int64_t)kk << (3 * L.lg)) + cx + (((cy - 1) & m) << L.lg) + (cz << (2 * L.lg))] : T(0);
    }
    {
        const int32_t kk = cy < m ? (int32_t)k : nb[3];
        s += kk >= 0 ? x[((int64_t)kk << (3 * L.lg)) + cx + (((cy + 1) & m) << L.lg) + (cz << (2 * L.lg))] : T(0);
    }
    {
        const int32_t kk = cz > 0 ? (int32_t)k : nb[4];
        s += kk >= 0 ? x[((int64_t)kk << (3 * L.lg)) + cx + (cy << L.lg) + (((cz - 1) & m) << (2 * L.lg))] : T(0);
    }
    {
        const int32_t kk = cz < m ? (int32_t)k : nb[5];
        s += kk >= 0 ? x[((int64_t)kk << (3 * L.lg)) + cx + (cy << L.lg) + (((cz + 1) & m) << (2 * L.lg))] : T(0);
    }
    return s;
}

// y = A x
__global__ void pk_matvec(LevelArgs L, const float* __restrict__ x, float* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L.cells; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = L.scale * (6.0f * x[i] - nb_sum(L, x, i));
}

// r = b - A x
__global__ void pk_residual(LevelArgs L, const float* __restrict__ x, const float* __restrict__ b, float* __restrict__ r) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L.cells; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = b[i] - L.scale * (6.0f * x[i] - nb_sum(L, x, i));
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
        if (x) xn[i] = omega * (b[i] + L.scale * nb_sum(L, x, i)) * inv_d + (1.0f - omega) * x[i];
        else xn[i] = omega * b[i] * inv_d;
    }
}

// Restriction: coarse cell = 1/8 of the sum of its (up to 8) active children.
// Children are visited in z-major order of their offset.
struct TransferArgs {
    const int32_t* fine_coords;   // [nf][3]
    const int32_t* parent;        // [nf] coarse slot
    int lgf, lgc;
    int64_t nf;
};

// The fine cells of one coarse cell are either 8 cells of the same block
// (same-grid levels) or one whole block of 8 cells (grid-halving levels); in
// both cases iterating over fine cells and writing by coarse index would need
// atomics, so the kernel runs over coarse cells with a child table.
__global__ void pk_restrict(const int32_t* __restrict__ child_slot, const int32_t* __restrict__ child_v0, int lgf,
                            int64_t nc_cells, const float* __restrict__ r, float* __restrict__ bc) {
    const int m = (1 << lgf) - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nc_cells; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t ks = child_slot[i];
        float s = 0.0f;
        if (ks >= 0) {
            const int v0 = child_v0[i];
            const float* p = r + ((int64_t)ks << (3 * lgf));
            const int x0 = v0 & m, y0 = (v0 >> lgf) & m, z0 = v0 >> (2 * lgf);
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                const int dx = d & 1, dy = (d >> 1) & 1, dz = d >> 2;
                s += p[(x0 + dx) | ((y0 + dy) << lgf) | ((z0 + dz) << (2 * lgf))];
            }
        }
        bc[i] = s * 0.125f;
    }
}

// Prolongation: x_f += x_c[parent cell] (injection).
__global__ void pk_prolong(TransferArgs T, const float* __restrict__ xc, float* __restrict__ xf) {
    const int bsf = 1 << T.lgf, mf = bsf - 1, mc = (1 << T.lgc) - 1;
    const int64_t total = T.nf << (3 * T.lgf);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i >> (3 * T.lgf);
        const int v = (int)(i & ((1 << (3 * T.lgf)) - 1));
        const int cx = v & mf, cy = (v >> T.lgf) & mf, cz = v >> (2 * T.lgf);
        const int gx = T.fine_coords[3 * k] * bsf + cx, gy = T.fine_coords[3 * k + 1] * bsf + cy,
                  gz = T.fine_coords[3 * k + 2] * bsf + cz;
        const int vc = ((gx >> 1) & mc) | (((gy >> 1) & mc) << T.lgc) | (((gz >> 1) & mc) << (2 * T.lgc));
        xf[i] += xc[((int64_t)T.parent[k] << (3 * T.lgc)) + vc];
    }
}

// x_c = A^-1 b_c with the FP64 inverse (column-major).
__global__ void pk_dense_solve(const double* __restrict__ ainv, int64_t n, const float* __restrict__ b, float* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int64_t j = 0; j < n; ++j) s += ainv[j * n + i] * (double)b[j];
        x[i] = (float)s;
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

// ---- host side -----------------------------------------------------------------
static unsigned grid_for(int64_t n) { return (unsigned)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 16); }

static LevelArgs level_args(const PLevelDev& L) {
    return LevelArgs{L.nbr.as<int32_t>(), L.lg, L.cells(), L.scale};
}

static void upload(msbg_ctx* ctx, DevBuf& d, const void* h, size_t bytes) {
    d.reserve(std::max<size_t>(bytes, 16));
    if (bytes) CUDA_CHECK(cudaMemcpyAsync(d.p, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
}

static void build(msbg_poisson* P, uint64_t sx, uint64_t sy, uint64_t sz, int bsx, const uint64_t* active, size_t n_active) {
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
    while (P->lv.back().cells() > kPoissonDirect) {
        const PLevelDev& F = P->lv.back();
        PLevelDev C;
        C.scale = F.scale * 0.5f;
        if (F.bs >= 4) {
            C.bs = F.bs / 2; C.nx = F.nx; C.ny = F.ny; C.nz = F.nz; C.bids = F.bids;
        } else {
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
    P->children.resize(P->lv.size());
    for (size_t l = 0; l < P->lv.size(); ++l) {
        PLevelDev& L = P->lv[l];
        std::unordered_map<uint64_t, int32_t> slot;
        for (int64_t k = 0; k < L.n(); ++k) slot[L.bids[k]] = (int32_t)k;
        std::vector<int32_t> nbr((size_t)L.n() * 6, -1), coords((size_t)L.n() * 3);
        for (int64_t k = 0; k < L.n(); ++k) {
            const int64_t b = (int64_t)L.bids[k], bx = b % L.nx, by = (b / L.nx) % L.ny, bz = b / (L.nx * L.ny);
            coords[3 * k] = (int32_t)bx; coords[3 * k + 1] = (int32_t)by; coords[3 * k + 2] = (int32_t)bz;
            const int64_t d[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
            for (int f = 0; f < 6; ++f) {
                const int64_t X2 = bx + d[f][0], Y2 = by + d[f][1], Z2 = bz + d[f][2];
                if (X2 < 0 || Y2 < 0 || Z2 < 0 || X2 >= L.nx || Y2 >= L.ny || Z2 >= L.nz) continue;
                auto it = slot.find((uint64_t)(X2 + Y2 * L.nx + Z2 * L.nx * L.ny));
                if (it != slot.end()) nbr[6 * k + f] = it->second;
            }
        }
        upload(ctx, L.nbr, nbr.data(), nbr.size() * 4);
        upload(ctx, L.coords, coords.data(), coords.size() * 4);
        const size_t cb = (size_t)L.cells() * 4;
        L.x.reserve(cb); L.b.reserve(cb); L.r.reserve(cb); L.t.reserve(cb);
        if (l + 1 < P->lv.size()) {
            const PLevelDev& C = P->lv[l + 1];
            std::unordered_map<uint64_t, int32_t> cslot;
            for (int64_t k = 0; k < C.n(); ++k) cslot[C.bids[k]] = (int32_t)k;
            std::vector<int32_t> parent(L.n());
            // child table of the coarse cells (coarse cell -> fine slot + origin cell)
            std::vector<int32_t> cs((size_t)C.cells(), -1), cv((size_t)C.cells(), 0);
            const int bsf = L.bs, bsc = C.bs, mc = bsc - 1;
            for (int64_t k = 0; k < L.n(); ++k) {
                const int64_t bx = coords[3 * k], by = coords[3 * k + 1], bz = coords[3 * k + 2];
                const int64_t cbx = (bx * bsf / 2) / bsc, cby = (by * bsf / 2) / bsc, cbz = (bz * bsf / 2) / bsc;
                const int32_t ps = cslot.at((uint64_t)(cbx + cby * C.nx + cbz * C.nx * C.ny));
                parent[k] = ps;
                for (int cz = 0; cz < bsf; cz += 2)
                    for (int cy = 0; cy < bsf; cy += 2)
                        for (int cx = 0; cx < bsf; cx += 2) {
                            const int64_t gx = (bx * bsf + cx) >> 1, gy = (by * bsf + cy) >> 1, gz = (bz * bsf + cz) >> 1;
                            const int64_t ci = ((int64_t)ps * bsc * bsc * bsc) + ((gx & mc) | ((gy & mc) << C.lg) | ((gz & mc) << (2 * C.lg)));
                            cs[ci] = (int32_t)k;
                            cv[ci] = cx | (cy << L.lg) | (cz << (2 * L.lg));
                        }
            }
            upload(ctx, L.parent, parent.data(), parent.size() * 4);
            upload(ctx, P->children[l + 1].slot, cs.data(), cs.size() * 4);
            upload(ctx, P->children[l + 1].v0, cv.data(), cv.size() * 4);
            sync(ctx);  // host vectors die at scope end
        }
    }
    // dense FP64 inverse of the coarsest operator
    const PLevelDev& C = P->lv.back();
    const int64_t n = C.cells();
    P->nc = n;
    std::unordered_map<uint64_t, int32_t> slot;
    for (int64_t k = 0; k < C.n(); ++k) slot[C.bids[k]] = (int32_t)k;
    std::vector<double> A((size_t)n * n, 0.0);
    const int bs = C.bs, m = bs - 1;
    for (int64_t k = 0; k < C.n(); ++k) {
        const int64_t b = (int64_t)C.bids[k], bx = b % C.nx, by = (b / C.nx) % C.ny, bz = b / (C.nx * C.ny);
        for (int v = 0; v < bs * bs * bs; ++v) {
            const int cx = v & m, cy = (v >> C.lg) & m, cz = v >> (2 * C.lg);
            const int64_t i = k * bs * bs * bs + v;
            A[(size_t)i * n + i] = 6.0 * C.scale;
            const int dd[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
            for (int f = 0; f < 6; ++f) {
                const int64_t gx = bx * bs + cx + dd[f][0], gy = by * bs + cy + dd[f][1], gz = bz * bs + cz + dd[f][2];
                if (gx < 0 || gy < 0 || gz < 0) continue;
                const int64_t nbx = gx / bs, nby = gy / bs, nbz = gz / bs;
                if (nbx >= C.nx || nby >= C.ny || nbz >= C.nz) continue;
                auto it = slot.find((uint64_t)(nbx + nby * C.nx + nbz * C.nx * C.ny));
                if (it == slot.end()) continue;
                const int64_t j = (int64_t)it->second * bs * bs * bs + ((gx & m) | ((gy & m) << C.lg) | ((gz & m) << (2 * C.lg)));
                A[(size_t)i * n + j] = -1.0 * C.scale;
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
    P->work.reserve((size_t)n0 * (4 * 4 + 8) + (DOT_BLOCKS + 16) * 8 + 1024);
    sync(ctx);
}

static void launch_matvec(msbg_poisson* P, int l, const float* x, float* y) {
    const PLevelDev& L = P->lv[l];
    begin_launch(P->ctx);
    pk_matvec<<<grid_for(L.cells()), 256, 0, P->ctx->stream>>>(level_args(L), x, y);
    after_launch(P->ctx, "pk_matvec");
}

static void launch_residual(msbg_poisson* P, int l, const float* x, const float* b, float* r) {
    const PLevelDev& L = P->lv[l];
    begin_launch(P->ctx);
    pk_residual<<<grid_for(L.cells()), 256, 0, P->ctx->stream>>>(level_args(L), x, b, r);
    after_launch(P->ctx, "pk_residual");
}

// `sweeps` Jacobi sweeps on x (in place through the level's t buffer); x_zero
// marks x as all zeros on entry.
static void jacobi(msbg_poisson* P, int l, float* x, const float* b, int sweeps, float omega, bool x_zero) {
    PLevelDev& L = P->lv[l];
    float* t = L.t.as<float>();
    for (int s = 0; s < sweeps; ++s) {
        const float* src = (s % 2 == 0) ? x : t;
        float* dst = (s % 2 == 0) ? t : x;
        begin_launch(P->ctx);
        pk_jacobi<<<grid_for(L.cells()), 256, 0, P->ctx->stream>>>(level_args(L), (s == 0 && x_zero) ? nullptr : src, b, dst, omega);
        after_launch(P->ctx, "pk_jacobi");
    }
    if (sweeps % 2 == 1) CUDA_CHECK(cudaMemcpyAsync(x, t, L.cells() * 4, cudaMemcpyDeviceToDevice, P->ctx->stream));
}

// One V-cycle on level l: x_l improved for A_l x_l = b_l (x_zero: x_l = 0 on entry).
static void vcycle(msbg_poisson* P, int l, float* x, const float* b, bool x_zero) {
    if (l == (int)P->lv.size() - 1) {
        begin_launch(P->ctx);
        pk_dense_solve<<<grid_for(P->nc), 256, 0, P->ctx->stream>>>(P->ainv.as<double>(), P->nc, b, x);
        after_launch(P->ctx, "pk_dense_solve");
        return;
    }
    PLevelDev& F = P->lv[l];
    PLevelDev& C = P->lv[l + 1];
    jacobi(P, l, x, b, P->nu1, P->omega, x_zero);
    launch_residual(P, l, x, b, F.r.as<float>());
    begin_launch(P->ctx);
    pk_restrict<<<grid_for(C.cells()), 256, 0, P->ctx->stream>>>(P->children[l + 1].slot.as<int32_t>(),
                                                                  P->children[l + 1].v0.as<int32_t>(), F.lg, C.cells(),
                                                                  F.r.as<float>(), C.b.as<float>());
    after_launch(P->ctx, "pk_restrict");
    vcycle(P, l + 1, C.x.as<float>(), C.b.as<float>(), true);
    TransferArgs T{F.coords.as<int32_t>(), F.parent.as<int32_t>(), F.lg, C.lg, F.n()};
    begin_launch(P->ctx);
    pk_prolong<<<grid_for(F.cells()), 256, 0, P->ctx->stream>>>(T, C.x.as<float>(), x);
    after_launch(P->ctx, "pk_prolong");
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
    CUDA_CHECK(cudaMemcpyAsync(&h, part + DOT_BLOCKS, 8, cudaMemcpyDeviceToHost, P->ctx->stream));
    sync(P->ctx);
    return h;
}

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

// method 0: V-cycles (x += V(b - A x)); 1: MG-preconditioned CG.  The solution
// accumulates in FP64 and convergence is judged on the true residual
// b - A x of that FP64 solution; PCG's recursively updated residual is
// replaced by the true one when it reaches the tolerance (and the iteration
// restarts from it if the true residual is still above).  Returns iterations.
static int solve(msbg_poisson* P, int method, float* x, const float* b, double tol, int max_iter, double* rel_out,
                 double* hist) {
    PLevelDev& F = P->lv[0];
    const int64_t n = F.cells();
    float* r = (float*)P->work.p;
    float* z = r + n;
    float* p = z + n;
    float* q = p + n;
    double* x64 = (double*)(q + n);
    const double bn = std::sqrt(dot(P, b, b, n));
    if (bn == 0.0) {
        CUDA_CHECK(cudaMemsetAsync(x, 0, n * 4, P->ctx->stream));
        if (rel_out) *rel_out = 0.0;
        return 0;
    }
    begin_launch(P->ctx);
    pk_widen<<<grid_for(n), 256, 0, P->ctx->stream>>>(n, x, x64);
    after_launch(P->ctx, "pk_widen");
    launch_residual64(P, x64, b, r);
    double rn = std::sqrt(dot(P, r, r, n));
    int it = 0;
    if (method == 0) {
        while (rn > tol * bn && it < max_iter) {
            vcycle(P, 0, z, r, true);
            add64(P, n, 1.0, z, x64);
            launch_residual64(P, x64, b, r);
            rn = std::sqrt(dot(P, r, r, n));
            if (!std::isfinite(rn)) MSBG_THROW(MSBG_ERR_NUMERIC, "multigrid residual is not finite");
            if (hist) hist[it] = rn / bn;
            ++it;
        }
    } else {
        double rz = 0.0;
        auto restart = [&]() {
            vcycle(P, 0, z, r, true);
            CUDA_CHECK(cudaMemcpyAsync(p, z, n * 4, cudaMemcpyDeviceToDevice, P->ctx->stream));
            rz = dot(P, r, z, n);
        };
        restart();
        while (rn > tol * bn && it < max_iter) {
            launch_matvec(P, 0, p, q);
            const double pq = dot(P, p, q, n);
            if (!(pq > 0.0) || !std::isfinite(rz)) MSBG_THROW(MSBG_ERR_NUMERIC, "PCG breakdown (p.Ap <= 0)");
            const double alpha = rz / pq;
            add64(P, n, alpha, p, x64);
            axpby(P, n, -alpha, q, 1.0, r);
            rn = std::sqrt(dot(P, r, r, n));
            ++it;
            if (rn <= tol * bn) {
                launch_residual64(P, x64, b, r);
                rn = std::sqrt(dot(P, r, r, n));
                if (hist) hist[it - 1] = rn / bn;
                if (rn <= tol * bn) break;
                restart();
                continue;
            }
            if (hist) hist[it - 1] = rn / bn;
            vcycle(P, 0, z, r, true);
            const double rz2 = dot(P, r, z, n);
            const double beta = rz2 / rz;
            rz = rz2;
            axpby(P, n, 1.0, z, beta, p);
        }
    }
    begin_launch(P->ctx);
    pk_narrow<<<grid_for(n), 256, 0, P->ctx->stream>>>(n, x64, x);
    after_launch(P->ctx, "pk_narrow");
    if (rel_out) *rel_out = rn / bn;
    return it;
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
    MSBG_REQUIRE(P && d_x && d_b && (method == 0 || method == 1) && max_iter >= 0 && tol > 0.0, "bad argument");
    set_device(P->ctx);
    int it = solve(P, method, d_x, d_b, tol, max_iter, rel_res_out, history);
    if (iters_out) *iters_out = it;
    MSBG_API_END
}

int msbg_poisson_solve(msbg_poisson* P, int method, float* x, const float* b, double tol, int max_iter, int* iters_out,
                       double* rel_res_out, double* history) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(P && x && b && (method == 0 || method == 1) && max_iter >= 0 && tol > 0.0, "bad argument");
    set_device(P->ctx);
    const int64_t n = P->lv[0].cells();
    DevBuf io;
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

}  // extern "C"
