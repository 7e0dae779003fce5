// sweep.cu -- the fused halo-gather + stencil colour phase of the 8-colour
// in-place block smoother (solver.rs:141-267, multires/halo.rs:31-358,
// math/{laplacian,meancurv,bilaplacian}.rs).
//
// One CTA updates one block of the current colour: it stages the block and
// the part of its halo the stencil reads into shared memory (resolving the
// Neumann boundary and dequantising on the way), synchronises, then every
// thread walks one z-column of the block computing the stencil from shared
// memory and writes the result straight back into the block (in place, as
// StoreBack does).  Blocks of one colour never share a halo, so the CTAs of a
// phase are independent; the 8 phases of an iteration are consecutive kernels
// on one stream (block Gauss-Seidel across colours, Jacobi inside a block on
// the staged snapshot, exactly the reference's schedule).
//
// Arithmetic is the reference's operation by operation: this file is built
// with --fmad=false so `a*b+c` is never contracted, and fmaf() appears exactly
// where the reference calls mul_add.  Results are bit-identical to the CPU
// restatement in oracle/.
#include <algorithm>

#include "sweep.cuh"

namespace msbg {

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// laplacian.rs:41-64 (7 taps)
__device__ __forceinline__ float stencil_laplacian(const float* h, int i, int dy, int dz, float dt, int clamp01) {
    float c = h[i], lx = h[i - 1], rx = h[i + 1], dyu = h[i - dy], dyd = h[i + dy], dzb = h[i - dz], dzf = h[i + dz];
    float nb = lx + rx;
    nb = nb + dyu;
    nb = nb + dyd;
    nb = nb + dzb;
    nb = nb + dzf;
    float lap = fmaf(c, -6.0f, nb);
    float fx = (rx - lx) * 0.5f, fy = (dyd - dyu) * 0.5f, fz = (dzf - dzb) * 0.5f;
    float g = sqrtf(fmaf(fx, fx, fmaf(fy, fy, fz * fz)));
    float nv = fmaf(dt * lap, g, c);
    return clamp01 ? clampf(nv, 0.0f, 1.0f) : nv;
}

// meancurv.rs:50-101 (19 taps)
__device__ __forceinline__ float stencil_meancurv(const float* h, int i, int dy, int dz, float dt, int clamp01) {
    float f0 = h[i], f1 = h[i - 1], f2 = h[i + 1], f3 = h[i - dy], f4 = h[i + dy], f5 = h[i - dz], f6 = h[i + dz];
    float fx = (f2 - f1) * 0.5f, fy = (f4 - f3) * 0.5f, fz = (f6 - f5) * 0.5f;
    float fxx = (f1 + f2) - 2.0f * f0, fyy = (f3 + f4) - 2.0f * f0, fzz = (f5 + f6) - 2.0f * f0;
    float d1 = h[i + 1 + dy], d2 = h[i + 1 - dy], d3 = h[i - 1 + dy], d4 = h[i - 1 - dy];
    float d5 = h[i + 1 + dz], d6 = h[i + 1 - dz], d7 = h[i - 1 + dz], d8 = h[i - 1 - dz];
    float d9 = h[i + dy + dz], d10 = h[i + dy - dz], d11 = h[i - dy + dz], d12 = h[i - dy - dz];
    float fyx = (((d1 - d2) - d3) + d4) * 0.25f;
    float fzx = (((d5 - d6) - d7) + d8) * 0.25f;
    float fzy = (((d9 - d10) - d11) + d12) * 0.25f;
    float cross = (fx * (fy * fyx) + fx * (fz * fzx)) + fy * (fz * fzy);
    float hnum = fmaf(fy * fy + fz * fz, fxx, fmaf(fx * fx + fz * fz, fyy, fmaf(fx * fx + fy * fy, fzz, -2.0f * cross)));
    float grad = fmaf(fx, fx, fmaf(fy, fy, fz * fz));
    float hc = grad > 1e-7f ? hnum / grad : 0.0f;
    float d = clampf(dt * hc, -0.1f, 0.1f);
    float nv = f0 + d;
    return clamp01 ? clampf(nv, 0.0f, 1.0f) : nv;
}

// bilaplacian.rs:45-92 (25 taps)
__device__ __forceinline__ float stencil_bilaplacian(const float* h, int i, int dy, int dz, float dt, int clamp01) {
    float f0 = h[i], f1 = h[i - 1], f2 = h[i + 1], f3 = h[i - dy], f4 = h[i + dy], f5 = h[i - dz], f6 = h[i + dz];
    float g1 = h[i - 2], g2 = h[i + 2], g3 = h[i - 2 * dy], g4 = h[i + 2 * dy], g5 = h[i - 2 * dz], g6 = h[i + 2 * dz];
    float s1 = f1 + f2;
    s1 = s1 + f3; s1 = s1 + f4; s1 = s1 + f5; s1 = s1 + f6;
    float s2 = g1 + g2;
    s2 = s2 + g3; s2 = s2 + g4; s2 = s2 + g5; s2 = s2 + g6;
    float sd = h[i + 1 + dy] + h[i + 1 - dy];
    sd = sd + h[i - 1 + dy]; sd = sd + h[i - 1 - dy];
    sd = sd + h[i + 1 + dz]; sd = sd + h[i + 1 - dz];
    sd = sd + h[i - 1 + dz]; sd = sd + h[i - 1 - dz];
    sd = sd + h[i + dy + dz]; sd = sd + h[i + dy - dz];
    sd = sd + h[i - dy + dz]; sd = sd + h[i - dy - dz];
    float hv = ((42.0f * f0 - 12.0f * s1) + s2) + 2.0f * sd;
    float fx = (f2 - f1) * 0.5f, fy = (f4 - f3) * 0.5f, fz = (f6 - f5) * 0.5f;
    float g = sqrtf(fmaf(fx, fx, fmaf(fy, fy, fz * fz)));
    float upd = (dt * hv) * g;
    float d = clampf(-upd, -0.1f, 0.1f);
    float nv = f0 + d;
    return clamp01 ? clampf(nv, 0.0f, 1.0f) : nv;
}

struct SweepArgs {
    void* payload;              // fine payload (grid dtype)
    const float* coarse;        // coarse payload (f32) for multiresolution halos
    const int32_t* nbr;         // [n][27]
    const int32_t* bxyz;        // [n][3]
    int32_t sx, sy, sz;
    float empty, full, dt;
    int clamp01;
};

template <int BSX> struct Lg { static constexpr int v = BSX == 4 ? 2 : BSX == 8 ? 3 : BSX == 16 ? 4 : 5; };

template <class E, int BSX, int ST>
__global__ void __launch_bounds__(BSX * BSX < 32 ? 32 : BSX * BSX)
sweep_phase_kernel(SweepArgs a, const int32_t* __restrict__ order, int n) {
    constexpr int HALO = ST == MSBG_BILAPLACIAN ? 2 : 1;
    constexpr int HSX = BSX + 2 * HALO;
    constexpr int LG = Lg<BSX>::v;
    constexpr int N = BSX * BSX * BSX;
    extern __shared__ float h[];  // HSX^3 staged halo block
    __shared__ int32_t nb[27];
    __shared__ int8_t ok[3][HSX], dd[3][HSX], ll[3][HSX];
    typename E::T* payload = (typename E::T*)a.payload;
    const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarp = nthr >> 5;

    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const int pi = order[t];
        __syncthreads();  // the previous block's compute is done with h
        for (int i = tid; i < 27 + 3 * HSX; i += nthr) {
            if (i < 27) {
                nb[i] = a.nbr[(size_t)pi * 27 + i];
            } else {
                int ax = (i - 27) / HSX, hh = (i - 27) % HSX;
                int32_t smax = ax == 0 ? a.sx : ax == 1 ? a.sy : a.sz;
                int32_t b0 = a.bxyz[(size_t)pi * 3 + ax];
                int32_t g = b0 * BSX + hh - HALO, r;
                bool o = resolve_axis(g, smax - 1, MSBG_NEUMANN, &r);  // solver.rs:205-209
                ok[ax][hh] = o;
                dd[ax][hh] = (int8_t)((r >> LG) - b0 + 1);
                ll[ax][hh] = (int8_t)(r & (BSX - 1));
            }
        }
        __syncthreads();
        // Stage the halo block: one warp per (hz, hy) row, lanes along x.
        for (int r = warp; r < HSX * HSX; r += nwarp) {
            const int hz = r / HSX, hy = r % HSX;
            const bool midy = hy >= HALO && hy < HALO + BSX, midz = hz >= HALO && hz < HALO + BSX;
            for (int hx = lane; hx < HSX; hx += 32) {
                const bool midx = hx >= HALO && hx < HALO + BSX;
                const int nout = (!midx) + (!midy) + (!midz);
                bool need;
                if (ST == MSBG_LAPLACIAN) {
                    need = nout <= 1;
                } else if (ST == MSBG_MEAN_CURVATURE) {
                    need = nout <= 2;
                } else {
                    const bool d1x = hx == HALO - 1 || hx == HALO + BSX, d1y = hy == HALO - 1 || hy == HALO + BSX,
                               d1z = hz == HALO - 1 || hz == HALO + BSX;
                    need = nout <= 1 || (nout == 2 && (midx || d1x) && (midy || d1y) && (midz || d1z));
                }
                if (!need) continue;
                float v = a.empty;
                if (ok[0][hx] && ok[1][hy] && ok[2][hz]) {
                    const int c = nb[dd[0][hx] + 3 * dd[1][hy] + 9 * dd[2][hz]];
                    const int lx = ll[0][hx], ly = ll[1][hy], lz = ll[2][hz];
                    if (c >= 0) {
                        v = E::load(payload[(size_t)c * N + (lx | (ly << LG) | (lz << (2 * LG)))]);
                    } else if (c == kCodeFull) {
                        v = a.full;
                    } else if (c <= kCodeCoarse0) {
                        constexpr int CLG = LG - 1;
                        const int cs = kCodeCoarse0 - c;
                        v = a.coarse[(size_t)cs * (N / 8) + ((lx >> 1) | ((ly >> 1) << CLG) | ((lz >> 1) << (2 * CLG)))];
                    }
                }
                h[(hz * HSX + hy) * HSX + hx] = v;
            }
        }
        __syncthreads();
        if (tid < BSX * BSX) {
            const int x = tid % BSX, y = tid / BSX;
            const int slot = nb[13];
            typename E::T* out = payload + (size_t)slot * N + x + y * BSX;
#pragma unroll 4
            for (int z = 0; z < BSX; ++z) {
                const int i = ((z + HALO) * HSX + (y + HALO)) * HSX + (x + HALO);
                float v;
                if (ST == MSBG_LAPLACIAN) v = stencil_laplacian(h, i, HSX, HSX * HSX, a.dt, a.clamp01);
                else if (ST == MSBG_MEAN_CURVATURE) v = stencil_meancurv(h, i, HSX, HSX * HSX, a.dt, a.clamp01);
                else v = stencil_bilaplacian(h, i, HSX, HSX * HSX, a.dt, a.clamp01);
                out[z * BSX * BSX] = E::store(v);
            }
        }
    }
}

template <class E, int BSX, int ST>
static void launch_phase(msbg_ctx* ctx, const SweepArgs& a, const int32_t* order, int n) {
    constexpr int HALO = ST == MSBG_BILAPLACIAN ? 2 : 1;
    constexpr int HSX = BSX + 2 * HALO;
    const size_t smem = sizeof(float) * HSX * HSX * HSX;
    static bool attr_set = false;  // per instantiation
    if (!attr_set) {
        CUDA_CHECK(cudaFuncSetAttribute(sweep_phase_kernel<E, BSX, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set = true;
    }
    const int threads = BSX * BSX < 32 ? 32 : BSX * BSX;
    begin_launch(ctx);
    sweep_phase_kernel<E, BSX, ST><<<(unsigned)n, threads, smem, ctx->stream>>>(a, order, n);
    after_launch(ctx, "sweep_phase_kernel");
}

template <class E, int BSX>
static void launch_phase_st(msbg_ctx* ctx, int st, const SweepArgs& a, const int32_t* order, int n) {
    if (st == MSBG_LAPLACIAN) launch_phase<E, BSX, MSBG_LAPLACIAN>(ctx, a, order, n);
    else if (st == MSBG_MEAN_CURVATURE) launch_phase<E, BSX, MSBG_MEAN_CURVATURE>(ctx, a, order, n);
    else launch_phase<E, BSX, MSBG_BILAPLACIAN>(ctx, a, order, n);
}

template <class E>
static void launch_phase_bsx(msbg_ctx* ctx, int bsx, int st, const SweepArgs& a, const int32_t* order, int n) {
    switch (bsx) {
        case 4: launch_phase_st<E, 4>(ctx, st, a, order, n); break;
        case 8: launch_phase_st<E, 8>(ctx, st, a, order, n); break;
        case 16: launch_phase_st<E, 16>(ctx, st, a, order, n); break;
        default: launch_phase_st<E, 32>(ctx, st, a, order, n); break;
    }
}

static uint64_t fnv(uint64_t h, uint64_t v) {
    for (int i = 0; i < 8; ++i) { h ^= (v >> (8 * i)) & 0xff; h *= 0x100000001b3ULL; }
    return h;
}

// Builds (or reuses) the plan for `active` on grid g (and coarse + levels for
// a multiresolution sweep).
static SweepPlan* get_plan(msbg_grid* g, msbg_grid* coarse, const uint8_t* levels, const uint64_t* active, size_t n) {
    uint64_t key = 0xcbf29ce484222325ULL;
    key = fnv(key, n);
    key = fnv(key, g->version);
    key = fnv(key, (uint64_t)(uintptr_t)coarse);
    if (coarse) {
        key = fnv(key, coarse->version);
        key = fnv(key, coarse->n_slots());
        for (uint64_t b = 0; b < g->n_blocks; b += 1) key = fnv(key, levels[b]);
    }
    for (size_t k = 0; k < n; ++k) key = fnv(key, active[k]);
    if (g->plan && g->plan->key == key) return g->plan;

    std::vector<std::vector<uint64_t>> buckets(8);
    std::unordered_map<uint64_t, char> seen;
    for (size_t k = 0; k < n; ++k) {
        uint64_t bid = active[k];
        MSBG_REQUIRE(bid < g->n_blocks, "active block id out of range");
        if (grid_code(g, bid) < 0) continue;  // dummy or absent: skipped (solver.rs:196-199)
        if (!seen.emplace(bid, 1).second) continue;
        int64_t bx, by, bz;
        block_coords(g, bid, &bx, &by, &bz);
        buckets[(bx & 1) | ((by & 1) << 1) | ((bz & 1) << 2)].push_back(bid);
    }
    auto plan = new SweepPlan;
    plan->key = key;
    std::vector<int32_t> nbr, bxyz, order;
    int32_t pi = 0;
    for (int c = 0; c < 8; ++c) {
        auto& bk = buckets[c];
        std::stable_sort(bk.begin(), bk.end(), [&](uint64_t a, uint64_t b) {
            int64_t ax, ay, az, bx, by, bz;
            block_coords(g, a, &ax, &ay, &az);
            block_coords(g, b, &bx, &by, &bz);
            return morton3(ax, ay, az) < morton3(bx, by, bz);
        });
        plan->color_off[c] = pi;
        for (uint64_t bid : bk) {
            int64_t bx, by, bz;
            block_coords(g, bid, &bx, &by, &bz);
            bxyz.push_back((int32_t)bx);
            bxyz.push_back((int32_t)by);
            bxyz.push_back((int32_t)bz);
            for (int k = 0; k < 27; ++k) {
                int64_t X = bx + k % 3 - 1, Y = by + (k / 3) % 3 - 1, Z = bz + k / 9 - 1;
                int32_t code = kCodeEmpty;
                if (X >= 0 && Y >= 0 && Z >= 0 && X < (int64_t)g->nx && Y < (int64_t)g->ny && Z < (int64_t)g->nz) {
                    uint64_t nbid = (uint64_t)X + (uint64_t)Y * g->nx + (uint64_t)Z * g->nxy;
                    if (coarse && levels[nbid] > levels[bid]) {
                        int32_t cs = grid_code(coarse, nbid);
                        code = cs >= 0 ? kCodeCoarse0 - cs : kCodeEmpty;
                    } else {
                        code = grid_code(g, nbid);
                        if (coarse && code == kCodeFull) code = kCodeEmpty;
                    }
                }
                nbr.push_back(code);
            }
            order.push_back(pi++);
        }
    }
    plan->color_off[8] = pi;
    plan->n = (size_t)pi;
    if (pi) {
        plan->nbr.reserve(nbr.size() * 4);
        plan->bxyz.reserve(bxyz.size() * 4);
        plan->order.reserve(order.size() * 4);
        CUDA_CHECK(cudaMemcpyAsync(plan->nbr.p, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice, g->ctx->stream));
        CUDA_CHECK(cudaMemcpyAsync(plan->bxyz.p, bxyz.data(), bxyz.size() * 4, cudaMemcpyHostToDevice, g->ctx->stream));
        CUDA_CHECK(cudaMemcpyAsync(plan->order.p, order.data(), order.size() * 4, cudaMemcpyHostToDevice, g->ctx->stream));
        sync(g->ctx);
    }
    delete g->plan;
    g->plan = plan;
    return plan;
}

static void sweep(msbg_grid* g, msbg_grid* coarse, const uint8_t* levels, const uint64_t* active, size_t n, int stencil,
                  float dt, int iterations, int clamp01) {
    MSBG_REQUIRE(stencil >= 0 && stencil <= 2, "bad stencil");
    MSBG_REQUIRE(iterations >= 0, "negative iteration count");
    MSBG_REQUIRE(g->bsx >= 4, "sweeps need bsx >= 4");
    if (coarse) {
        MSBG_REQUIRE(g->dtype == MSBG_F32 && coarse->dtype == MSBG_F32, "multiresolution sweep needs f32 levels");
        MSBG_REQUIRE(coarse->bsx * 2 == g->bsx && coarse->nx == g->nx && coarse->ny == g->ny && coarse->nz == g->nz,
                     "coarse level must have half the block size on the same block grid");
        MSBG_REQUIRE(levels, "null levels");
    }
    set_device(g->ctx);
    SweepPlan* plan = get_plan(g, coarse, levels, active, n);
    if (!plan->n || !iterations) return;
    SweepArgs a;
    a.payload = g->payload.p;
    a.coarse = coarse ? coarse->payload.as<float>() : nullptr;
    a.nbr = plan->nbr.as<int32_t>();
    a.bxyz = plan->bxyz.as<int32_t>();
    a.sx = (int32_t)g->sx; a.sy = (int32_t)g->sy; a.sz = (int32_t)g->sz;
    a.empty = coarse ? 0.0f : quantize_roundtrip(g->dtype, g->empty_value);
    a.full = coarse ? 0.0f : quantize_roundtrip(g->dtype, g->full_value);
    a.dt = dt;
    a.clamp01 = clamp01 ? 1 : 0;
    const int32_t* order = plan->order.as<int32_t>();
    for (int it = 0; it < iterations; ++it)
        for (int c = 0; c < 8; ++c) {
            int cnt = plan->color_off[c + 1] - plan->color_off[c];
            if (!cnt) continue;
            const int32_t* o = order + plan->color_off[c];
            if (g->dtype == MSBG_F32) launch_phase_bsx<ElemF32>(g->ctx, g->bsx, stencil, a, o, cnt);
            else if (g->dtype == MSBG_U16) launch_phase_bsx<ElemU16>(g->ctx, g->bsx, stencil, a, o, cnt);
            else launch_phase_bsx<ElemBF16>(g->ctx, g->bsx, stencil, a, o, cnt);
        }
}

}  // namespace msbg

using namespace msbg;

extern "C" {

int msbg_sweep(msbg_grid* g, const uint64_t* active, size_t n, int stencil, float dt, int iterations, int clamp01) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(g && (active || !n), "null argument");
    sweep(g, nullptr, nullptr, active, n, stencil, dt, iterations, clamp01);
    MSBG_API_END
}

int msbg_sweep_multires(msbg_grid* fine, msbg_grid* coarse, const uint8_t* levels, const uint64_t* active, size_t n,
                        int stencil, float dt, int iterations, int clamp01) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(fine && coarse && (active || !n), "null argument");
    MSBG_REQUIRE(fine->ctx == coarse->ctx, "levels on different contexts");
    sweep(fine, coarse, levels, active, n, stencil, dt, iterations, clamp01);
    MSBG_API_END
}

}  // extern "C"
