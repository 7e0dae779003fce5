// flip.cu -- one FLIP transfer step through host arrays: the composition of
// the crate's transfer entry points that a simulation loop makes per step
// (bucket/sort the particles, particles_to_grid, smooth, MacSampler::sample
// + g2p_blend; fluid/p2g.rs:141-164, solver.rs:166-185, fluid/g2p.rs:15-45),
// with the host-device copies inside the call.
//
// The step keeps its device arrays between calls (sized for the largest n
// seen).  The positions go up first on the context stream; the velocities and
// masses go up on a second stream while the positions are sorted, and the
// sort's permutation is applied to them once they have arrived.  The new
// velocities are scattered back to the caller's particle order on the device,
// so vel_out[i] belongs to input particle i.
#include <algorithm>

#include "mac.cuh"
#include "sort.cuh"

struct msbg_flip {
    msbg_mac* mac = nullptr;
    msbg_grid* coarse = nullptr;
    std::vector<uint8_t> levels;  // per block of the MAC grid
    cudaStream_t up = nullptr;    // second upload stream
    cudaEvent_t start = nullptr, uploaded = nullptr;
    msbg::DevBuf buf;
    size_t cap = 0;
    std::vector<uint64_t> fine;
    ~msbg_flip() {
        if (start) cudaEventDestroy(start);
        if (uploaded) cudaEventDestroy(uploaded);
        if (up) cudaStreamDestroy(up);
    }
};

namespace msbg {

// dst[perm[i]] = src[i] for rows of 3 floats (the inverse of the sort's gather).
__global__ void scatter_rows3_kernel(const uint32_t* __restrict__ perm, size_t n, const float* __restrict__ src,
                                     float* __restrict__ dst) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t d = perm[i];
        dst[3 * d] = src[3 * i];
        dst[3 * d + 1] = src[3 * i + 1];
        dst[3 * d + 2] = src[3 * i + 2];
    }
}

static void check(int st) {
    if (st != MSBG_OK) MSBG_THROW(st, msbg_last_error());
}

}  // namespace msbg

using namespace msbg;

extern "C" {

int msbg_flip_create(msbg_mac* mac, msbg_grid* coarse, const uint8_t* levels, size_t n_levels, msbg_flip** out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(mac && coarse && levels && out, "null argument");
    MSBG_REQUIRE(coarse->ctx == mac->ctx, "coarse grid on another context");
    msbg_grid* u = mac->ch[3];
    MSBG_REQUIRE(coarse->bsx * 2 == u->bsx, "the coarse grid must have half the block size of the MAC grid");
    MSBG_REQUIRE(n_levels == u->n_blocks, "levels must hold one entry per block of the MAC grid");
    set_device(mac->ctx);
    auto* f = new msbg_flip();
    f->mac = mac;
    f->coarse = coarse;
    f->levels.assign(levels, levels + n_levels);
    cudaError_t e = cudaStreamCreateWithFlags(&f->up, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f->start, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f->uploaded, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        delete f;
        MSBG_THROW(MSBG_ERR_CUDA, std::string("msbg_flip_create: ") + cudaGetErrorString(e));
    }
    *out = f;
    MSBG_API_END
}

int msbg_flip_destroy(msbg_flip* f) {
    MSBG_API_BEGIN
    if (f) {
        set_device(f->mac->ctx);
        sync(f->mac->ctx);
        delete f;
    }
    MSBG_API_END
}

int msbg_flip_step(msbg_flip* f, const float* pos, const float* vel, const float* mass, size_t n, float r_p, int stencil,
                   float dt, int sweeps, float alpha, float* vel_out) {
    MSBG_API_BEGIN
    MSBG_REQUIRE(f && ((pos && vel && mass && vel_out) || !n), "null argument");
    MSBG_REQUIRE(n < (1ULL << 31), "msbg_flip_step supports < 2^31 particles");
    msbg_ctx* ctx = f->mac->ctx;
    set_device(ctx);
    if (!n) return MSBG_OK;
    const size_t b3 = (n * 12 + 255) & ~size_t(255), b1 = (n * 4 + 255) & ~size_t(255), b8 = (n * 8 + 255) & ~size_t(255);
    if (n > f->cap) {
        sync(ctx);
        f->buf.release();
        f->buf.reserve(8 * b3 + 2 * b1 + b8 + b1);
        f->cap = n;
    }
    char* p = (char*)f->buf.p;
    float* d_pos = (float*)p;  p += b3;
    float* d_vel = (float*)p;  p += b3;
    float* s_pos = (float*)p;  p += b3;
    float* s_vel = (float*)p;  p += b3;
    float* d_u = (float*)p;    p += b3;
    float* d_new = (float*)p;  p += b3;
    float* d_out = (float*)p;  p += b3;
    p += b3;  // spare row buffer (keeps the layout 256-byte aligned for any n)
    float* d_mass = (float*)p; p += b1;
    float* s_mass = (float*)p; p += b1;
    uint64_t* keys = (uint64_t*)p; p += b8;
    uint32_t* perm = (uint32_t*)p;
    // positions on the context stream; velocities and masses beside the sort
    CUDA_CHECK(cudaMemcpyAsync(d_pos, pos, n * 12, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_CHECK(cudaEventRecord(f->start, ctx->stream));
    CUDA_CHECK(cudaStreamWaitEvent(f->up, f->start, 0));
    CUDA_CHECK(cudaMemcpyAsync(d_vel, vel, n * 12, cudaMemcpyHostToDevice, f->up));
    CUDA_CHECK(cudaMemcpyAsync(d_mass, mass, n * 4, cudaMemcpyHostToDevice, f->up));
    CUDA_CHECK(cudaEventRecord(f->uploaded, f->up));
    check(msbg_morton_sort_device(ctx, d_pos, n, keys, perm));
    check(msbg_permute_device(ctx, perm, n, 3, d_pos, s_pos));
    CUDA_CHECK(cudaStreamWaitEvent(ctx->stream, f->uploaded, 0));
    check(msbg_permute_device(ctx, perm, n, 3, d_vel, s_vel));
    check(msbg_permute_device(ctx, perm, n, 1, d_mass, s_mass));
    check(msbg_p2g_sorted_device(f->mac, s_pos, s_vel, s_mass, keys, n, r_p, nullptr));
    // smooth the x-face mass over the level-0 blocks of the new active set,
    // halos of coarser neighbours sampled from its 2^3 downsample
    f->fine.clear();
    for (uint64_t b : f->mac->active)
        if (b < f->levels.size() && f->levels[b] == 0) f->fine.push_back(b);
    if (sweeps > 0) {
        check(msbg_downsample_avg(f->coarse, f->mac->ch[3]));
        check(msbg_sweep_multires(f->mac->ch[3], f->coarse, f->levels.data(), f->fine.data(), f->fine.size(), stencil, dt,
                                  sweeps, 0));
    }
    check(msbg_g2p_device(f->mac, s_pos, n, MSBG_CLAMP, d_u));
    check(msbg_g2p_blend_device(ctx, s_vel, d_u, d_u, n, alpha, d_new));
    begin_launch(ctx);
    scatter_rows3_kernel<<<std::min<unsigned>(div_up(n, 256), 148 * 32), 256, 0, ctx->stream>>>(perm, n, d_new, d_out);
    after_launch(ctx, "scatter_rows3_kernel");
    CUDA_CHECK(cudaMemcpyAsync(vel_out, d_out, n * 12, cudaMemcpyDeviceToHost, ctx->stream));
    check_device_status(ctx);
    sync(ctx);
    MSBG_API_END
}

}  // extern "C"
