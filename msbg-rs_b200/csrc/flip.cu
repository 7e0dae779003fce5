// flip.cu -- one FLIP transfer step through host arrays: the composition of
// the crate's transfer entry points that a simulation loop makes per step
// (bucket/sort the particles, particles_to_grid, smooth, MacSampler::sample
// + g2p_blend; fluid/p2g.rs:141-164, solver.rs:166-185, fluid/g2p.rs:15-45),
// with the host-device copies inside the call.
//
// The step keeps its device arrays between calls (sized for the largest n
// seen).  The positions go up first on the context stream; the velocities and
// masses go up on a second stream while the positions are sorted.  P2G reads
// the particles in the caller's order through the sort's permutation
// (msbg_p2g_permuted_device), and G2P and the blend run in the caller's
// order, so vel_out[i] belongs to input particle i and no particle array is
// ever permuted.
#include <algorithm>

#include "mac.cuh"
#include "sort.cuh"

struct msbg_flip {
    msbg_mac* mac = nullptr;
    msbg_grid* coarse = nullptr;
    std::vector<uint8_t> levels;  // per block of the MAC grid
    cudaStream_t up = nullptr;    // second upload stream
    cudaEvent_t start = nullptr, uploaded = nullptr, downloaded = nullptr;
    static constexpr int kOutChunks = 8;  // G2P chunks whose results return while the next computes
    cudaEvent_t chunk_done[kOutChunks] = {};
    msbg::DevBuf buf;
    size_t cap = 0;
    std::vector<uint64_t> fine;
    ~msbg_flip() {
        if (start) cudaEventDestroy(start);
        if (uploaded) cudaEventDestroy(uploaded);
        if (downloaded) cudaEventDestroy(downloaded);
        for (cudaEvent_t ev : chunk_done)
            if (ev) cudaEventDestroy(ev);
        if (up) cudaStreamDestroy(up);
    }
};

namespace msbg {

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
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f->downloaded, cudaEventDisableTiming);
    for (int c = 0; c < msbg_flip::kOutChunks && e == cudaSuccess; ++c)
        e = cudaEventCreateWithFlags(&f->chunk_done[c], cudaEventDisableTiming);
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
        f->buf.reserve(3 * b3 + 2 * b1 + b8);
        f->cap = n;
    }
    char* p = (char*)f->buf.p;
    float* d_pos = (float*)p;  p += b3;
    float* d_vel = (float*)p;  p += b3;
    float* d_out = (float*)p;  p += b3;
    float* d_mass = (float*)p; p += b1;
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
    CUDA_CHECK(cudaStreamWaitEvent(ctx->stream, f->uploaded, 0));
    check(msbg_p2g_permuted_device(f->mac, d_pos, d_vel, d_mass, keys, perm, n, r_p, nullptr));
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
    // G2P and the blend per particle in the caller's order (unsorted
    // positions and velocities: the same values as the sorted pass, and the
    // grid, a few tens of MB, sits in L2), in chunks whose new velocities
    // return to the host on the upload stream while the next chunk computes
    const size_t per = ((n + msbg_flip::kOutChunks - 1) / msbg_flip::kOutChunks + 255) & ~size_t(255);
    int used = 0;
    for (size_t lo = 0; lo < n; lo += per, ++used) {
        const size_t cnt = std::min(per, n - lo);
        check(msbg_g2p_flip_device(f->mac, d_pos + 3 * lo, cnt, MSBG_CLAMP, d_vel + 3 * lo, nullptr, alpha, d_out + 3 * lo));
        CUDA_CHECK(cudaEventRecord(f->chunk_done[used], ctx->stream));
        CUDA_CHECK(cudaStreamWaitEvent(f->up, f->chunk_done[used], 0));
        CUDA_CHECK(cudaMemcpyAsync(vel_out + 3 * lo, d_out + 3 * lo, cnt * 12, cudaMemcpyDeviceToHost, f->up));
    }
    CUDA_CHECK(cudaEventRecord(f->downloaded, f->up));
    CUDA_CHECK(cudaStreamWaitEvent(ctx->stream, f->downloaded, 0));
    check_device_status(ctx);
    sync(ctx);
    MSBG_API_END
}

}  // extern "C"
