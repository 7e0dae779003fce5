// common.cuh -- runtime shared by every kernel file: status handling, the
// context (stream + scratch arena + launch counter) and small device helpers.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/msbg_cuda.h"

namespace msbg {

// Error carrying an ABI status code; thrown inside the library, converted to a
// status at every extern "C" boundary by MSBG_API_BEGIN/END.
struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const std::string& msg);

#define MSBG_THROW(code, msg) throw ::msbg::Error((code), (msg))
#define MSBG_REQUIRE(cond, msg) \
    do { if (!(cond)) MSBG_THROW(MSBG_ERR_ARG, msg); } while (0)
#define CUDA_CHECK(expr)                                                                  \
    do {                                                                                  \
        cudaError_t e_ = (expr);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            int code_ = (e_ == cudaErrorMemoryAllocation) ? MSBG_ERR_OOM : MSBG_ERR_CUDA; \
            MSBG_THROW(code_, std::string(#expr) + ": " + cudaGetErrorString(e_));        \
        }                                                                                 \
    } while (0)

#define MSBG_API_BEGIN try {
#define MSBG_API_END                                                    \
    }                                                                   \
    catch (const ::msbg::Error& e) {                                    \
        ::msbg::set_last_error(e.what());                               \
        return e.status;                                                \
    }                                                                   \
    catch (const std::bad_alloc&) {                                     \
        ::msbg::set_last_error("host allocation failed");               \
        return MSBG_ERR_OOM;                                            \
    }                                                                   \
    catch (const std::exception& e) {                                   \
        ::msbg::set_last_error(e.what());                               \
        return MSBG_ERR_STATE;                                          \
    }                                                                   \
    return MSBG_OK;

// Device allocation owned by the library (RAII).
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    // Grows to at least `n` bytes; contents are not preserved.
    void reserve(size_t n) {
        if (n <= bytes) return;
        release();
        CUDA_CHECK(cudaMalloc(&p, n));
        bytes = n;
    }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

}  // namespace msbg

// The context: one device, one stream, a scratch arena that grows
// monotonically (kernels that need temporary global memory carve it from
// here), a device status word for bounded waits and a launch counter.
struct msbg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t launches = 0;
    msbg::DevBuf scratch;
    msbg::DevBuf status;  // int32 device status word
    // Page-locked, device-mapped buffer for the library's own small device ->
    // host reads (status words, counts, block lists): a kernel writes them
    // there, so they never queue behind a caller's large transfer on a copy
    // engine.
    void* rb_host = nullptr;
    void* rb_dev = nullptr;
    size_t rb_cap = 0;

    // Per-kernel CUDA-event timing (off by default): every launch between
    // begin_launch and after_launch is bracketed by two events on the stream.
    struct Pending {
        const char* name;
        cudaEvent_t a, b;
    };
    bool timing = false;
    cudaEvent_t open = nullptr;
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    std::unordered_map<std::string, std::pair<uint64_t, double>> totals;  // name -> (launches, ms)
};

namespace msbg {

// Layout of one call's temporaries inside the context scratch arena:
//   ScratchLayout L; size_t a = L.add<T>(n); ...; char* base = scratch(ctx, L);
//   T* pa = L.at<T>(base, a);
struct ScratchLayout {
    size_t size = 0;
    template <class T> size_t add(size_t n) {
        size_t off = (size + 255) & ~size_t(255);
        size = off + n * sizeof(T) + 16;
        return off;
    }
    template <class T> static T* at(char* base, size_t off) { return reinterpret_cast<T*>(base + off); }
};

// Returns the arena base with at least L.size bytes.  Growing synchronises the
// stream first, so kernels still in flight never see their scratch freed.
char* scratch(msbg_ctx* ctx, const ScratchLayout& L);

// Nanoseconds of the GPU's global timer (bounded waits measure with it).
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The device status word collects bits from bounded waits that gave up: 1 =
// an mbarrier wait in a tensor-core kernel, 2 = a radix-sort look-back, 4 = a
// P2G tile-order wait, 8 = a one-launch sweep's wait for its
// neighbours.  Every such wait gives up after kWaitLimitNs.
constexpr uint64_t kWaitLimitNs = 1000000000ull;
// raise_device_status(ctx, word) clears the word and throws when it is
// non-zero; check_device_status reads it (synchronising) and does the same.
void raise_device_status(msbg_ctx* ctx, int word);
void check_device_status(msbg_ctx* ctx);

inline int ilog2i(uint64_t v) { int l = 0; while ((uint64_t(1) << l) < v) ++l; return l; }
inline bool is_pow2(uint64_t v) { return v && !(v & (v - 1)); }
inline unsigned div_up(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

inline cudaEvent_t pooled_event(msbg_ctx* ctx) {
    if (!ctx->pool.empty()) {
        cudaEvent_t e = ctx->pool.back();
        ctx->pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    CUDA_CHECK(cudaEventCreate(&e));
    return e;
}

// Marks the start of a kernel launch (records an event when timing is on).
inline void begin_launch(msbg_ctx* ctx) {
    if (!ctx->timing) return;
    if (!ctx->open) ctx->open = pooled_event(ctx);
    CUDA_CHECK(cudaEventRecord(ctx->open, ctx->stream));
}

// Counts a launch, checks the launch error and closes its timing bracket.
inline void after_launch(msbg_ctx* ctx, const char* what) {
    ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) MSBG_THROW(MSBG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    if (ctx->timing && ctx->open) {
        cudaEvent_t b = pooled_event(ctx);
        CUDA_CHECK(cudaEventRecord(b, ctx->stream));
        ctx->pending.push_back({what, ctx->open, b});
        ctx->open = nullptr;
    }
}

// Folds completed timing brackets into ctx->totals (synchronises).
void resolve_timing(msbg_ctx* ctx);

inline void sync(msbg_ctx* ctx) { CUDA_CHECK(cudaStreamSynchronize(ctx->stream)); }

// Device -> host reads of a few bytes each through the context's mapped
// read-back buffer (a kernel copies them there; no copy engine): add() enqueues
// on the context stream, wait() synchronises the stream and copies the values
// out.  Reads that do not fit in the buffer fall back to cudaMemcpyAsync.
class SmallReads {
  public:
    explicit SmallReads(msbg_ctx* ctx) : ctx_(ctx) {}
    void add(void* host_dst, const void* dev_src, size_t bytes);
    void wait();

  private:
    struct Item {
        void* dst;
        size_t off, bytes;
        bool staged;
    };
    msbg_ctx* ctx_;
    size_t used_ = 0;
    std::vector<Item> items_;
};

// One small read, waited for.
inline void read_small(msbg_ctx* ctx, void* host_dst, const void* dev_src, size_t bytes) {
    SmallReads r(ctx);
    r.add(host_dst, dev_src, bytes);
    r.wait();
}

inline void set_device(msbg_ctx* ctx) { CUDA_CHECK(cudaSetDevice(ctx->device)); }

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------

// Morton interleave: the low 21 bits of v spread to every third bit
// (multires/sort.rs:8-17).
__host__ __device__ inline uint64_t spread3(uint64_t v) {
    v &= 0x1fffffULL;
    v = (v | (v << 32)) & 0x001f00000000ffffULL;
    v = (v | (v << 16)) & 0x001f0000ff0000ffULL;
    v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
    v = (v | (v << 2)) & 0x1249249249249249ULL;
    return v;
}
__host__ __device__ inline uint64_t morton3(uint64_t x, uint64_t y, uint64_t z) {
    return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}
// Inverse of spread3.
__host__ __device__ inline uint64_t compact3(uint64_t v) {
    v &= 0x1249249249249249ULL;
    v = (v | (v >> 2)) & 0x10c30c30c30c30c3ULL;
    v = (v | (v >> 4)) & 0x100f00f00f00f00fULL;
    v = (v | (v >> 8)) & 0x001f0000ff0000ffULL;
    v = (v | (v >> 16)) & 0x001f00000000ffffULL;
    v = (v | (v >> 32)) & 0x1fffffULL;
    return v;
}

// math/boundary.rs:33-56 resolve_axis.  Returns false only for Dirichlet out
// of range.
__host__ __device__ inline bool resolve_axis(int32_t g, int32_t max, int bc, int32_t* out) {
    if (g >= 0 && g <= max) { *out = g; return true; }
    if (bc == MSBG_CLAMP) { *out = g < 0 ? 0 : max; return true; }
    if (bc == MSBG_NEUMANN) {
        int32_t period = 2 * (max + 1);
        int32_t r = g % period;
        if (r < 0) r += period;
        *out = r > max ? period - 1 - r : r;
        return true;
    }
    return false;
}

// Storage element conversions (stencil.rs:142-192 StoreBack and
// sample.rs:45-70 Dequant).
struct ElemF32 {
    using T = float;
    __device__ static float load(T v) { return v; }
    __device__ static T store(float v) { return v; }
};
struct ElemU16 {  // `Density`
    using T = uint16_t;
    __device__ static float load(T v) { return __fmul_rn((float)v, 1.0f / 65535.0f); }
    __device__ static T store(float v) {
        float r = roundf(__fmul_rn(v, 65535.0f));
        r = r > 0.0f ? r : 0.0f;
        r = r < 65535.0f ? r : 65535.0f;
        return (T)r;
    }
};
struct ElemBF16 {
    using T = uint16_t;
    __device__ static float load(T v) { return __uint_as_float((uint32_t)v << 16); }
    __device__ static T store(float v) {
        uint32_t u = __float_as_uint(v);
        if ((u & 0x7fffffffu) > 0x7f800000u) return (T)((u >> 16) | 0x40);
        u += 0x7fffu + ((u >> 16) & 1u);
        return (T)(u >> 16);
    }
};

struct ElemU8 {  // `Density8`: read linearly as q / 255 (sample.rs:64-70)
    using T = uint8_t;
    __device__ static float load(T v) { return __fmul_rn((float)v, 1.0f / 255.0f); }
    // Quant::from_unit (channel.rs:378-382): round(v * 255), saturating
    __device__ static T store(float v) {
        float r = roundf(__fmul_rn(v, 255.0f));
        r = r > 0.0f ? r : 0.0f;
        r = r < 255.0f ? r : 255.0f;
        return (T)r;
    }
};
struct ElemF16 {  // IEEE binary16 bits, store rounds to nearest even
    using T = uint16_t;
    __device__ static float load(T v) { return __half2float(__ushort_as_half(v)); }
    __device__ static T store(float v) { return __half_as_ushort(__float2half_rn(v)); }
};

// The sweep's write-back (StoreBack::store_chunk, stencil.rs:142-192).  Every
// type but Density8 stores deterministically; Density8 compresses with sqrt
// and rounds stochastically against the lane generator's next draw (the
// SimdRng state after its multiply, stencil.rs:125-131, 176-192).  `state`
// is that state for this element's chunk and lane.
template <class E> struct StoreBack {
    __device__ static typename E::T store(float v, uint32_t) { return E::store(v); }
};
template <> struct StoreBack<ElemU8> {
    __device__ static uint8_t store(float v, uint32_t state) {
        const float vf = __fmul_rn(__fsqrt_rn(v), 255.0f);
        const float fl = floorf(vf);
        const float frac = __fsub_rn(vf, fl);
        const float u = __fsub_rn(__uint_as_float((state >> 9) | 0x3f800000u), 1.0f);
        const float r = u < frac ? __fadd_rn(fl, 1.0f) : fl;
        // the float -> i32 conversion of the x86 build (invalid or out of
        // range gives INT_MIN), then the wrapping i32 -> u8 cast
        const int32_t i = (r >= -2147483648.0f && r < 2147483648.0f) ? (int32_t)r : INT32_MIN;
        return (uint8_t)(i & 0xff);
    }
};

// Lane seeds of the stochastic-rounding generator (SimdRng::seed,
// stencil.rs:108-121): a murmur finaliser over seed ^ lane * 0x9e3779b9,
// zero replaced by 0xdeadbeef.
__host__ __device__ inline uint32_t sr_lane_seed(uint32_t seed, uint32_t lane) {
    uint32_t h = seed ^ (lane * 0x9e3779b9u);
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h ? h : 0xdeadbeefu;
}
// 16807^e mod 2^32: the generator state after e draws is seed * 16807^e.
__host__ __device__ inline uint32_t sr_pow(uint64_t e) {
    uint32_t r = 1u, b = 16807u;
    while (e) {
        if (e & 1) r *= b;
        b *= b;
        e >>= 1;
    }
    return r;
}

inline size_t dtype_size(int dtype) { return dtype == MSBG_F32 ? 4 : dtype == MSBG_U8 ? 1 : 2; }

// Host-side conversions of a float constant to the stored representation and
// back (the value a dummy block reads after dequantisation).
float quantize_roundtrip(int dtype, float v);

}  // namespace msbg
