// Common device/host helpers for the B200 PDHG library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>

namespace vk {

// Host-side error types. The C ABI maps them to status codes; nothing throws
// across the ABI.
struct CudaFailure : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct InvalidInput : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};
struct Unsupported : std::runtime_error {
    using std::runtime_error::runtime_error;
};

[[noreturn]] inline void throw_cuda(cudaError_t e, const char *what, const char *file, int line) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "CUDA error %s (%d) at %s:%d in %s", cudaGetErrorString(e),
                  static_cast<int>(e), file, line, what);
    throw CudaFailure(buf);
}

#define VK_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t vk_e_ = (call);                                                        \
        if (vk_e_ != cudaSuccess) ::vk::throw_cuda(vk_e_, #call, __FILE__, __LINE__);      \
    } while (0)

#define VK_LAUNCH_CHECK() VK_CUDA(cudaGetLastError())

// Owning device buffer (cudaMalloc / cudaFree). Size in elements.
template <class T>
class DevBuf {
public:
    DevBuf() = default;
    explicit DevBuf(size_t n) { reset(n); }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p_(std::exchange(o.p_, nullptr)), n_(std::exchange(o.n_, 0)) {}
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) {
            release();
            p_ = std::exchange(o.p_, nullptr);
            n_ = std::exchange(o.n_, 0);
        }
        return *this;
    }
    void reset(size_t n) {
        release();
        if (n > 0) VK_CUDA(cudaMalloc(reinterpret_cast<void **>(&p_), n * sizeof(T)));
        n_ = n;
    }
    void release() noexcept {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    T *get() const noexcept { return p_; }
    size_t size() const noexcept { return n_; }
    size_t bytes() const noexcept { return n_ * sizeof(T); }

private:
    T *p_ = nullptr;
    size_t n_ = 0;
};

// Pinned host buffer.
template <class T>
class HostBuf {
public:
    HostBuf() = default;
    explicit HostBuf(size_t n) { reset(n); }
    ~HostBuf() { release(); }
    HostBuf(const HostBuf &) = delete;
    HostBuf &operator=(const HostBuf &) = delete;
    void reset(size_t n) {
        release();
        if (n > 0) VK_CUDA(cudaMallocHost(reinterpret_cast<void **>(&p_), n * sizeof(T)));
        n_ = n;
    }
    void release() noexcept {
        if (p_) cudaFreeHost(p_);
        p_ = nullptr;
        n_ = 0;
    }
    T *get() const noexcept { return p_; }
    T &operator[](size_t i) const noexcept { return p_[i]; }
    size_t size() const noexcept { return n_; }

private:
    T *p_ = nullptr;
    size_t n_ = 0;
};

inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// Device helpers with the reference's std:: semantics.
//   std::max(a, b) == (a < b) ? b : a      (NaN in b is ignored, NaN in a kept)
//   std::min(a, b) == (b < a) ? b : a
//   project_box: std::min(std::max(x, lo), hi)   (cpu_ops.cpp:382; NaN passes)
// ---------------------------------------------------------------------------
template <class T>
__host__ __device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }
template <class T>
__host__ __device__ __forceinline__ T smin(T a, T b) { return (b < a) ? b : a; }
template <class T>
__host__ __device__ __forceinline__ T clampbox(T x, T lo, T hi) { return smin(smax(x, lo), hi); }

// Atomic max for non-negative doubles through their bit patterns (monotone for
// x >= 0, +inf included). NaN is skipped, as std::max(result, NaN) keeps result.
__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
    if (!(v >= 0.0)) return;
    atomicMax(reinterpret_cast<unsigned long long *>(addr),
              static_cast<unsigned long long>(__double_as_longlong(v)));
}

// ---------------------------------------------------------------------------
// mbarrier + 1-D bulk copy (TMA, non-tensor) helpers, sm_90+ PTX.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// Makes barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Orders this thread's generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) writes to the same buffer.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase of `bar` with the given parity, giving up after
// `limit` polls (each poll may suspend the thread briefly). Returns false on
// timeout: the caller records an error and leaves.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t limit = 1u << 24) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// Bulk copy of `bytes` (multiple of 16; both addresses 16-byte aligned) from
// global to this CTA's shared memory, completing on `bar` as tx bytes.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Codes a kernel writes to the device error flag (first one wins).
enum DeviceError : int { kDevErrNone = 0, kDevErrBarrierTimeout = 1 };

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max_nonneg(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = smax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum of NR doubles; result valid in thread 0. `scratch` holds
// 32*NR doubles of shared memory. Fixed tree: deterministic for a fixed
// blockDim.
template <int NR>
__device__ __forceinline__ void block_sum(double (&v)[NR], double *scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int r = 0; r < NR; ++r) v[r] = warp_sum(v[r]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int r = 0; r < NR; ++r) scratch[warp * NR + r] = v[r];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            double t = lane < nw ? scratch[lane * NR + r] : 0.0;
            v[r] = warp_sum(t);
        }
    }
}

__device__ __forceinline__ double block_max_nonneg(double v, double *scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = warp_max_nonneg(v);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double t = lane < nw ? scratch[lane] : 0.0;
        v = warp_max_nonneg(t);
    }
    return v;
}

} // namespace vk
