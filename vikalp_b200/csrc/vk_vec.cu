// Vector reductions of the ExecutionBackend contract on device arrays:
// dot (ExecutionBackend.hpp:49-50, cuda_ops.cu:407-430) and norm_inf
// (ExecutionBackend.hpp:51, cuda_ops.cu:432-451). The reference finishes both
// on the host after a device-to-host copy of block partials; here a second
// one-block kernel finishes on the device, in a fixed order, so the result is
// deterministic and stays on the GPU (the caller reads it when it needs it).
#include "vk_vec.cuh"

#include <mutex>

namespace vk {

__global__ void __launch_bounds__(kReduceThreads)
    dot_partials_kernel(const double *__restrict__ x, const double *__restrict__ y, int64_t n,
                        double *__restrict__ partials) {
    __shared__ double scratch[32];
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kReduceChunk;
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < kReducePerThread; ++j) {
        const int64_t i = base + static_cast<int64_t>(j) * kReduceThreads + threadIdx.x;
        if (i < n) s += x[i] * y[i];
    }
    double v[1] = {s};
    block_sum<1>(v, scratch);
    if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

__global__ void __launch_bounds__(kReduceThreads)
    absmax_partials_kernel(const double *__restrict__ x, int64_t n, double *__restrict__ partials) {
    __shared__ double scratch[32];
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kReduceChunk;
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < kReducePerThread; ++j) {
        const int64_t i = base + static_cast<int64_t>(j) * kReduceThreads + threadIdx.x;
        if (i < n) s = smax(s, fabs(x[i]));
    }
    s = block_max_nonneg(s, scratch);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kReduceThreads)
    finish_sum_kernel(const double *__restrict__ partials, int count, double *__restrict__ result) {
    __shared__ double scratch[32];
    double s = 0.0;
    for (int t = threadIdx.x; t < count; t += kReduceThreads) s += partials[t];
    double v[1] = {s};
    block_sum<1>(v, scratch);
    if (threadIdx.x == 0) *result = v[0];
}

__global__ void __launch_bounds__(kReduceThreads)
    finish_max_kernel(const double *__restrict__ partials, int count, double *__restrict__ result) {
    __shared__ double scratch[32];
    double s = 0.0;
    for (int t = threadIdx.x; t < count; t += kReduceThreads) s = smax(s, partials[t]);
    s = block_max_nonneg(s, scratch);
    if (threadIdx.x == 0) *result = s;
}

namespace {

struct Scratch {
    double *p = nullptr;
    int64_t cap = 0;
};

std::mutex g_scratch_mu;
Scratch g_scratch[64];

} // namespace

// Per-device partials buffer, grown on demand (cudaMalloc), kept until exit --
// the reference CUDA backend's reduction workspace (cuda_ops.cu:654-664).
double *reduction_scratch(int64_t blocks) {
    int dev = 0;
    VK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw CudaFailure("device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    Scratch &s = g_scratch[dev];
    if (s.cap < blocks) {
        double *p = nullptr;
        VK_CUDA(cudaMalloc(&p, static_cast<size_t>(blocks) * sizeof(double)));
        if (s.p) cudaFree(s.p);
        s.p = p;
        s.cap = blocks;
    }
    return s.p;
}

void launch_dot(const double *x, const double *y, int64_t n, double *partials, double *result, cudaStream_t s) {
    const int blocks = reduction_blocks(n);
    if (n > 0) {
        dot_partials_kernel<<<blocks, kReduceThreads, 0, s>>>(x, y, n, partials);
        VK_LAUNCH_CHECK();
    }
    finish_sum_kernel<<<1, kReduceThreads, 0, s>>>(partials, n > 0 ? blocks : 0, result);
    VK_LAUNCH_CHECK();
}

void launch_norm_inf(const double *x, int64_t n, double *partials, double *result, cudaStream_t s) {
    const int blocks = reduction_blocks(n);
    if (n > 0) {
        absmax_partials_kernel<<<blocks, kReduceThreads, 0, s>>>(x, n, partials);
        VK_LAUNCH_CHECK();
    }
    finish_max_kernel<<<1, kReduceThreads, 0, s>>>(partials, n > 0 ? blocks : 0, result);
    VK_LAUNCH_CHECK();
}

} // namespace vk
