// Device vector reductions (dot, infinity norm) shared by the C-ABI entry
// points: one block per kReduceChunk elements writes a partial, one block
// sums the partials in a fixed order.
#pragma once

#include "vk_common.cuh"

namespace vk {

constexpr int kReduceThreads = 256;
constexpr int kReducePerThread = 8;
constexpr int64_t kReduceChunk = static_cast<int64_t>(kReduceThreads) * kReducePerThread; // elements per block

inline int reduction_blocks(int64_t n) { return static_cast<int>((n + kReduceChunk - 1) / kReduceChunk); }

// partials[b] = sum over block b's chunk of x[i] * y[i].
__global__ void __launch_bounds__(kReduceThreads)
    dot_partials_kernel(const double *__restrict__ x, const double *__restrict__ y, int64_t n,
                        double *__restrict__ partials);
// partials[b] = max over block b's chunk of |x[i]| (NaN ignored, as std::max
// in the reference's norm_inf, cpu_ops.cpp:358-364).
__global__ void __launch_bounds__(kReduceThreads)
    absmax_partials_kernel(const double *__restrict__ x, int64_t n, double *__restrict__ partials);
// *result = sum (max) of partials[0 .. count), fixed order; 0 when count == 0.
__global__ void __launch_bounds__(kReduceThreads)
    finish_sum_kernel(const double *__restrict__ partials, int count, double *__restrict__ result);
__global__ void __launch_bounds__(kReduceThreads)
    finish_max_kernel(const double *__restrict__ partials, int count, double *__restrict__ result);

// Per-device partials buffer (cudaMalloc, grown on demand, kept until exit).
double *reduction_scratch(int64_t blocks);

void launch_dot(const double *x, const double *y, int64_t n, double *partials, double *result, cudaStream_t s);
void launch_norm_inf(const double *x, int64_t n, double *partials, double *result, cudaStream_t s);

} // namespace vk
