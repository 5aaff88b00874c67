#pragma once

// The B200 execution backend (VIKALP include/vikalp/backend/CudaBackend.hpp:18-20):
// the same factory name, returning the ExecutionBackend contract over this
// library's device vectors and sparse operators (vikalp_b200.h: vk_dvec_*,
// vk_spmat_*). All operations are FP64 on CUDA device 0 (as the reference
// pins device 0), on the calling thread's default stream; device memory is
// RAII. Thread safety: none -- create one backend per thread.
//
// Errors follow the reference's backends: a size mismatch or a malformed CSR
// pattern throws std::invalid_argument ("CudaBackend: ..."), a CUDA failure
// std::runtime_error.

#include "vikalp/contracts/ExecutionBackend.hpp"

#include <memory>

namespace vikalp {

// Sparse product order of multiply(): Fast (the autotuned kernels; equal to
// the CPU backend up to rounding) or Sequential (every row summed left to
// right in CSR order, bit-identical to the CPU backend).
enum class CudaProductOrder { Fast, Sequential };

[[nodiscard]] std::unique_ptr<ExecutionBackend> make_cuda_backend();
[[nodiscard]] std::unique_ptr<ExecutionBackend> make_cuda_backend(CudaProductOrder order);

} // namespace vikalp
