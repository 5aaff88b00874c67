// A dot product on device arrays that allocates no memory.
//
// Some callers cannot call cudaMalloc: code running where a custom allocator
// owns all device memory (a framework's caching allocator or a memory pool
// that must account for every byte), code in a process whose memory budget is
// fixed up front, or code that must not trigger an allocation at this point
// of its run. vk_vec_dot_device (vk_vec.cu) keeps its block partials in a
// buffer it allocates on first use; this variant runs the same two kernels
// with its partials in a fixed array compiled into the library instead.
//
// That array is a file-scope static __device__ array of kNoAllocMaxBlocks
// doubles (32 KB). Every GPU that loads the library holds it until the
// process exits, and every call shares it: each call fully overwrites the
// partials it reads, so nothing has to start at zero, but two calls that
// overlap on the GPU (different streams, or different host threads) race on
// the array and may return wrong sums -- serialise them.
//
// Host code cannot pass the array's name to a kernel (there it is only a
// host-side stand-in for the symbol): the first call on each device, with that
// device current, asks the runtime for the array's device address
// (cudaGetSymbolAddress) and caches it. Make that first call before any
// stream capture.
#include "vikalp_b200.h"
#include "vk_vec.cuh"

#include <mutex>
#include <string>

namespace vk {
int record_error(int code, const std::string &msg); // vk_capi.cu
}

namespace {

constexpr int kNoAllocMaxBlocks = 4096;
constexpr int64_t kNoAllocMaxN = static_cast<int64_t>(kNoAllocMaxBlocks) * vk::kReduceChunk; // 8,388,608

static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxBlocks];

std::mutex g_mu;
double *g_addr[64] = {nullptr};

// Device address of g_noalloc_partials on the current device (looked up once).
int partials_address(double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return vk::record_error(VK_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return vk::record_error(VK_ERR_CUDA, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess)
            return vk::record_error(VK_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_addr[dev] = static_cast<double *>(p);
    }
    *out = g_addr[dev];
    return VK_OK;
}

} // namespace

extern "C" int vk_vec_dot_device_noalloc(const double *x, const double *y, int64_t n, double *result,
                                         void *stream) {
    if (!result || n < 0 || (n > 0 && (!x || !y))) return vk::record_error(VK_ERR_INVALID, "invalid argument");
    if (n > kNoAllocMaxN)
        return vk::record_error(VK_ERR_INVALID,
                                "vk_vec_dot_device_noalloc: n = " + std::to_string(n) +
                                    " exceeds its maximum of 8388608 elements (its fixed scratch holds 4096 "
                                    "block partials); use vk_vec_dot_device for longer vectors");
    double *partials = nullptr;
    const int rc = partials_address(&partials);
    if (rc != VK_OK) return rc;
    try {
        vk::launch_dot(x, y, n, partials, result, static_cast<cudaStream_t>(stream));
    } catch (const std::exception &ex) {
        return vk::record_error(VK_ERR_CUDA, ex.what());
    }
    return VK_OK;
}
