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
// (cudaGetSymbolAddress) and caches it together with the unique ID of the
// CUDA context it belongs to. A call made in a different context (after a
// cudaDeviceReset, say, which unloads the module and creates a new primary
// context) looks the address up again instead of using a stale one. Make the
// first call on a device before any stream capture: with lazy module loading
// the driver loads the library's device code (and places the array) on that
// call.
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

struct CachedAddress {
    unsigned long long context_id = 0; // 0: not looked up yet (context IDs start at 1)
    double *address = nullptr;
};
CachedAddress g_addr[64];

// The current context's unique ID (cuCtxGetId, CUDA 12.0+), reached through
// the runtime's driver entry points so the library keeps no link-time
// dependency on the driver library. 0 when it cannot be had: the address is
// then looked up on every call.
using CtxGetCurrentFn = int (*)(void **);
using CtxGetIdFn = int (*)(void *, unsigned long long *);

unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
    });
    if (!get_current || !get_id) return 0;
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of g_noalloc_partials in the current device's context (looked
// up once per context).
int partials_address(double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return vk::record_error(VK_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return vk::record_error(VK_ERR_CUDA, "device ordinal out of range");
    // 0 before the runtime has made this thread's context current; the lookup
    // below does that, and the ID is read again for the cache
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_mu);
    CachedAddress &c = g_addr[dev];
    if (ctx == 0 || c.context_id != ctx || !c.address) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess)
            return vk::record_error(VK_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        c.address = static_cast<double *>(p);
        c.context_id = ctx != 0 ? ctx : current_context_id();
    }
    *out = c.address;
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
