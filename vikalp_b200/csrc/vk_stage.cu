// Staged host <-> device copies (vk_stage.cuh).
#include "vk_stage.cuh"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <exception>
#include <mutex>
#include <system_error>
#include <thread>
#include <vector>

namespace vk {
namespace {

// Process-wide pool of pinned kStageChunk-byte buffers. Buffers are kept for
// the life of the process (freeing pinned memory from a static destructor
// can run after the CUDA runtime has shut down).
std::mutex g_pool_mu;
std::vector<void *> g_pool;

void *acquire_pinned() {
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        if (!g_pool.empty()) {
            void *p = g_pool.back();
            g_pool.pop_back();
            return p;
        }
    }
    void *p = nullptr;
    VK_CUDA(cudaHostAlloc(&p, kStageChunk, cudaHostAllocPortable));
    return p;
}

void release_pinned(void *p) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    g_pool.push_back(p);
}

// 0: pool not started, 1: being allocated, 2: ready, 3: pinned memory unavailable
std::atomic<int> g_pool_state{0};

// The allocating thread; joined at process exit (function-local static, so
// destroyed before the CUDA runtime linked into this library shuts down).
struct PoolWarmup {
    std::thread t;
    ~PoolWarmup() {
        if (t.joinable()) t.join();
    }
};
PoolWarmup &pool_warmup() {
    static PoolWarmup w;
    return w;
}

// True once the pool holds a buffer per staging thread; the first call starts
// the allocation on a background thread and returns false.
bool pool_ready() {
    int st = g_pool_state.load();
    if (st == 2) return true;
    if (st == 0 && g_pool_state.compare_exchange_strong(st, 1)) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) {
            g_pool_state.store(3);
            return false;
        }
        pool_warmup().t = std::thread([dev] {
            std::vector<void *> bufs;
            if (cudaSetDevice(dev) == cudaSuccess)
                for (int i = 0; i < kStageThreads; ++i) {
                    void *p = nullptr;
                    if (cudaHostAlloc(&p, kStageChunk, cudaHostAllocPortable) != cudaSuccess) break;
                    bufs.push_back(p);
                }
            const bool ok = static_cast<int>(bufs.size()) == kStageThreads;
            {
                std::lock_guard<std::mutex> lk(g_pool_mu);
                for (void *p : bufs) g_pool.push_back(p);
            }
            g_pool_state.store(ok ? 2 : 3);
        });
    }
    return false;
}

// Runs body(chunk, buffer, event, pending) for chunks 0..nchunks-1, chunk i on
// thread i % T, each thread with its own pinned buffer and event; `pending`
// says a DMA touching the buffer may still be running (set before its event
// is recorded). A thread waits for its last DMA before its buffer goes back to
// the pool; after an error it waits for the whole stream s. The first error is
// rethrown on the calling thread.
template <class Body>
void run_staged(int64_t nchunks, cudaStream_t s, Body body, int max_threads = kStageThreads) {
    int dev = 0;
    VK_CUDA(cudaGetDevice(&dev));
    const unsigned hw = std::thread::hardware_concurrency();
    const int T = static_cast<int>(std::max<int64_t>(
        1, std::min<int64_t>({static_cast<int64_t>(max_threads), nchunks, static_cast<int64_t>(hw == 0 ? 1 : hw)})));
    std::vector<std::exception_ptr> errs(T);
    auto work = [&](int t) {
        void *buf = nullptr;
        cudaEvent_t ev = nullptr;
        bool pending = false;
        try {
            VK_CUDA(cudaSetDevice(dev));
            buf = acquire_pinned();
            VK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            for (int64_t i = t; i < nchunks; i += T) body(i, buf, ev, pending);
            if (pending) VK_CUDA(cudaEventSynchronize(ev));
            pending = false;
        } catch (...) {
            errs[t] = std::current_exception();
            if (pending) cudaStreamSynchronize(s);
            pending = false;
        }
        if (ev) cudaEventDestroy(ev);
        if (buf) release_pinned(buf);
    };
    std::vector<std::thread> pool;
    pool.reserve(T - 1);
    int started = 1;
    try {
        for (; started < T; ++started) pool.emplace_back(work, started);
    } catch (const std::system_error &) {
        // fewer threads to be had: the calling thread takes the shares not started
    }
    work(0);
    for (int t = started; t < T; ++t) work(t);
    for (std::thread &th : pool) th.join();
    for (const std::exception_ptr &e : errs)
        if (e) std::rethrow_exception(e);
}

__global__ void narrow_kernel(const int64_t *__restrict__ src, int *__restrict__ dst, int64_t n) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[i] = static_cast<int>(src[i]);
}

} // namespace

void stage_h2d(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return;
    if (bytes < kStageMin || !pool_ready()) {
        VK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        VK_CUDA(cudaStreamSynchronize(s));
        return;
    }
    char *d = static_cast<char *>(dst);
    const char *h = static_cast<const char *>(src);
    const int64_t nchunks = static_cast<int64_t>((bytes + kStageChunk - 1) / kStageChunk);
    run_staged(nchunks, s, [&](int64_t i, void *buf, cudaEvent_t ev, bool &pending) {
        const size_t off = static_cast<size_t>(i) * kStageChunk;
        const size_t n = std::min(kStageChunk, bytes - off);
        if (pending) VK_CUDA(cudaEventSynchronize(ev));
        std::memcpy(buf, h + off, n);
        pending = true;
        VK_CUDA(cudaMemcpyAsync(d + off, buf, n, cudaMemcpyHostToDevice, s));
        VK_CUDA(cudaEventRecord(ev, s));
    });
}

void stage_h2d_narrow(int *dst, const int64_t *src, int64_t count, cudaStream_t s) {
    if (count <= 0) return;
    constexpr int64_t kPer = static_cast<int64_t>(kStageChunk / sizeof(int)); // int32 outputs per chunk
    if (static_cast<size_t>(count) * sizeof(int64_t) < kStageMin) {
        std::vector<int> tmp(static_cast<size_t>(count));
        for (int64_t i = 0; i < count; ++i) tmp[static_cast<size_t>(i)] = static_cast<int>(src[i]);
        VK_CUDA(cudaMemcpyAsync(dst, tmp.data(), count * sizeof(int), cudaMemcpyHostToDevice, s));
        VK_CUDA(cudaStreamSynchronize(s));
        return;
    }
    if (!pool_ready()) {
        // plain copy of the int64 values, narrowed on the device
        DevBuf<int64_t> t(static_cast<size_t>(count));
        VK_CUDA(cudaMemcpyAsync(t.get(), src, count * sizeof(int64_t), cudaMemcpyHostToDevice, s));
        const int64_t blocks = std::min<int64_t>((count + 255) / 256, 65535);
        narrow_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(t.get(), dst, count);
        VK_LAUNCH_CHECK();
        VK_CUDA(cudaStreamSynchronize(s));
        return;
    }
    const int64_t nchunks = (count + kPer - 1) / kPer;
    run_staged(nchunks, s, [&](int64_t i, void *buf, cudaEvent_t ev, bool &pending) {
        const int64_t b = i * kPer, n = std::min(kPer, count - b);
        if (pending) VK_CUDA(cudaEventSynchronize(ev));
        int *o = static_cast<int *>(buf);
        const int64_t *in = src + b;
        for (int64_t k = 0; k < n; ++k) o[k] = static_cast<int>(in[k]);
        pending = true;
        VK_CUDA(cudaMemcpyAsync(dst + b, buf, n * sizeof(int), cudaMemcpyHostToDevice, s));
        VK_CUDA(cudaEventRecord(ev, s));
    }, kStageThreadsNarrow);
}

void stage_d2h(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return;
    if (bytes < kStageMin || !pool_ready()) {
        VK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        VK_CUDA(cudaStreamSynchronize(s));
        return;
    }
    char *h = static_cast<char *>(dst);
    const char *d = static_cast<const char *>(src);
    const int64_t nchunks = static_cast<int64_t>((bytes + kStageChunk - 1) / kStageChunk);
    run_staged(nchunks, s, [&](int64_t i, void *buf, cudaEvent_t ev, bool &pending) {
        const size_t off = static_cast<size_t>(i) * kStageChunk;
        const size_t n = std::min(kStageChunk, bytes - off);
        pending = true;
        VK_CUDA(cudaMemcpyAsync(buf, d + off, n, cudaMemcpyDeviceToHost, s));
        VK_CUDA(cudaEventRecord(ev, s));
        VK_CUDA(cudaEventSynchronize(ev));
        pending = false;
        std::memcpy(h + off, buf, n);
    }, kStageThreadsD2H);
}

void stage_d2h_many(const StageCopy *copies, int64_t count, cudaStream_t s) {
    size_t total = 0;
    for (int64_t i = 0; i < count; ++i) total += copies[i].bytes;
    if (total == 0) return;
    if (total < kStageMin || !pool_ready()) {
        for (int64_t i = 0; i < count; ++i)
            if (copies[i].bytes > 0)
                VK_CUDA(cudaMemcpyAsync(copies[i].dst, copies[i].src, copies[i].bytes, cudaMemcpyDeviceToHost, s));
        VK_CUDA(cudaStreamSynchronize(s));
        return;
    }
    run_staged(count, s, [&](int64_t i, void *buf, cudaEvent_t ev, bool &pending) {
        char *h = static_cast<char *>(copies[i].dst);
        const char *d = static_cast<const char *>(copies[i].src);
        for (size_t off = 0; off < copies[i].bytes; off += kStageChunk) {
            const size_t n = std::min(kStageChunk, copies[i].bytes - off);
            pending = true;
            VK_CUDA(cudaMemcpyAsync(buf, d + off, n, cudaMemcpyDeviceToHost, s));
            VK_CUDA(cudaEventRecord(ev, s));
            VK_CUDA(cudaEventSynchronize(ev));
            pending = false;
            std::memcpy(h + off, buf, n);
        }
    }, kStageThreadsD2H);
}

} // namespace vk
