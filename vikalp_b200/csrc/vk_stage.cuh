// Large host <-> device copies of caller (pageable) memory through pinned
// staging buffers that several host threads fill or drain at once.
//
// A copy from pageable memory goes through the driver's own staging at the
// speed of one host thread's memcpy (~10 GB/s); here each of up to
// kStageThreads threads owns one pinned buffer of kStageChunk bytes and takes
// every T-th chunk of the transfer: it copies (or converts) the chunk into its
// buffer and queues the DMA on the caller's stream, waiting for its previous
// DMA before refilling the buffer. The host copies run in parallel and the
// DMA engine streams at PCIe rate. Every function returns when the transfer
// has completed (the caller's memory may be reused at once). Copies below
// kStageMin bytes go straight through cudaMemcpyAsync + a stream wait, and so
// do all copies until the pinned buffers exist: the first large transfer of
// the process starts their allocation on a background thread (pinning costs
// ~0.1 s the first time) and does not wait for it.
#pragma once

#include "vk_common.cuh"

namespace vk {

constexpr size_t kStageChunk = size_t(4) << 20; // bytes per staged chunk (and per pinned buffer)
constexpr size_t kStageMin = size_t(16) << 20;  // smaller transfers are not staged
constexpr int kStageThreads = 4;
// Device -> host copies write into the caller's memory, which is often fresh
// (a first touch faults each page in); the kernel serves page faults on
// different pages in parallel, so downloads spread over more threads. Their
// extra pinned buffers join the process-wide pool on first use.
constexpr int kStageThreadsD2H = 16;
// int64 -> int32 uploads convert on the host threads (the CSR's indices), which
// bounds them by the threads' loads and stores, not by the DMA: more threads.
constexpr int kStageThreadsNarrow = 8;

// dst (device) <- src (host), `bytes` bytes.
void stage_h2d(void *dst, const void *src, size_t bytes, cudaStream_t s);
// dst (device, int32) <- src (host, int64) converted element by element; the
// caller guarantees every value fits in int32.
void stage_h2d_narrow(int *dst, const int64_t *src, int64_t count, cudaStream_t s);
// dst (host) <- src (device), `bytes` bytes; work queued earlier on s is
// complete before the copy starts.
void stage_d2h(void *dst, const void *src, size_t bytes, cudaStream_t s);

// Many device -> host copies (e.g. one result array per batch instance),
// spread over up to kStageThreadsD2H threads: copy i goes to thread i % T, in pieces of
// at most kStageChunk bytes. Staged when the copies add up to kStageMin bytes.
struct StageCopy {
    void *dst;
    const void *src;
    size_t bytes;
};
void stage_d2h_many(const StageCopy *copies, int64_t count, cudaStream_t s);

} // namespace vk
