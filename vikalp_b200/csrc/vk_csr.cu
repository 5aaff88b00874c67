// Device-side CSR setup: int64 -> int32 conversion, tile schedules, stable
// transpose. All O(nnz) on the GPU.
#include "vk_csr.cuh"
#include "vk_stage.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <mutex>
#include <unordered_map>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

namespace vk {

namespace {

// flags[r] = 1 where a tile starts at row r (r == rows marks the end): rows
// longer than `short_max` alone, others grouped while their starts fall in
// one `window`-sized window of the nonzero array, at most `rows_max` rows.
__global__ void tile_flags_kernel(const int *__restrict__ ro, int rows, const unsigned char *__restrict__ breaks,
                                  int window, int short_max, int rows_max, int *__restrict__ flags) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > rows) return;
    int f;
    if (r == 0 || r == rows || (breaks && breaks[r])) {
        f = 1;
    } else {
        const int a = ro[r - 1], b = ro[r], c = ro[r + 1];
        const bool long_prev = (b - a) > short_max;
        const bool long_here = (c - b) > short_max;
        f = (long_prev || long_here || (a / window) != (b / window) || (r % rows_max) == 0) ? 1 : 0;
    }
    flags[r] = f;
}

__global__ void tile_scatter_kernel(const int *__restrict__ flags, const int *__restrict__ idx, int rows,
                                    int *__restrict__ tiles) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > rows) return;
    if (flags[r]) tiles[idx[r]] = r;
}

__global__ void iota_kernel(int *__restrict__ a, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = static_cast<int>(i);
}

__global__ void count_cols_kernel(const int *__restrict__ ci, int64_t nnz, int *__restrict__ cnt) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(cnt + ci[k] + 1, 1);
}

__global__ void expand_rows_kernel(const int *__restrict__ ro, int rows, int *__restrict__ rowidx) {
    // one warp per row
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= rows) return;
    for (int k = ro[warp] + lane; k < ro[warp + 1]; k += 32) rowidx[k] = warp;
}

__global__ void gather_rows_kernel(const int *__restrict__ perm, const int *__restrict__ rowidx, int64_t nnz,
                                   int *__restrict__ out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnz; t += (int64_t)gridDim.x * blockDim.x)
        out[t] = rowidx[perm[t]];
}

// ci[k] = rank[ci[k]] (column renaming, in place)
__global__ void rename_cols_kernel(int *__restrict__ ci, const int *__restrict__ rank, int64_t nnz) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnz; t += (int64_t)gridDim.x * blockDim.x)
        ci[t] = rank[ci[t]];
}

// stats[0] = max cnt[j], stats[1] = sum of cnt[j]^2 (integers: exact, order-free)
__global__ void count_stats_kernel(const int *__restrict__ cnt, int n, unsigned long long *__restrict__ stats) {
    unsigned long long mx = 0, sq = 0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const unsigned long long c = static_cast<unsigned long long>(cnt[j]);
        mx = c > mx ? c : mx;
        sq += c * c;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long m2 = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = m2 > mx ? m2 : mx;
        sq += __shfl_xor_sync(0xffffffffu, sq, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(stats, mx);
        atomicAdd(stats + 1, sq);
    }
}

// keys[j] = most - cnt[j] (ascending keys: most nonzeros first), iota[j] = j
__global__ void order_keys_kernel(const int *__restrict__ cnt, int n, int most, int *__restrict__ keys,
                                  int *__restrict__ iota) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        keys[j] = most - cnt[j];
        iota[j] = j;
    }
}

// rank[new_to_old[i]] = i
__global__ void invert_perm_kernel(const int *__restrict__ new_to_old, int n, int *__restrict__ rank) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) rank[new_to_old[i]] = i;
}

// dst[perm[t]] = src[t]
__global__ void scatter_values_kernel(const int *__restrict__ perm, const double *__restrict__ src,
                                      double *__restrict__ dst, int64_t n) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        dst[perm[t]] = src[t];
}

__global__ void tile_k_kernel(const int *__restrict__ ro, const int *__restrict__ tiles, int count,
                              int *__restrict__ tile_k) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) tile_k[t] = ro[tiles[t]];
}

template <class TD, class TS>
__global__ void convert_values_kernel(const TS *__restrict__ src, TD *__restrict__ dst, int64_t n) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        dst[t] = static_cast<TD>(src[t]);
}

template <class TD, class TS>
__global__ void gather_values_kernel(const int *__restrict__ perm, const TS *__restrict__ src, TD *__restrict__ dst,
                                     int64_t nnz) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnz; t += (int64_t)gridDim.x * blockDim.x)
        dst[t] = static_cast<TD>(src[perm[t]]);
}

// chunks[c] = first row r with cost(r) >= c * kChunkCost, cost(r) = ro[r] +
// kRowCost * r (monotone); chunks[nchunks] = rows. Thread per r in [0, rows].
__global__ void chunk_rows_kernel(const int *__restrict__ ro, int rows, int nchunks, int *__restrict__ chunks) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > rows) return;
    const int64_t hi = static_cast<int64_t>(ro[r]) + static_cast<int64_t>(kRowCost) * r;
    const int64_t lo = r == 0 ? -1 : static_cast<int64_t>(ro[r - 1]) + static_cast<int64_t>(kRowCost) * (r - 1);
    // chunk boundaries c * K in (lo, hi]
    int64_t c0 = lo < 0 ? 0 : lo / kChunkCost + 1;
    const int64_t c1 = hi / kChunkCost;
    for (int64_t c = c0; c <= c1 && c < nchunks; ++c) chunks[c] = r;
    if (r == rows) chunks[nchunks] = rows;
}

int grid_for(int64_t n, int threads = 256) {
    const int64_t b = (n + threads - 1) / threads;
    return static_cast<int>(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

int bits_for(int v) {
    int b = 1;
    while (b < 31 && (1 << b) <= v) ++b;
    return b;
}

} // namespace

int *device_error_flag() {
    static int *flags[64] = {nullptr};
    int dev = 0;
    VK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw CudaFailure("device ordinal out of range");
    if (!flags[dev]) {
        int *p = nullptr;
        VK_CUDA(cudaMalloc(&p, sizeof(int)));
        VK_CUDA(cudaMemset(p, 0, sizeof(int)));
        flags[dev] = p;
    }
    return flags[dev];
}

void check_device_error(cudaStream_t s) {
    int *f = device_error_flag();
    int h = 0;
    VK_CUDA(cudaMemcpyAsync(&h, f, sizeof(int), cudaMemcpyDeviceToHost, s));
    VK_CUDA(cudaStreamSynchronize(s));
    if (h != 0) {
        VK_CUDA(cudaMemsetAsync(f, 0, sizeof(int), s));
        VK_CUDA(cudaStreamSynchronize(s));
        throw CudaFailure(h == kDevErrBarrierTimeout ? "a sparse pass timed out waiting for its staged tile"
                                                     : "a kernel reported a device error");
    }
}

namespace {
// One tile schedule: tiles[t] = first row, tile_k[t] = first nonzero.
int schedule(const CsrPattern32 &p, cudaStream_t s, const unsigned char *breaks, int window, int short_max,
             int rows_max, DevBuf<int> &tiles, DevBuf<int> &tile_k) {
    const int rows = p.rows;
    DevBuf<int> flags(rows + 1), idx(rows + 1);
    tile_flags_kernel<<<ceil_div(rows + 1, 256), 256, 0, s>>>(p.ro.get(), rows, breaks, window, short_max, rows_max,
                                                              flags.get());
    VK_LAUNCH_CHECK();
    size_t tb = 0;
    VK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, flags.get(), idx.get(), rows + 1, s));
    DevBuf<unsigned char> tmp(tb > 0 ? tb : 1);
    VK_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, flags.get(), idx.get(), rows + 1, s));
    int last_idx = 0, last_flag = 0;
    VK_CUDA(cudaMemcpyAsync(&last_idx, idx.get() + rows, sizeof(int), cudaMemcpyDeviceToHost, s));
    VK_CUDA(cudaMemcpyAsync(&last_flag, flags.get() + rows, sizeof(int), cudaMemcpyDeviceToHost, s));
    VK_CUDA(cudaStreamSynchronize(s));
    const int count = last_idx + last_flag; // number of boundaries (tiles + 1)
    tiles.reset(count);
    tile_scatter_kernel<<<ceil_div(rows + 1, 256), 256, 0, s>>>(flags.get(), idx.get(), rows, tiles.get());
    VK_LAUNCH_CHECK();
    tile_k.reset(count);
    tile_k_kernel<<<ceil_div(count, 256), 256, 0, s>>>(p.ro.get(), tiles.get(), count, tile_k.get());
    VK_LAUNCH_CHECK();
    VK_CUDA(cudaStreamSynchronize(s));
    return count - 1;
}
} // namespace

void build_tiles(CsrPattern32 &p, cudaStream_t s, const unsigned char *breaks) {
    const int rows = p.rows;
    if (breaks) {
        // forced tile starts change the schedule: fold them into the identity
        std::vector<unsigned char> h(static_cast<size_t>(rows) + 1);
        VK_CUDA(cudaMemcpyAsync(h.data(), breaks, h.size(), cudaMemcpyDeviceToHost, s));
        VK_CUDA(cudaStreamSynchronize(s));
        uint64_t f = 0x62726561u; // "brea"
        for (size_t r = 0; r < h.size(); ++r)
            if (h[r]) f = mix_fingerprint(f, r);
        p.fp = mix_fingerprint(p.fp, f);
    }
    p.ntiles = schedule(p, s, breaks, kChunk, kShortMax, kTileRows, p.tiles, p.tile_k);
    p.nstiles = schedule(p, s, nullptr, kStageWindow, kStageShort, kStageRows, p.stiles, p.stile_k);
    // cost-balanced row ranges for the hybrid kernel
    int nnz_total = 0;
    VK_CUDA(cudaMemcpyAsync(&nnz_total, p.ro.get() + rows, sizeof(int), cudaMemcpyDeviceToHost, s));
    VK_CUDA(cudaStreamSynchronize(s));
    const int64_t cost = static_cast<int64_t>(nnz_total) + static_cast<int64_t>(kRowCost) * rows;
    p.nchunks = rows > 0 ? static_cast<int>((cost - 1) / kChunkCost + 1) : 0;
    p.chunks.reset(p.nchunks + 1);
    chunk_rows_kernel<<<ceil_div(rows + 1, 256), 256, 0, s>>>(p.ro.get(), rows, p.nchunks, p.chunks.get());
    VK_LAUNCH_CHECK();
    VK_CUDA(cudaStreamSynchronize(s));
}

void upload_pattern(int64_t rows, int64_t cols, const int64_t *h_ro, const int64_t *h_ci, CsrPattern32 &out,
                    cudaStream_t s) {
    const int64_t nnz = h_ro[rows];
    device_error_flag(); // allocate before any kernel (or graph capture) needs it
    out.rows = static_cast<int>(rows);
    out.cols = static_cast<int>(cols);
    out.nnz = nnz;
    out.ro.reset(rows + 1);
    out.ci.reset(padded(nnz));
    VK_CUDA(cudaMemsetAsync(out.ci.get(), 0, padded(nnz) * sizeof(int), s));
    // int64 -> int32 while staging (validated: every offset and index fits)
    stage_h2d_narrow(out.ro.get(), h_ro, rows + 1, s);
    stage_h2d_narrow(out.ci.get(), h_ci, nnz, s);
    int mr = 0;
    for (int64_t r = 0; r < rows; ++r) mr = std::max<int>(mr, static_cast<int>(h_ro[r + 1] - h_ro[r]));
    out.max_row = mr;
    out.fp = pattern_fingerprint(rows, cols, h_ro, h_ci);
    build_tiles(out, s);
}

void expand_rows(const CsrPattern32 &p, int *rowidx, cudaStream_t s) {
    if (p.rows == 0) return;
    expand_rows_kernel<<<ceil_div(static_cast<int64_t>(p.rows) * 32, 256), 256, 0, s>>>(p.ro.get(), p.rows, rowidx);
    VK_LAUNCH_CHECK();
}

void transpose_pattern(const CsrPattern32 &a, CsrPattern32 &at, DevBuf<int> &perm, cudaStream_t s) {
    const int64_t nnz = a.nnz;
    at.rows = a.cols;
    at.cols = a.rows;
    at.nnz = nnz;
    at.fp = mix_fingerprint(a.fp, 0x7472616e73706f73ull); // "transpos"
    at.ro.reset(a.cols + 1);
    at.ci.reset(padded(nnz));
    VK_CUDA(cudaMemsetAsync(at.ci.get(), 0, padded(nnz) * sizeof(int), s));
    perm.reset(nnz > 0 ? nnz : 1);
    VK_CUDA(cudaMemsetAsync(at.ro.get(), 0, (a.cols + 1) * sizeof(int), s));
    if (nnz > 0) {
        DevBuf<int> keys_out(nnz), vals_in(nnz), rowidx(nnz);
        iota_kernel<<<grid_for(nnz), 256, 0, s>>>(vals_in.get(), nnz);
        VK_LAUNCH_CHECK();
        const int end_bit = bits_for(a.cols > 0 ? a.cols - 1 : 0);
        size_t tb = 0;
        VK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, a.ci.get(), keys_out.get(), vals_in.get(), perm.get(),
                                                static_cast<int>(nnz), 0, end_bit, s));
        DevBuf<unsigned char> tmp(tb > 0 ? tb : 1);
        VK_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, a.ci.get(), keys_out.get(), vals_in.get(), perm.get(),
                                                static_cast<int>(nnz), 0, end_bit, s));
        count_cols_kernel<<<grid_for(nnz), 256, 0, s>>>(a.ci.get(), nnz, at.ro.get());
        VK_LAUNCH_CHECK();
        size_t tb2 = 0;
        VK_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb2, at.ro.get(), at.ro.get(), a.cols + 1, s));
        DevBuf<unsigned char> tmp2(tb2 > 0 ? tb2 : 1);
        VK_CUDA(cub::DeviceScan::InclusiveSum(tmp2.get(), tb2, at.ro.get(), at.ro.get(), a.cols + 1, s));
        expand_rows(a, rowidx.get(), s);
        gather_rows_kernel<<<grid_for(nnz), 256, 0, s>>>(perm.get(), rowidx.get(), nnz, at.ci.get());
        VK_LAUNCH_CHECK();
        VK_CUDA(cudaStreamSynchronize(s));
    }
    // longest transposed row
    {
        std::vector<int> h(a.cols + 1);
        VK_CUDA(cudaMemcpyAsync(h.data(), at.ro.get(), (a.cols + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
        VK_CUDA(cudaStreamSynchronize(s));
        int mr = 0;
        for (int j = 0; j < a.cols; ++j) mr = std::max(mr, h[j + 1] - h[j]);
        at.max_row = mr;
    }
    build_tiles(at, s);
}

ColumnOrder column_order_mode() {
    const char *e = std::getenv("VIKALP_B200_COLUMN_ORDER");
    if (!e || !*e || std::strcmp(e, "auto") == 0) return ColumnOrder::Auto;
    if (std::strcmp(e, "keep") == 0) return ColumnOrder::Keep;
    if (std::strcmp(e, "count") == 0) return ColumnOrder::Count;
    throw InvalidInput("VIKALP_B200_COLUMN_ORDER must be auto, keep or count");
}

bool order_columns_by_count(CsrPattern32 &a, ColumnOrder mode, DevBuf<int> &new_to_old, cudaStream_t s) {
    const int n = a.cols;
    const int64_t nnz = a.nnz;
    if (mode == ColumnOrder::Keep || n <= 1 || nnz <= 0) return false;
    if (mode == ColumnOrder::Auto && nnz < kOrderMinNnz) return false;
    // nonzeros per column (cnt[j + 1]) and their largest value and sum of squares
    DevBuf<int> cnt(static_cast<size_t>(n) + 1);
    DevBuf<unsigned long long> stats(2);
    VK_CUDA(cudaMemsetAsync(cnt.get(), 0, cnt.bytes(), s));
    VK_CUDA(cudaMemsetAsync(stats.get(), 0, stats.bytes(), s));
    count_cols_kernel<<<grid_for(nnz), 256, 0, s>>>(a.ci.get(), nnz, cnt.get());
    count_stats_kernel<<<grid_for(n), 256, 0, s>>>(cnt.get() + 1, n, stats.get());
    VK_LAUNCH_CHECK();
    unsigned long long h[2] = {0, 0};
    VK_CUDA(cudaMemcpyAsync(h, stats.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    VK_CUDA(cudaStreamSynchronize(s));
    const int most = static_cast<int>(h[0]);
    const double mean = static_cast<double>(nnz) / n;
    const double var = std::max(0.0, static_cast<double>(h[1]) / n - mean * mean);
    if (mode == ColumnOrder::Auto && std::sqrt(var) < kOrderMinSpread * mean) return false;
    // stable sort on (most - count): most nonzeros first, ties in the caller's order
    DevBuf<int> keys(static_cast<size_t>(n)), keys_out(static_cast<size_t>(n)), iota(static_cast<size_t>(n)),
        rank(static_cast<size_t>(n));
    new_to_old.reset(static_cast<size_t>(n));
    order_keys_kernel<<<grid_for(n), 256, 0, s>>>(cnt.get() + 1, n, most, keys.get(), iota.get());
    VK_LAUNCH_CHECK();
    size_t tb = 0;
    const int end_bit = bits_for(most);
    VK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.get(), keys_out.get(), iota.get(), new_to_old.get(), n, 0,
                                            end_bit, s));
    DevBuf<unsigned char> tmp(tb > 0 ? tb : 1);
    VK_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, keys.get(), keys_out.get(), iota.get(), new_to_old.get(), n,
                                            0, end_bit, s));
    invert_perm_kernel<<<grid_for(n), 256, 0, s>>>(new_to_old.get(), n, rank.get());
    rename_cols_kernel<<<grid_for(nnz), 256, 0, s>>>(a.ci.get(), rank.get(), nnz);
    VK_LAUNCH_CHECK();
    VK_CUDA(cudaStreamSynchronize(s)); // the temporaries go out of scope
    a.fp = mix_fingerprint(a.fp, 0x636f6c636f756e74ull); // "colcount"
    return true;
}

void scatter_values(const int *perm, const double *src, double *dst, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    scatter_values_kernel<<<grid_for(n), 256, 0, s>>>(perm, src, dst, n);
    VK_LAUNCH_CHECK();
}

template <class TD, class TS>
void gather_values(const int *perm, const TS *src, TD *dst, int64_t nnz, cudaStream_t s) {
    if (nnz <= 0) return;
    gather_values_kernel<TD, TS><<<grid_for(nnz), 256, 0, s>>>(perm, src, dst, nnz);
    VK_LAUNCH_CHECK();
}

template <class TD, class TS>
void convert_values(const TS *src, TD *dst, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    convert_values_kernel<TD, TS><<<grid_for(n), 256, 0, s>>>(src, dst, n);
    VK_LAUNCH_CHECK();
}

template void convert_values<float, double>(const double *, float *, int64_t, cudaStream_t);
template void convert_values<double, float>(const float *, double *, int64_t, cudaStream_t);
template void convert_values<double, double>(const double *, double *, int64_t, cudaStream_t);

template void gather_values<double, double>(const int *, const double *, double *, int64_t, cudaStream_t);
template void gather_values<float, double>(const int *, const double *, float *, int64_t, cudaStream_t);
template void gather_values<float, float>(const int *, const float *, float *, int64_t, cudaStream_t);

// ---- autotuner ----------------------------------------------------------------
namespace {
// A stand-in for the fused passes: four per-row inputs loaded ahead of the
// sums and a clamped update stored, so variants that run short of registers
// with a real epilogue lose here too.
template <class T>
struct TuneEpi : EpiBase<T> {
    T *y;
    const T *a, *b, *lo, *hi;
    struct Pre {
        T a, b, lo, hi;
    };
    __device__ Pre load(int i) const { return Pre{a[i], b[i], lo[i], hi[i]}; }
    template <int NV, int NR>
    __device__ void row_pre(int i, const T (&s)[NV], const Pre &p, double (&red)[NR]) const {
        const T v = clampbox(p.a * s[0] + p.b, p.lo, p.hi);
        y[i] = v;
        red[0] = smax(red[0], static_cast<double>(fabs(v - s[0])));
    }
};

template <class T>
__global__ void fill_kernel(T *a, int64_t n, T v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = v;
}
} // namespace

int forced_variant() {
    const char *e = std::getenv("VIKALP_B200_VARIANT");
    if (!e || !*e) return -1;
    const int v = std::atoi(e);
    return v >= 0 && v < kFastVariants ? v : -1;
}

uint64_t mix_fingerprint(uint64_t a, uint64_t b) {
    uint64_t h = a ^ 0x9e3779b97f4a7c15ull;
    for (int k = 0; k < 8; ++k) {
        h ^= (b >> (8 * k)) & 0xffu;
        h *= 0x100000001b3ull;
    }
    return h;
}

uint64_t pattern_fingerprint(int64_t rows, int64_t cols, const int64_t *ro, const int64_t *ci) {
    uint64_t h = 0xcbf29ce484222325ull;
    h = mix_fingerprint(h, static_cast<uint64_t>(rows));
    h = mix_fingerprint(h, static_cast<uint64_t>(cols));
    // a strided sample (the fingerprint only keys the tuning cache: a collision
    // reuses another pattern's kernel picks, every one of which is correct)
    for (int64_t r = 0; r <= rows; r += 61) h = mix_fingerprint(h, static_cast<uint64_t>(ro[r]));
    h = mix_fingerprint(h, static_cast<uint64_t>(ro[rows]));
    const int64_t nnz = ro[rows];
    for (int64_t k = 0; k < nnz; k += 61) h = mix_fingerprint(h, static_cast<uint64_t>(ci[k]));
    if (nnz > 0) h = mix_fingerprint(h, static_cast<uint64_t>(ci[nnz - 1]));
    return h;
}

namespace {
std::mutex g_tune_mu;
std::unordered_map<uint64_t, int> &tune_cache() {
    static auto *m = new std::unordered_map<uint64_t, int>(); // lives until exit
    return *m;
}
// the current device and its SM count: picks are per GPU model and device
uint64_t device_key() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 0;
    return (static_cast<uint64_t>(static_cast<uint32_t>(dev)) << 32) | static_cast<uint32_t>(sms);
}
} // namespace

uint64_t tune_key(uint64_t fingerprint, const char *tag, int value_bytes) {
    uint64_t h = mix_fingerprint(fingerprint, device_key());
    for (const char *c = tag; *c; ++c) h = mix_fingerprint(h, static_cast<unsigned char>(*c));
    return mix_fingerprint(h, static_cast<uint64_t>(value_bytes));
}

bool cached_pick(uint64_t key, int &variant) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = tune_cache().find(key);
    if (it == tune_cache().end()) return false;
    variant = it->second;
    return true;
}

int store_pick(uint64_t key, int variant) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    return tune_cache().emplace(key, variant).first->second;
}

template <class T>
void autotune_pattern(CsrPattern32 &p, const T *val, cudaStream_t s, int64_t min_nnz) {
    p.variant = 0;
    if (const int f = forced_variant(); f >= 0) {
        p.variant = f;
        return;
    }
    if (p.nnz < min_nnz || p.rows == 0 || p.cols == 0) return;
    const uint64_t key = tune_key(p.fp, "pattern", sizeof(T));
    if (cached_pick(key, p.variant)) return;
    DevBuf<T> x(p.cols), y(p.rows), pre(static_cast<size_t>(p.rows) * 4);
    fill_kernel<T><<<grid_for(p.cols), 256, 0, s>>>(x.get(), p.cols, T(1));
    fill_kernel<T><<<grid_for(int64_t(p.rows) * 4), 256, 0, s>>>(pre.get(), int64_t(p.rows) * 4, T(1));
    VK_LAUNCH_CHECK();
    TuneEpi<T> e;
    e.y = y.get();
    e.a = pre.get();
    e.b = pre.get() + p.rows;
    e.lo = pre.get() + 2 * static_cast<size_t>(p.rows);
    e.hi = pre.get() + 3 * static_cast<size_t>(p.rows);
    float best[kFastVariants];
    const int best_v = tune_variants(
        [&](int v) {
            p.variant = v;
            launch_tiles<T, T, 1, false>(view(p, val), Gathers<T, 1>{{x.get()}}, e, s);
        },
        s, best);
    p.variant = store_pick(key, best_v);
}

template void autotune_pattern<double>(CsrPattern32 &, const double *, cudaStream_t, int64_t);
template void autotune_pattern<float>(CsrPattern32 &, const float *, cudaStream_t, int64_t);

} // namespace vk
