// Device CSR storage and the sparse passes used by every product.
//
// Layout in HBM (per matrix): int32 row offsets [rows+1], int32 column indices
// [nnz], values [nnz] (float64 or float32) -- both padded by kPad elements --
// and a schedule of warp-tiles: tiles[t] = first row, tile_k[t] = first
// nonzero (ntiles+1 entries each). A warp-tile is either
//   * a run of at most kTileRows consecutive rows whose row starts fall in the
//     same kChunk-sized window of the nonzero array and that are each at most
//     kShortMax long (so it holds at most kChunk - 1 + kShortMax = kCap
//     nonzeros), or
//   * one row longer than kShortMax.
//
// FAST order (tile_kernel_fast): each warp of a persistent grid walks its own
// sequence of tiles. Per tile, a short prologue loads the tile's row offsets
// and the epilogue's per-row inputs (y, bounds, ...) into a small
// warp-private shared-memory area and marks each row's last nonzero in a
// bitmask. The warp then streams the tile 32 nonzeros per step, U steps per
// batch with every load of the batch in flight at once (column indices and
// values fully coalesced, the gathers of x independent; optionally the next
// batch's loads issued before this batch is reduced), and forms row sums
// with a segmented warp scan over the bitmask; the lane holding a row's last
// nonzero runs the fused epilogue (the PDHG primal or dual update, a
// residual, ...). No product vector goes back to HBM, there is no CTA-wide
// barrier in the loop, and only ~40 registers per thread are live, so each
// SM keeps 48+ warps of loads in flight. Rows longer than kCap are streamed by
// the whole warp.
//
// The FAST order has four kernel families, all with the same epilogue
// interface; the setup autotuner (autotune_pattern, and the reference engine's
// per-pass tuning) times every variant on the matrix and keeps the fastest:
// the segmented-scan warp-tile kernel above (tile_kernel_fast), sub-warps of L
// lanes per row (tile_kernel_sub), lanes owning short rows with longer rows
// shared by sub-warps or the warp over cost-balanced row chunks
// (tile_kernel_hyb, the kernel for power-law transposes), and bulk-copy
// (TMA) staging of each piece's indices and values into shared memory
// (tile_kernel_tma). Matrices of power-law and uniform rows alike are bound by
// the random gathers of x (about one L1TEX tag lookup per gather), not by HBM.
//
// SEQUENTIAL order (tile_kernel_exact): one thread per row, left to right with
// each product rounded on its own -- the reference CPU order
// (cpu_ops.cpp:418-427, 444-458), so results are bit-identical to it. It is
// the parity mode, not the fast path.
#pragma once

#include "vk_common.cuh"

#include <algorithm>
#include <vector>

namespace vk {

constexpr int kWarps = 4;                  // warps per CTA
constexpr int kTileThreads = kWarps * 32;  // threads per CTA
constexpr int kChunk = 768;                // nonzero window that groups short rows
constexpr int kShortMax = 256;             // longer rows get a tile of their own
constexpr int kCap = kChunk + kShortMax;   // max nonzeros of a multi-row tile
constexpr int kTileRows = 64;              // max rows per warp-tile
constexpr int kPad = 8;                    // padding (elements) of index / value arrays
constexpr int kMaxGridPerSM = 16;          // persistent CTAs per SM (upper bound)
// The staged kernel's schedule: at most kStageRows rows whose starts fall in
// one kStageWindow-sized window of the nonzero array, each at most
// kStageShort long (so at most kStageCap nonzeros), or one longer row.
constexpr int kStageWindow = 384;
constexpr int kStageShort = 128;
constexpr int kStageCap = kStageWindow + kStageShort; // 512
constexpr int kStageRows = 32;
constexpr int kStageSlots = kStageCap + 8; // staged elements per stage incl. the 16-byte widening
// Dynamic shared memory of the staged kernel for value type T.
template <class T>
constexpr int stage_smem_bytes() {
    return kWarps * 2 * kStageSlots * static_cast<int>(sizeof(int) + sizeof(T));
}
constexpr int kMaxGrid = 160 * kMaxGridPerSM; // partial-sum buffers are sized for this

inline int64_t padded(int64_t nnz) { return nnz + kPad; }

// Owning device CSR pattern + tile schedule (values are stored by the user,
// padded(nnz) elements).
struct CsrPattern32 {
    int rows = 0, cols = 0;
    int64_t nnz = 0;
    DevBuf<int> ro, ci, tiles, tile_k;
    DevBuf<int> chunks; // cost-balanced row ranges for the hybrid kernel (nchunks+1 row starts)
    DevBuf<int> stiles, stile_k; // the staged kernel's schedule (<= kStageRows rows, <= kStageCap nonzeros)
    int ntiles = 0, nchunks = 0, nstiles = 0;
    int max_row = 0;
    int variant = 0; // FAST kernel variant picked by autotune_pattern
    // Identity of the pattern for the tuning cache (tuned_pick): a hash of
    // its dimensions, row offsets, a sample of its column indices and its
    // tile breaks; the transpose derives its own from the source's.
    uint64_t fp = 0;
};

// Per-device error flag the kernels write (first error wins).
int *device_error_flag();
// Reads and clears the flag; throws CudaFailure when a kernel reported one.
void check_device_error(cudaStream_t s);

// Non-owning views passed to kernels.
template <class T>
struct CsrView {
    const int *__restrict__ ro;
    const int *__restrict__ ci;
    const T *__restrict__ val;
    const int *__restrict__ tiles;
    const int *__restrict__ tile_k;
    const int *__restrict__ chunks;
    const int *__restrict__ stiles;
    const int *__restrict__ stile_k;
    int *err;
    int rows, cols, ntiles, nchunks, nstiles;
    int variant; // FAST kernel variant (autotuned per matrix)
};

template <class T>
inline CsrView<T> view(const CsrPattern32 &p, const T *val) {
    return CsrView<T>{p.ro.get(),         p.ci.get(),    val,      p.tiles.get(), p.tile_k.get(),
                      p.chunks.get(),     p.stiles.get(), p.stile_k.get(), device_error_flag(), p.rows,
                      p.cols,             p.ntiles,      p.nchunks, p.nstiles,     p.variant};
}

// Rounded multiply / add that the compiler never contracts into an FMA, so the
// sequential order matches a plain C++ `acc += v * x` on x86-64 bit for bit.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

template <class T, int NV>
struct Gathers {
    const T *__restrict__ p[NV];
};

// Epilogue interface (EpiBase has defaults for all but row_pre / row):
//   static constexpr int NR;                            reduction slots (>= 1)
//   struct Pre; __device__ Pre load(int row) const;     per-row inputs, loaded early
//   __device__ bool skip() const;                       whole launch is a no-op
//   __device__ A init(int row, int q) const;            accumulator start value
//   __device__ A gscale(int q) const;                   factor on gathered values
//   __device__ void row_pre(int row, const A (&s)[NV], const Pre &, double (&red)[NR]) const;
//   __device__ void finish(double (&red)[NR], double *scratch, int block) const;
// row_pre is called exactly once per matrix row with
//   s[q] = init(row, q) + sum_k v_k * (gscale(q) * x_q[c_k]).
// finish is called once by every thread of every CTA after its last row; it
// does the CTA-level reduction itself (scratch: 32*8 doubles of shared memory).

// Kernel variants of the FAST pass (the autotuner picks one per matrix):
//   SUB   0: the warp streams the tile's nonzeros 32 at a time and forms row
//         sums with a segmented scan (tile_kernel_fast);
//         L > 0: sub-warps of L lanes take one row each, 32/L rows per warp
//         step, and reduce with L-wide shuffles (tile_kernel_sub)
//   U     loads in flight per lane (32-nonzero steps, or L-strided steps)
//   PIPE  prefetch the next batch's indices / values while the current batch
//         gathers and reduces (SUB = 0 only)
//   MINB  resident CTAs per SM the register allocation is held to
//   HYB   > 0: the hybrid kernel (tile_kernel_hyb): a lane sums its own row
//         when it has at most HYB nonzeros, longer rows are shared by
//         sub-warps of SUB lanes (or by the whole warp)
//   STAGE > 0: the staged kernel (tile_kernel_tma) with STAGE shared-memory
//         stages per warp (HYB, SUB as in the hybrid kernel's row sums)
//   LATE  hybrid kernel only: the epilogue's per-row inputs are loaded after
//         the row sums instead of before the gathers, so they hold no
//         registers across them (for the 32-register, 16-CTA builds)
struct FastVariant {
    int u, pipe, minb, sub, hyb, stage = 0, late = 0;
};
constexpr int kFastVariants = 18;
constexpr int kTuneRounds = 4;    // timed rounds per variant in the autotuners
constexpr float kTuneKeep = 1.25f; // variants slower than this x the best leave after the first timed round
constexpr float kTuneTie = 1.02f;  // variants within this x the fastest count as tied: the lowest index wins
__host__ __device__ constexpr FastVariant fast_variant(int v) {
    return v == 0   ? FastVariant{4, 1, 12, 0, 0}
           : v == 1 ? FastVariant{8, 1, 8, 0, 0}
           : v == 2 ? FastVariant{8, 0, 12, 0, 0}
           : v == 3 ? FastVariant{16, 0, 8, 0, 0}
           : v == 4 ? FastVariant{2, 1, 16, 0, 0}
           : v == 5 ? FastVariant{2, 0, 12, 8, 0}
           : v == 6 ? FastVariant{4, 0, 12, 4, 0}
           : v == 7 ? FastVariant{2, 0, 12, 16, 0}
           : v == 8 ? FastVariant{4, 0, 8, 8, 4}
           : v == 9 ? FastVariant{2, 0, 12, 8, 2}
           : v == 10 ? FastVariant{2, 0, 12, 4, 4}
           : v == 11 ? FastVariant{8, 0, 4, 8, 8, 2}
           : v == 12 ? FastVariant{4, 0, 4, 4, 4, 2}
           : v == 13 ? FastVariant{2, 0, 16, 8, 2}
           : v == 14 ? FastVariant{4, 0, 16, 4, 1}
           : v == 15 ? FastVariant{2, 0, 16, 8, 2, 0, 1}
           : v == 16 ? FastVariant{2, 0, 16, 4, 1, 0, 1}
                     : FastVariant{2, 0, 16, 16, 2, 0, 1};
}

template <class T, class A, int NV, class Epi, int U, bool PIPE, int MINB>
__global__ void __launch_bounds__(kTileThreads, MINB)
    tile_kernel_fast(CsrView<T> M, Gathers<T, NV> g, Epi epi) {
    if (epi.skip()) return;
    constexpr int NR = Epi::NR;
    static_assert(NR >= 1, "epilogues declare at least one reduction slot");
    using Pre = typename Epi::Pre;
    __shared__ uint32_t s_mask[kWarps][kCap / 32];
    __shared__ uint8_t s_rows[kWarps][kTileRows];
    __shared__ Pre s_pre[kWarps][kTileRows];
    __shared__ double scratch[32 * 8];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    double red[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) red[r] = 0.0;
    A gs[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) gs[q] = epi.gscale(q);
    uint32_t *mask = s_mask[warp];
    uint8_t *lrows = s_rows[warp];
    Pre *lpre = s_pre[warp];

    // Per-tile reduction (opt-in): the warp's sums of this tile go to
    // epi.tile_done and start again from zero.
    auto after_tile = [&](int tile) {
        if constexpr (Epi::kPerTile) {
#pragma unroll
            for (int r = 0; r < NR; ++r) red[r] = warp_sum(red[r]);
            if (lane == 0) epi.tile_done(tile, red);
#pragma unroll
            for (int r = 0; r < NR; ++r) red[r] = 0.0;
        }
    };

    for (int tile = blockIdx.x * kWarps + warp; tile < M.ntiles; tile += gridDim.x * kWarps) {
        if (epi.skip_tile(tile)) continue;
        const int r0 = __ldg(M.tiles + tile), r1 = __ldg(M.tiles + tile + 1);
        const int k0 = __ldg(M.tile_k + tile), k1 = __ldg(M.tile_k + tile + 1);
        const int nz = k1 - k0, nrows = r1 - r0;
        if (nz > kCap) {
            // One long row, streamed by the whole warp, U loads per lane in flight.
            const Pre pre = epi.load(r0);
            A part[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) part[q] = A(0);
            for (int kb = k0; kb < k1; kb += 32 * U) {
                int c[U];
                T v[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int k = kb + 32 * u + lane;
                    c[u] = k < k1 ? __ldg(M.ci + k) : 0;
                    v[u] = k < k1 ? __ldg(M.val + k) : T(0);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (kb + 32 * u + lane < k1) {
#pragma unroll
                        for (int q = 0; q < NV; ++q)
                            part[q] += static_cast<A>(v[u]) * (gs[q] * static_cast<A>(__ldg(g.p[q] + c[u])));
                    }
                }
            }
            A sum[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) sum[q] = epi.init(r0, q) + warp_sum(part[q]);
            if (lane == 0) epi.row_pre(r0, sum, pre, red);
            after_tile(tile);
            continue;
        }
        // The first batch's loads go out before the prologue's.
        int cn[U];
        T vn[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = 32 * u + lane;
            cn[u] = k < nz ? __ldg(M.ci + k0 + k) : 0;
            vn[u] = k < nz ? __ldg(M.val + k0 + k) : T(0);
        }
        // Prologue: row-end bitmask, non-empty rows in order, per-row inputs.
        const int nwords = (nz + 31) >> 5; // kCap / 32 == 32 words: one per lane
        if (lane < nwords) mask[lane] = 0u;
        __syncwarp();
        int ne_count = 0;
#pragma unroll
        for (int rb = 0; rb < kTileRows; rb += 32) {
            if (rb >= nrows) break;
            const int i = rb + lane;
            const bool valid = i < nrows;
            bool nonempty = false;
            if (valid) {
                const int a = __ldg(M.ro + r0 + i), b = __ldg(M.ro + r0 + i + 1);
                const Pre pre = epi.load(r0 + i);
                lpre[i] = pre;
                nonempty = b > a;
                if (nonempty) {
                    const int e = b - 1 - k0;
                    atomicOr(&mask[e >> 5], 1u << (e & 31));
                } else {
                    A sum[NV];
#pragma unroll
                    for (int q = 0; q < NV; ++q) sum[q] = epi.init(r0 + i, q);
                    epi.row_pre(r0 + i, sum, pre, red);
                }
            }
            const unsigned nem = __ballot_sync(FULL, nonempty);
            if (nonempty) lrows[ne_count + __popc(nem & lt_mask)] = static_cast<uint8_t>(i);
            ne_count += __popc(nem);
        }
        __syncwarp();
        // Streaming steps with a segmented scan.
        A carry[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) carry[q] = A(0);
        int ends = 0;
        for (int jb = 0; jb < nz; jb += 32 * U) {
            int c[U];
            T v[U];
            if (!PIPE && jb > 0) {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int k = jb + 32 * u + lane;
                    c[u] = k < nz ? __ldg(M.ci + k0 + k) : 0;
                    v[u] = k < nz ? __ldg(M.val + k0 + k) : T(0);
                }
            } else {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    c[u] = cn[u];
                    v[u] = vn[u];
                }
            }
            A xv[NV][U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const bool in = jb + 32 * u + lane < nz;
#pragma unroll
                for (int q = 0; q < NV; ++q) xv[q][u] = in ? static_cast<A>(__ldg(g.p[q] + c[u])) : A(0);
            }
            const int jn = jb + 32 * U;
            if (PIPE && jn < nz) {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int k = jn + 32 * u + lane;
                    cn[u] = k < nz ? __ldg(M.ci + k0 + k) : 0;
                    vn[u] = k < nz ? __ldg(M.val + k0 + k) : T(0);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int pos = jb + 32 * u;
                if (pos >= nz) break;
                const uint32_t F = mask[pos >> 5];
                const int seg = 32 - __clz(F & lt_mask); // first lane of this lane's segment
                A p[NV];
#pragma unroll
                for (int q = 0; q < NV; ++q) p[q] = static_cast<A>(v[u]) * (gs[q] * xv[q][u]);
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
                    for (int q = 0; q < NV; ++q) {
                        const A t = __shfl_up_sync(FULL, p[q], d);
                        if (lane - d >= seg) p[q] += t;
                    }
                }
                if (seg == 0) {
#pragma unroll
                    for (int q = 0; q < NV; ++q) p[q] += carry[q];
                }
                if ((F >> lane) & 1u) {
                    const int li = lrows[ends + __popc(F & lt_mask)];
                    A sum[NV];
#pragma unroll
                    for (int q = 0; q < NV; ++q) sum[q] = epi.init(r0 + li, q) + p[q];
                    epi.row_pre(r0 + li, sum, lpre[li], red);
                }
                const bool open = ((F >> 31) & 1u) == 0u;
#pragma unroll
                for (int q = 0; q < NV; ++q) {
                    const A t = __shfl_sync(FULL, p[q], 31);
                    carry[q] = open ? t : A(0);
                }
                ends += __popc(F);
            }
        }
        __syncwarp();
        after_tile(tile);
    }
    epi.finish(red, scratch, blockIdx.x);
}

// Sub-warp variant: within a row-aligned tile, sub-warps of L lanes take one
// row each (32/L rows per warp step); the lanes of a sub-warp stride through
// the row's nonzeros U at a time and reduce with L-wide shuffles; lane 0 of
// the sub-warp runs the epilogue. Rows of a multi-row tile are short
// (<= kShortMax), so no segmented scan and no shared-memory prologue is
// needed; a single-row tile (a long row) is streamed by the whole warp. Same
// tile schedule, grid and epilogue interface as tile_kernel_fast.
template <class T, class A, int NV, class Epi, int L, int U, int MINB>
__global__ void __launch_bounds__(kTileThreads, MINB)
    tile_kernel_sub(CsrView<T> M, Gathers<T, NV> g, Epi epi) {
    static_assert(L == 2 || L == 4 || L == 8 || L == 16 || L == 32, "sub-warp width");
    if (epi.skip()) return;
    constexpr int NR = Epi::NR;
    constexpr int G = 32 / L;
    using Pre = typename Epi::Pre;
    __shared__ double scratch[32 * 8];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sl = lane % L, sw = lane / L;
    double red[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) red[r] = 0.0;
    A gs[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) gs[q] = epi.gscale(q);

    // One long row (a single-row tile), streamed by the whole warp.
    auto long_row = [&](int r0, int k0, int k1) {
        const Pre pre = epi.load(r0);
        A part[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) part[q] = A(0);
        for (int kb = k0; kb < k1; kb += 32 * U) {
            int c[U];
            T v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = kb + 32 * u + lane;
                c[u] = k < k1 ? __ldg(M.ci + k) : 0;
                v[u] = k < k1 ? __ldg(M.val + k) : T(0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (kb + 32 * u + lane < k1) {
#pragma unroll
                    for (int q = 0; q < NV; ++q)
                        part[q] += static_cast<A>(v[u]) * (gs[q] * static_cast<A>(__ldg(g.p[q] + c[u])));
                }
            }
        }
        A sum[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) sum[q] = epi.init(r0, q) + warp_sum(part[q]);
        if (lane == 0) epi.row_pre(r0, sum, pre, red);
    };
    // Short rows [r0, r1): G rows per warp step, one per sub-warp.
    auto short_rows = [&](int r0, int r1) {
        for (int rb = r0; rb < r1; rb += G) {
            const int r = rb + sw;
            const bool valid = r < r1;
            int a = 0, b = 0;
            if (valid) {
                a = __ldg(M.ro + r);
                b = __ldg(M.ro + r + 1);
            }
            Pre pre{};
            if (valid && sl == 0) pre = epi.load(r);
            A part[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) part[q] = A(0);
            int k = a + sl;
            for (; k + (U - 1) * L < b; k += U * L) {
                int c[U];
                T v[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    c[u] = __ldg(M.ci + k + u * L);
                    v[u] = __ldg(M.val + k + u * L);
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q = 0; q < NV; ++q)
                        part[q] += static_cast<A>(v[u]) * (gs[q] * static_cast<A>(__ldg(g.p[q] + c[u])));
            }
            for (; k < b; k += L) {
                const int c = __ldg(M.ci + k);
                const A v = static_cast<A>(__ldg(M.val + k));
#pragma unroll
                for (int q = 0; q < NV; ++q) part[q] += v * (gs[q] * static_cast<A>(__ldg(g.p[q] + c)));
            }
#pragma unroll
            for (int o = L / 2; o > 0; o >>= 1)
#pragma unroll
                for (int q = 0; q < NV; ++q) part[q] += __shfl_xor_sync(FULL, part[q], o, L);
            if (valid && sl == 0) {
                A sum[NV];
#pragma unroll
                for (int q = 0; q < NV; ++q) sum[q] = epi.init(r, q) + part[q];
                epi.row_pre(r, sum, pre, red);
            }
        }
    };

    if constexpr (Epi::kPerTile || Epi::kSkipTiles) {
        // Tile by tile (round robin): per-tile sums and skipped tiles.
        for (int tile = blockIdx.x * kWarps + warp; tile < M.ntiles; tile += gridDim.x * kWarps) {
            if (epi.skip_tile(tile)) continue;
            const int r0 = __ldg(M.tiles + tile), r1 = __ldg(M.tiles + tile + 1);
            const int k0 = __ldg(M.tile_k + tile), k1 = __ldg(M.tile_k + tile + 1);
            if (k1 - k0 > kCap)
                long_row(r0, k0, k1);
            else
                short_rows(r0, r1);
            if constexpr (Epi::kPerTile) {
#pragma unroll
                for (int r = 0; r < NR; ++r) red[r] = warp_sum(red[r]);
                if (lane == 0) epi.tile_done(tile, red);
#pragma unroll
                for (int r = 0; r < NR; ++r) red[r] = 0.0;
            }
        }
    } else {
        // A contiguous range of tiles per warp; consecutive short-row tiles
        // form one row span, so sub-warp steps are only partial at span ends.
        const long long W = static_cast<long long>(gridDim.x) * kWarps;
        const long long wid = static_cast<long long>(blockIdx.x) * kWarps + warp;
        const int ta = static_cast<int>(M.ntiles * wid / W), tb = static_cast<int>(M.ntiles * (wid + 1) / W);
        int t = ta;
        while (t < tb) {
            const int k0 = __ldg(M.tile_k + t), k1 = __ldg(M.tile_k + t + 1);
            if (k1 - k0 > kCap) {
                long_row(__ldg(M.tiles + t), k0, k1);
                ++t;
                continue;
            }
            int te = t + 1;
            while (te < tb && __ldg(M.tile_k + te + 1) - __ldg(M.tile_k + te) <= kCap) ++te;
            short_rows(__ldg(M.tiles + t), __ldg(M.tiles + te));
            t = te;
        }
    }
    epi.finish(red, scratch, blockIdx.x);
}

// Hybrid variant. Rows go in groups of 32, one per lane; every lane loads its
// row's bounds and epilogue inputs first. A lane with at most S nonzeros sums
// its own row (S loads in flight, left to right). The group's longer rows are
// then taken, in order, by the whole warp one at a time when a row is long
// (more than 4*L*U nonzeros), else 32/L at a time by sub-warps of L lanes
// (U loads per lane in flight, L-wide shuffle reduction); each sum goes back
// to the row's own lane by a shuffle, and every lane runs its row's epilogue,
// so the epilogue's loads and stores are coalesced across the group. With
// LATE the epilogue's inputs are loaded after the sums (other warps hide that
// latency at full occupancy) rather than held in registers across the gathers.
// Work: cost-balanced row ranges (chunks, about kChunkCost nonzeros-plus-4-
// per-row each) round robin over the persistent grid, or the tile schedule's
// tiles when the epilogue reduces per tile or skips tiles.
constexpr int kChunkCost = 1024;
constexpr int kRowCost = 4;

template <class T, class A, int NV, class Epi, int S, int L, int U, int MINB, bool LATE>
__global__ void __launch_bounds__(kTileThreads, MINB)
    tile_kernel_hyb(CsrView<T> M, Gathers<T, NV> g, Epi epi) {
    static_assert(L == 2 || L == 4 || L == 8 || L == 16, "sub-warp width");
    if (epi.skip()) return;
    constexpr int NR = Epi::NR;
    constexpr int G = 32 / L;
    constexpr int kWarpRow = 4 * L * U; // longer rows take the whole warp
    using Pre = typename Epi::Pre;
    __shared__ double scratch[32 * 8];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sl = lane % L, sw = lane / L;
    const unsigned lt_mask = (1u << lane) - 1u;
    double red[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) red[r] = 0.0;
    A gs[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) gs[q] = epi.gscale(q);

    // rows [rb, re), re - rb <= 32; a, b: this lane's row bounds (0 when r >= re)
    auto group = [&](int rb, int re, int a, int b) {
        const int r = rb + lane;
        const bool valid = r < re;
        Pre pre{};
        if (!LATE && valid) pre = epi.load(r);
        const int len = b - a;
        A sum[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) sum[q] = A(0);
        if (valid && len <= S) {
            int c[S];
            T v[S];
#pragma unroll
            for (int u = 0; u < S; ++u) {
                c[u] = u < len ? __ldg(M.ci + a + u) : 0;
                v[u] = u < len ? __ldg(M.val + a + u) : T(0);
            }
#pragma unroll
            for (int u = 0; u < S; ++u)
                if (u < len) {
#pragma unroll
                    for (int q = 0; q < NV; ++q)
                        sum[q] += static_cast<A>(v[u]) * (gs[q] * static_cast<A>(__ldg(g.p[q] + c[u])));
                }
        }
        unsigned lm = __ballot_sync(FULL, valid && len > S);
        while (lm) {
            const int first = __ffs(lm) - 1;
            const int fa = __shfl_sync(FULL, a, first), fb = __shfl_sync(FULL, b, first);
            if (fb - fa > kWarpRow) {
                // one long row, the whole warp
                A part[NV];
#pragma unroll
                for (int q = 0; q < NV; ++q) part[q] = A(0);
                for (int kb = fa; kb < fb; kb += 32 * U) {
                    int c[U];
                    T v[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int k = kb + 32 * u + lane;
                        c[u] = k < fb ? __ldg(M.ci + k) : 0;
                        v[u] = k < fb ? __ldg(M.val + k) : T(0);
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        if (kb + 32 * u + lane < fb) {
#pragma unroll
                            for (int q = 0; q < NV; ++q)
                                part[q] += static_cast<A>(v[u]) * (gs[q] * static_cast<A>(__ldg(g.p[q] + c[u])));
                        }
                }
#pragma unroll
                for (int q = 0; q < NV; ++q) {
                    const A t = warp_sum(part[q]);
                    if (lane == first) sum[q] = t;
                }
                lm &= lm - 1u;
                continue;
            }
            // up to G rows, one per sub-warp: sub-warp w takes the (w+1)-th set bit
            const unsigned pos = __fns(lm, 0, sw + 1);
            const bool has = pos < 32u;
            const int src = has ? static_cast<int>(pos) : 0;
            const int ra = __shfl_sync(FULL, a, src), rz = __shfl_sync(FULL, b, src);
            A part[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) part[q] = A(0);
            if (has) {
                for (int kb = ra + sl; kb < rz; kb += U * L) {
                    int c[U];
                    T v[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int k = kb + u * L;
                        c[u] = k < rz ? __ldg(M.ci + k) : 0;
                        v[u] = k < rz ? __ldg(M.val + k) : T(0);
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        if (kb + u * L < rz) {
#pragma unroll
                            for (int q = 0; q < NV; ++q)
                                part[q] += static_cast<A>(v[u]) * (gs[q] * static_cast<A>(__ldg(g.p[q] + c[u])));
                        }
                }
            }
#pragma unroll
            for (int o = L / 2; o > 0; o >>= 1)
#pragma unroll
                for (int q = 0; q < NV; ++q) part[q] += __shfl_xor_sync(FULL, part[q], o, L);
            // back to the owners: the lane of the k-th set bit (k < G) reads sub-warp k's lane 0
            const int rank = __popc(lm & lt_mask);
            const bool mine = ((lm >> lane) & 1u) && rank < G;
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                const A t = __shfl_sync(FULL, part[q], mine ? rank * L : 0);
                if (mine) sum[q] = t;
            }
#pragma unroll
            for (int i = 0; i < G; ++i) lm &= lm - 1u;
        }
        if (valid) {
            if constexpr (LATE) pre = epi.load(r);
            A s2[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) s2[q] = epi.init(r, q) + sum[q];
            epi.row_pre(r, s2, pre, red);
        }
    };

    const int W = gridDim.x * kWarps;
    const int wid = blockIdx.x * kWarps + warp;
    if constexpr (Epi::kPerTile || Epi::kSkipTiles) {
        for (int tile = wid; tile < M.ntiles; tile += W) {
            if (epi.skip_tile(tile)) continue;
            const int r0 = __ldg(M.tiles + tile), r1 = __ldg(M.tiles + tile + 1);
            for (int rb = r0; rb < r1; rb += 32) {
                const int re = rb + 32 < r1 ? rb + 32 : r1;
                int a = 0, b = 0;
                if (rb + lane < re) {
                    a = __ldg(M.ro + rb + lane);
                    b = __ldg(M.ro + rb + lane + 1);
                }
                group(rb, re, a, b);
            }
            if constexpr (Epi::kPerTile) {
#pragma unroll
                for (int r = 0; r < NR; ++r) red[r] = warp_sum(red[r]);
                if (lane == 0) epi.tile_done(tile, red);
#pragma unroll
                for (int r = 0; r < NR; ++r) red[r] = 0.0;
            }
        }
    } else {
        for (int ch = wid; ch < M.nchunks; ch += W) {
            const int r0 = __ldg(M.chunks + ch), r1 = __ldg(M.chunks + ch + 1);
            for (int rb = r0; rb < r1; rb += 32) {
                const int re = rb + 32 < r1 ? rb + 32 : r1;
                int a = 0, b = 0;
                if (rb + lane < re) {
                    a = __ldg(M.ro + rb + lane);
                    b = __ldg(M.ro + rb + lane + 1);
                }
                group(rb, re, a, b);
            }
        }
    }
    epi.finish(red, scratch, blockIdx.x);
}

// Staged variant (sm_90+ bulk copies). Each warp runs its own two-stage
// pipeline over the staged schedule (tiles of <= kStageRows rows and
// <= kStageCap nonzeros, or one longer row taken in kStageCap pieces): one
// lane issues cp.async.bulk copies of the next piece's column indices and
// values (16-byte aligned: the piece is widened to whole 4-element groups,
// inside the kPad padding) into shared memory, completing on an mbarrier,
// while the warp works on the current piece. So the nonzero streams bypass
// the L1 load path and only the random gathers of x (and the epilogue's
// per-row inputs) go through it. Per piece: every lane loads its row's bounds
// and epilogue inputs (one row per lane), the warp gathers x for all the
// piece's nonzeros (U per lane in flight) and overwrites each staged value
// with its product, then the row sums are read back from shared memory: a
// lane sums its own row when it has at most S nonzeros, longer rows go to
// sub-warps of L lanes or to the whole warp; each lane runs its row's
// epilogue. A long row's pieces accumulate in a warp-wide carry. Waits are
// bounded: a barrier that never completes sets the device error flag, the
// warp stops taking work and waits (bounded) for its own copies in flight.
// Not for epilogues that reduce per tile or skip tiles (they use the main
// schedule's tile numbers); launch_fast gives those the hybrid kernel.
template <class T, class A, int NV, class Epi, int S, int L, int U, int MINB>
__global__ void __launch_bounds__(kTileThreads, MINB)
    tile_kernel_tma(CsrView<T> M, Gathers<T, NV> g, Epi epi) {
    static_assert(NV == 1 && sizeof(A) == sizeof(T), "products overwrite the staged values");
    static_assert(L == 2 || L == 4 || L == 8 || L == 16, "sub-warp width");
    if (epi.skip()) return;
    constexpr int NR = Epi::NR;
    constexpr int G = 32 / L;
    constexpr int CAPR = kStageSlots;
    using Pre = typename Epi::Pre;
    // dynamic shared memory: [warp][stage][CAPR] indices, then values
    extern __shared__ __align__(16) unsigned char stage_smem[];
    auto s_ci = reinterpret_cast<int (*)[2][CAPR]>(stage_smem);
    auto s_v = reinterpret_cast<T (*)[2][CAPR]>(stage_smem + sizeof(int) * kWarps * 2 * CAPR);
    __shared__ alignas(8) uint64_t s_bar[kWarps][2];
    __shared__ double scratch[32 * 8];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sl = lane % L, sw = lane / L;
    const unsigned lt_mask = (1u << lane) - 1u;
    uint64_t *bar = s_bar[warp];
    if (lane == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncwarp();
    double red[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) red[r] = 0.0;
    const A gs = epi.gscale(0);
    const T *__restrict__ x = g.p[0];

    const int W = gridDim.x * kWarps;
    const int wid = blockIdx.x * kWarps + warp;
    // the warp's pieces: tiles wid, wid + W, ...; a tile of n nonzeros has
    // max(1, ceil(n / kStageCap)) pieces
    auto next = [&](int &t, int &p) {
        const int n = __ldg(M.stile_k + t + 1) - __ldg(M.stile_k + t);
        if ((p + 1) * kStageCap < n) {
            ++p;
        } else {
            t += W;
            p = 0;
        }
    };
    auto issue = [&](int st, int t, int p) {
        if (lane == 0) {
            const int a = __ldg(M.stile_k + t), b = __ldg(M.stile_k + t + 1);
            const int k0 = a + p * kStageCap, k1 = min(b, k0 + kStageCap);
            const int kb = k0 & ~3;
            const int n = (k1 - kb + 3) & ~3;
            mbar_arrive_expect_tx(&bar[st], static_cast<uint32_t>(n * (4 + sizeof(T))));
            if (n > 0) {
                bulk_g2s(s_ci[warp][st], M.ci + kb, static_cast<uint32_t>(n * 4), &bar[st]);
                bulk_g2s(s_v[warp][st], M.val + kb, static_cast<uint32_t>(n * sizeof(T)), &bar[st]);
            }
        }
    };

    uint32_t phase[2] = {0u, 0u};
    bool pending[2] = {false, false};
    bool failed = false;
    int t = wid, p = 0, st = 0;
    A carry = A(0); // a long row's sum over its earlier pieces
    if (t < M.nstiles) {
        issue(0, t, 0);
        pending[0] = true;
    }
    while (t < M.nstiles) {
        int tn = t, pn = p;
        next(tn, pn);
        if (tn < M.nstiles) {
            issue(st ^ 1, tn, pn);
            pending[st ^ 1] = true;
        }
        const int r0 = __ldg(M.stiles + t), r1 = __ldg(M.stiles + t + 1);
        const int a = __ldg(M.stile_k + t), b = __ldg(M.stile_k + t + 1);
        const int k0 = a + p * kStageCap, k1 = min(b, k0 + kStageCap);
        const bool last_piece = k1 == b;
        const bool long_row = b - a > kStageCap; // one row in several pieces
        // this piece's rows: bounds and epilogue inputs, one row per lane
        const int r = r0 + lane;
        const bool valid = !long_row && r < r1;
        int ra = 0, rz = 0;
        Pre pre{};
        if (valid) {
            ra = __ldg(M.ro + r);
            rz = __ldg(M.ro + r + 1);
            pre = epi.load(r);
        } else if (long_row && lane == 0 && last_piece) {
            pre = epi.load(r0);
        }
        if (!__all_sync(FULL, mbar_wait_bounded(&bar[st], phase[st]))) {
            if (lane == 0) atomicCAS(M.err, 0, static_cast<int>(kDevErrBarrierTimeout));
            failed = true;
            break;
        }
        phase[st] ^= 1u;
        pending[st] = false;
        const int kb = k0 & ~3, off = k0 - kb, nz = k1 - k0;
        const int *sc = s_ci[warp][st] + off;
        T *sv = s_v[warp][st] + off;
        // gathers: products over the staged values
        for (int j = lane; j < nz; j += 32 * U) {
            int c[U];
            T xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) c[u] = j + 32 * u < nz ? sc[j + 32 * u] : 0;
#pragma unroll
            for (int u = 0; u < U; ++u) xv[u] = j + 32 * u < nz ? __ldg(x + c[u]) : T(0);
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (j + 32 * u < nz) sv[j + 32 * u] = static_cast<T>(static_cast<A>(sv[j + 32 * u]) * (gs * static_cast<A>(xv[u])));
        }
        __syncwarp();
        if (long_row) {
            A part = A(0);
            for (int j = lane; j < nz; j += 32) part += static_cast<A>(sv[j]);
            carry += warp_sum(part);
            if (last_piece) {
                if (lane == 0) {
                    A s2[1] = {epi.init(r0, 0) + carry};
                    epi.row_pre(r0, s2, pre, red);
                }
                carry = A(0);
            }
        } else {
            // row sums from shared memory; local offsets relative to k0
            const int la = ra - k0, len = rz - ra;
            A sum = A(0);
            if (valid && len <= S)
                for (int j = 0; j < len; ++j) sum += static_cast<A>(sv[la + j]);
            unsigned lm = __ballot_sync(FULL, valid && len > S);
            while (lm) {
                const int first = __ffs(lm) - 1;
                const int fa = __shfl_sync(FULL, la, first), fl = __shfl_sync(FULL, len, first);
                if (fl > 4 * L) {
                    A part = A(0);
                    for (int j = lane; j < fl; j += 32) part += static_cast<A>(sv[fa + j]);
                    part = warp_sum(part);
                    if (lane == first) sum = part;
                    lm &= lm - 1u;
                    continue;
                }
                const unsigned pos = __fns(lm, 0, sw + 1);
                const bool has = pos < 32u;
                const int src = has ? static_cast<int>(pos) : 0;
                const int qa = __shfl_sync(FULL, la, src), ql = __shfl_sync(FULL, len, src);
                A part = A(0);
                if (has)
                    for (int j = sl; j < ql; j += L) part += static_cast<A>(sv[qa + j]);
#pragma unroll
                for (int o = L / 2; o > 0; o >>= 1) part += __shfl_xor_sync(FULL, part, o, L);
                const int rank = __popc(lm & lt_mask);
                const bool mine = ((lm >> lane) & 1u) && rank < G;
                const A tv = __shfl_sync(FULL, part, mine ? rank * L : 0);
                if (mine) sum = tv;
#pragma unroll
                for (int i = 0; i < G; ++i) lm &= lm - 1u;
            }
            if (valid) {
                A s2[1] = {epi.init(r, 0) + sum};
                epi.row_pre(r, s2, pre, red);
            }
        }
        // every lane is done with this stage before a copy overwrites it
        fence_proxy_async_smem();
        __syncwarp();
        t = tn;
        p = pn;
        st ^= 1;
    }
    if (failed) {
        // wait (bounded) for this warp's copies still in flight
        for (int i = 0; i < 2; ++i)
            if (pending[i]) mbar_wait_bounded(&bar[i], phase[i]);
    }
    epi.finish(red, scratch, blockIdx.x);
}

// Parity kernel: one thread per row, the reference's left-to-right order.
template <class T, class A, int NV, class Epi>
__global__ void __launch_bounds__(kTileThreads)
    tile_kernel_exact(CsrView<T> M, Gathers<T, NV> g, Epi epi) {
    if (epi.skip()) return;
    constexpr int NR = Epi::NR;
    __shared__ double scratch[32 * 8];
    double red[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) red[r] = 0.0;
    A gs[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) gs[q] = epi.gscale(q);
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M.rows; r += gridDim.x * blockDim.x) {
        const auto pre = epi.load(r);
        A s[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) s[q] = epi.init(r, q);
        const int b = M.ro[r], e = M.ro[r + 1];
        for (int k = b; k < e; ++k) {
            const int c = M.ci[k];
            const A v = static_cast<A>(M.val[k]);
#pragma unroll
            for (int q = 0; q < NV; ++q) s[q] = add_rn(s[q], mul_rn(v, mul_rn(gs[q], static_cast<A>(g.p[q][c]))));
        }
        epi.row_pre(r, s, pre, red);
    }
    epi.finish(red, scratch, blockIdx.x);
}

template <class K>
inline int resident_grid(K kernel, int smem = 0) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kTileThreads, smem);
    per = per < 1 ? 1 : (per > kMaxGridPerSM ? kMaxGridPerSM : per);
    const int r = sms * per;
    return r < kMaxGrid ? r : kMaxGrid;
}

template <class T, class A, int NV, class Epi, int V>
inline int launch_fast(const CsrView<T> &M, const Gathers<T, NV> &g, const Epi &epi, cudaStream_t s) {
    constexpr FastVariant fv = fast_variant(V);
    void (*kernel)(CsrView<T>, Gathers<T, NV>, Epi);
    constexpr bool staged_ok = NV == 1 && sizeof(A) == sizeof(T) && !Epi::kPerTile && !Epi::kSkipTiles;
    if constexpr (fv.stage > 0 && staged_ok)
        kernel = tile_kernel_tma<T, A, NV, Epi, fv.hyb, fv.sub, fv.u, fv.minb>;
    else if constexpr (fv.hyb > 0)
        kernel = tile_kernel_hyb<T, A, NV, Epi, fv.hyb, fv.sub, fv.u, fv.minb, fv.late != 0>;
    else if constexpr (fv.sub > 0)
        kernel = tile_kernel_sub<T, A, NV, Epi, (fv.sub > 0 ? fv.sub : 32), fv.u, fv.minb>;
    else
        kernel = tile_kernel_fast<T, A, NV, Epi, fv.u, fv.pipe != 0, fv.minb>;
    constexpr bool staged = fv.stage > 0 && staged_ok;
    constexpr int smem = staged ? stage_smem_bytes<T>() : 0;
    static const int resident = [&] {
        if (smem > 0) VK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        return resident_grid(kernel, smem);
    }();
    const int need = ((staged ? M.nstiles : M.ntiles) + kWarps - 1) / kWarps;
    const int grid = need < resident ? (need > 0 ? need : 1) : resident;
    kernel<<<grid, kTileThreads, smem, s>>>(M, g, epi);
    VK_LAUNCH_CHECK();
    return grid;
}

// Times launch(v) -- one launch of a pass with FAST variant v on stream s --
// for every variant and returns the pick: one untimed round, one timed
// round over all variants, then kTuneRounds - 1 rounds over those within
// kTuneKeep of the best. Rounds interleave the variants (clock drift hits
// them alike) and each variant keeps its best round in best[v] (a dropped
// variant: its first timed round). A round's launches queue back to back,
// one event pair each, and the host waits once per round. The pick is the
// lowest-numbered variant within kTuneTie of the fastest, so near-ties (which
// timing noise could order either way) resolve the same way every time.
template <class L>
int tune_variants(L &&launch, cudaStream_t s, float (&best)[kFastVariants]) {
    cudaEvent_t ev[2 * kFastVariants];
    for (cudaEvent_t &e : ev) VK_CUDA(cudaEventCreate(&e));
    bool keep[kFastVariants];
    for (int v = 0; v < kFastVariants; ++v) {
        launch(v);
        best[v] = 1e30f;
        keep[v] = true;
    }
    for (int round = 0; round < kTuneRounds; ++round) {
        for (int v = 0; v < kFastVariants; ++v) {
            if (!keep[v]) continue;
            VK_CUDA(cudaEventRecord(ev[2 * v], s));
            launch(v);
            VK_CUDA(cudaEventRecord(ev[2 * v + 1], s));
        }
        VK_CUDA(cudaStreamSynchronize(s));
        float lo = 1e30f;
        for (int v = 0; v < kFastVariants; ++v) {
            if (!keep[v]) continue;
            float ms = 0.f;
            VK_CUDA(cudaEventElapsedTime(&ms, ev[2 * v], ev[2 * v + 1]));
            best[v] = std::min(best[v], ms);
            lo = std::min(lo, best[v]);
        }
        if (round == 0)
            for (int v = 0; v < kFastVariants; ++v) keep[v] = best[v] <= kTuneKeep * lo;
    }
    for (cudaEvent_t &e : ev) cudaEventDestroy(e);
    const float lo = *std::min_element(best, best + kFastVariants);
    for (int v = 0; v < kFastVariants; ++v)
        if (best[v] <= kTuneTie * lo) return v;
    return static_cast<int>(std::min_element(best, best + kFastVariants) - best);
}

// Launches the pass; returns the number of CTAs (the entries a per-CTA
// partial-sum epilogue writes), 0 when the matrix has no rows. The grid is
// persistent: resident CTAs per SM (occupancy calculator, at most
// kMaxGridPerSM) times the SM count, or fewer when there is less work.
template <class T, class A, int NV, bool EXACT, class Epi>
inline int launch_tiles(const CsrView<T> &M, const Gathers<T, NV> &g, const Epi &epi, cudaStream_t s) {
    if (M.rows <= 0) return 0;
    if (EXACT) {
        static const int resident = resident_grid(tile_kernel_exact<T, A, NV, Epi>);
        const int need = (M.rows + kTileThreads - 1) / kTileThreads;
        const int grid = need < resident ? need : resident;
        tile_kernel_exact<T, A, NV, Epi><<<grid, kTileThreads, 0, s>>>(M, g, epi);
        VK_LAUNCH_CHECK();
        return grid;
    }
    switch (M.variant) {
    case 1: return launch_fast<T, A, NV, Epi, 1>(M, g, epi, s);
    case 2: return launch_fast<T, A, NV, Epi, 2>(M, g, epi, s);
    case 3: return launch_fast<T, A, NV, Epi, 3>(M, g, epi, s);
    case 4: return launch_fast<T, A, NV, Epi, 4>(M, g, epi, s);
    case 5: return launch_fast<T, A, NV, Epi, 5>(M, g, epi, s);
    case 6: return launch_fast<T, A, NV, Epi, 6>(M, g, epi, s);
    case 7: return launch_fast<T, A, NV, Epi, 7>(M, g, epi, s);
    case 8: return launch_fast<T, A, NV, Epi, 8>(M, g, epi, s);
    case 9: return launch_fast<T, A, NV, Epi, 9>(M, g, epi, s);
    case 10: return launch_fast<T, A, NV, Epi, 10>(M, g, epi, s);
    case 11: return launch_fast<T, A, NV, Epi, 11>(M, g, epi, s);
    case 12: return launch_fast<T, A, NV, Epi, 12>(M, g, epi, s);
    case 13: return launch_fast<T, A, NV, Epi, 13>(M, g, epi, s);
    case 14: return launch_fast<T, A, NV, Epi, 14>(M, g, epi, s);
    case 15: return launch_fast<T, A, NV, Epi, 15>(M, g, epi, s);
    case 16: return launch_fast<T, A, NV, Epi, 16>(M, g, epi, s);
    case 17: return launch_fast<T, A, NV, Epi, 17>(M, g, epi, s);

    default: return launch_fast<T, A, NV, Epi, 0>(M, g, epi, s);
    }
}

// Epilogue base: one unused reduction slot, no prefetch, unit gather scale,
// zero start, never skipped. Derived epilogues define row() (through EpiRow)
// or row_pre().
template <class A>
struct EpiBase {
    static constexpr int NR = 1;
    // kPerTile: after each warp-tile the warp's reductions are summed and
    // passed to tile_done(tile, red) (FAST order only); skip_tile(tile) lets
    // a pass leave whole tiles untouched.
    static constexpr bool kPerTile = false;
    static constexpr bool kSkipTiles = false; // true when skip_tile is overridden
    struct Pre {};
    __device__ Pre load(int) const { return Pre{}; }
    __device__ A init(int, int) const { return A(0); }
    __device__ A gscale(int) const { return A(1); }
    __device__ bool skip() const { return false; }
    __device__ bool skip_tile(int) const { return false; }
    template <int NR>
    __device__ void tile_done(int, double (&)[NR]) const {}
    template <int NR>
    __device__ void finish(double (&)[NR], double *, int) const {}
};

// Adapter: epilogues without a prefetch implement row(i, s, red).
template <class A, class Derived>
struct EpiRow : EpiBase<A> {
    template <int NV, int NR>
    __device__ void row_pre(int i, const A (&s)[NV], const typename EpiBase<A>::Pre &, double (&red)[NR]) const {
        static_cast<const Derived *>(this)->row(i, s, red);
    }
};

// ---- setup (vk_csr.cu) ------------------------------------------------------

// Uploads an int64 CSR pattern, converts it to int32 on the device and builds
// the tile schedule. The pattern must already be validated.
void upload_pattern(int64_t rows, int64_t cols, const int64_t *h_ro, const int64_t *h_ci, CsrPattern32 &out,
                    cudaStream_t s);
// Builds the tile schedule of an int32 pattern already on the device.
// `breaks` (device, rows+1 bytes, optional): a tile must start where breaks[r] != 0.
void build_tiles(CsrPattern32 &p, cudaStream_t s, const unsigned char *breaks = nullptr);
// Transposes `a` on the device by a stable radix sort of the column indices
// (rows ascend within each column). perm[t] = source position of entry t.
void transpose_pattern(const CsrPattern32 &a, CsrPattern32 &at, DevBuf<int> &perm, cudaStream_t s);

// Column order of the FAST passes (VIKALP_B200_COLUMN_ORDER = auto | keep |
// count): `count` renames a pattern's columns in order of decreasing
// nonzero count, ties in their original order; `auto` does so when the
// pattern has at least kOrderMinNnz nonzeros and the counts' coefficient of
// variation is at least kOrderMinSpread (skewed, power-law columns). The
// transpose's rows then come longest first, which evens the work of the
// warps of the transposed pass, and the most gathered entries of x sit
// together. Parity modes keep the order.
enum class ColumnOrder { Auto, Keep, Count };
constexpr int64_t kOrderMinNnz = int64_t(1) << 20;
constexpr double kOrderMinSpread = 1.0;
ColumnOrder column_order_mode(); // throws InvalidInput on a bad value
// Renames a's columns (a.ci, a.fp) when `mode` asks for it, all on the
// device (a stable radix sort of the counts); new_to_old[j'] is the original
// column of new column j'. Returns false, leaving everything untouched, when
// the order is kept.
bool order_columns_by_count(CsrPattern32 &a, ColumnOrder mode, DevBuf<int> &new_to_old, cudaStream_t s);
// dst[perm[t]] = src[t], t < n
void scatter_values(const int *perm, const double *src, double *dst, int64_t n, cudaStream_t s);
// dst[t] = src[perm[t]] (optionally converting the value type).
template <class TD, class TS>
void gather_values(const int *perm, const TS *src, TD *dst, int64_t nnz, cudaStream_t s);
// dst[k] = (TD) src[k].
template <class TD, class TS>
void convert_values(const TS *src, TD *dst, int64_t n, cudaStream_t s);
// Expands row offsets to a row index per nonzero.
void expand_rows(const CsrPattern32 &p, int *rowidx, cudaStream_t s);
// Autotuner: times every FAST kernel variant on this matrix (a plain product
// into scratch vectors, a few launches each) and stores the fastest in
// p.variant. Matrices below `min_nnz` keep variant 0.
// The environment variable VIKALP_B200_VARIANT=<v> (0 <= v < kFastVariants)
// pins every pattern (and every tuned pass) to variant v instead, at any size:
// a knob for tests that run whole solves on each kernel variant.
template <class T>
void autotune_pattern(CsrPattern32 &p, const T *val, cudaStream_t s, int64_t min_nnz = 200000);
// The pinned variant, or -1.
int forced_variant();

// Process-wide cache of tuning results. `key` identifies what was tuned: a
// pattern fingerprint (CsrPattern32::fp) mixed with a tag naming the pass and
// precision (tune_key). The first call for a key on a device runs tune() and
// stores its pick; later calls -- another handle on the same matrix, another
// solve -- return the stored pick without timing anything, so the same input
// runs the same kernel variant (and gives the same bits) for the life of the
// process. Thread-safe; if two threads tune one key at once, the first stored
// pick is the one both return.
template <class F>
int tuned_pick(uint64_t key, F &&tune);
uint64_t tune_key(uint64_t fingerprint, const char *tag, int value_bytes);
// Looks up a stored pick; false when the key has none yet.
bool cached_pick(uint64_t key, int &variant);
// Stores a pick (unless one is stored already) and returns the stored one.
int store_pick(uint64_t key, int variant);

template <class F>
int tuned_pick(uint64_t key, F &&tune) {
    int v = 0;
    if (cached_pick(key, v)) return v;
    return store_pick(key, tune());
}

// Fingerprint of a host CSR pattern (rows, cols, every 61st row offset and
// column index and the last of each), FNV-1a over 64-bit words; it keys the
// kernel-pick cache only.
uint64_t pattern_fingerprint(int64_t rows, int64_t cols, const int64_t *ro, const int64_t *ci);
uint64_t mix_fingerprint(uint64_t a, uint64_t b);

} // namespace vk
