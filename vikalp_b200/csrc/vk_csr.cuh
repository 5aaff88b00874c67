// Device CSR storage and the tile-stream sparse pass used by every product.
//
// Layout in HBM (per matrix): int32 row offsets [rows+1], int32 column indices
// [nnz], values [nnz] (float64 or float32), and an int32 tile schedule
// [ntiles+1] of row starts. A tile is either
//   * a run of consecutive rows holding at most kNzTile nonzeros and at most
//     kRowsMax rows, or
//   * one row longer than kNzTile / 2 ("long row").
// One CTA streams one tile: the nonzeros of the tile are contiguous in memory,
// so column indices and values are read fully coalesced, the gathers of x are
// all independent, and the products land in shared memory. Rows are then
// summed from shared memory -- one thread per row, left to right (the
// reference CPU order, cpu_ops.cpp:418-427) for short rows, one warp per row
// for rows longer than kShortRow -- and handed to a fused epilogue (the PDHG
// primal or dual update, a residual, ...), so no product vector is written
// back to HBM.
#pragma once

#include "vk_common.cuh"

namespace vk {

constexpr int kTileThreads = 256;
constexpr int kNzTile = 2048;            // max nonzeros per multi-row tile
constexpr int kHalfTile = kNzTile / 2;   // rows longer than this get their own tile
constexpr int kRowsMax = 512;            // max rows per tile
constexpr int kShortRow = 32;            // rows up to this length: one thread
constexpr int kPer = kNzTile / kTileThreads;

// Owning device CSR pattern + tile schedule (values are stored by the user).
struct CsrPattern32 {
    int rows = 0, cols = 0;
    int64_t nnz = 0;
    DevBuf<int> ro, ci, tiles;
    int ntiles = 0;
    int max_row = 0;
};

// Non-owning views passed to kernels.
template <class T>
struct CsrView {
    const int *__restrict__ ro;
    const int *__restrict__ ci;
    const T *__restrict__ val;
    const int *__restrict__ tiles;
    int rows, cols, ntiles;
};

template <class T>
inline CsrView<T> view(const CsrPattern32 &p, const T *val) {
    return CsrView<T>{p.ro.get(), p.ci.get(), val, p.tiles.get(), p.rows, p.cols, p.ntiles};
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

// Shared memory of one tile pass.
template <class A, int NV>
struct TileSmem {
    A prod[NV][kNzTile];
    int rofs[kRowsMax + 1];
    int long_list[kRowsMax];
    int n_long;
    double red[32 * 8];
};

// The tile pass. Epi must provide:
//   static constexpr int NR;                           reduction slots
//   __device__ A init(int row, int q) const;           accumulator start value
//   __device__ A gscale(int q) const;                  factor on gathered values (1 = none)
//   __device__ void row(int row, const A (&s)[NV], double (&red)[NR]) const;
//   __device__ void finish(double (&red)[NR], double *scratch, int tile) const;
// `row` is called exactly once per row of the tile. `finish` is called by
// every thread of the CTA after all rows are done (it must do its own block
// reduction; scratch is 32*8 doubles of shared memory).
template <class T, class A, int NV, bool EXACT, class Epi>
__device__ __forceinline__ void tile_pass(const CsrView<T> &M, const Gathers<T, NV> &g, const Epi &epi,
                                          TileSmem<A, NV> &sm) {
    constexpr int NR = Epi::NR;
    static_assert(NR >= 1, "epilogues declare at least one reduction slot");
    const int tile = blockIdx.x;
    const int tid = threadIdx.x;
    const int r0 = M.tiles[tile], r1 = M.tiles[tile + 1];
    const int k0 = M.ro[r0], k1 = M.ro[r1];
    const int nz = k1 - k0, nrows = r1 - r0;
    double red[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) red[r] = 0.0;

    if (nz > kNzTile) {
        // One long row, streamed straight from HBM by the whole CTA.
        A s[NV];
        if (EXACT) {
            if (tid == 0) {
#pragma unroll
                for (int q = 0; q < NV; ++q) s[q] = epi.init(r0, q);
                for (int k = k0; k < k1; ++k) {
                    const int c = M.ci[k];
                    const A v = static_cast<A>(M.val[k]);
#pragma unroll
                    for (int q = 0; q < NV; ++q)
                        s[q] = add_rn(s[q], mul_rn(v, mul_rn(epi.gscale(q), static_cast<A>(g.p[q][c]))));
                }
                epi.row(r0, s, red);
            }
        } else {
            double part[NV > 0 ? NV : 1];
#pragma unroll
            for (int q = 0; q < NV; ++q) part[q] = 0.0;
#pragma unroll 4
            for (int k = k0 + tid; k < k1; k += kTileThreads) {
                const int c = __ldg(M.ci + k);
                const A v = static_cast<A>(__ldg(M.val + k));
#pragma unroll
                for (int q = 0; q < NV; ++q) part[q] += static_cast<double>(v * static_cast<A>(__ldg(g.p[q] + c)));
            }
            block_sum<NV>(part, sm.red);
            if (tid == 0) {
#pragma unroll
                for (int q = 0; q < NV; ++q)
                    s[q] = epi.init(r0, q) + static_cast<A>(part[q]) * epi.gscale(q);
                epi.row(r0, s, red);
            }
        }
        __syncthreads();
        epi.finish(red, sm.red, tile);
        return;
    }

    // Multi-row tile: stage the products in shared memory.
    if (tid == 0) sm.n_long = 0;
    for (int i = tid; i <= nrows; i += kTileThreads) sm.rofs[i] = M.ro[r0 + i] - k0;
    {
        int cidx[kPer];
        T v[kPer];
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int k = tid + j * kTileThreads;
            if (k < nz) {
                cidx[j] = __ldg(M.ci + k0 + k);
                v[j] = __ldg(M.val + k0 + k);
            }
        }
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int k = tid + j * kTileThreads;
            if (k < nz) {
#pragma unroll
                for (int q = 0; q < NV; ++q) {
                    A xv = static_cast<A>(__ldg(g.p[q] + cidx[j]));
                    if (EXACT) xv = mul_rn(epi.gscale(q), xv);
                    sm.prod[q][k] = mul_rn(static_cast<A>(v[j]), xv);
                }
            }
        }
    }
    __syncthreads();
    for (int i = tid; i < nrows; i += kTileThreads) {
        const int a = sm.rofs[i], b = sm.rofs[i + 1];
        if (EXACT || b - a <= kShortRow) {
            A s[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                A acc = epi.init(r0 + i, q);
                if (EXACT) {
                    for (int k = a; k < b; ++k) acc = add_rn(acc, sm.prod[q][k]);
                } else {
                    A t = A(0);
                    for (int k = a; k < b; ++k) t += sm.prod[q][k];
                    acc = acc + t * epi.gscale(q);
                }
                s[q] = acc;
            }
            epi.row(r0 + i, s, red);
        } else {
            const int slot = atomicAdd(&sm.n_long, 1);
            sm.long_list[slot] = i;
        }
    }
    if (!EXACT) {
        __syncthreads();
        const int nl = sm.n_long;
        const int lane = tid & 31, warp = tid >> 5;
        for (int w = warp; w < nl; w += kTileThreads / 32) {
            const int i = sm.long_list[w];
            const int a = sm.rofs[i], b = sm.rofs[i + 1];
            A s[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                A t = A(0);
                for (int k = a + lane; k < b; k += 32) t += sm.prod[q][k];
                t = warp_sum(t);
                s[q] = epi.init(r0 + i, q) + t * epi.gscale(q);
            }
            if (lane == 0) epi.row(r0 + i, s, red);
        }
    }
    __syncthreads();
    epi.finish(red, sm.red, tile);
}

template <class T, class A, int NV, bool EXACT, class Epi>
__global__ void __launch_bounds__(kTileThreads)
    tile_kernel(CsrView<T> M, Gathers<T, NV> g, Epi epi) {
    if (epi.skip()) return;
    __shared__ TileSmem<A, NV> sm;
    tile_pass<T, A, NV, EXACT, Epi>(M, g, epi, sm);
}

template <class T, class A, int NV, bool EXACT, class Epi>
inline void launch_tiles(const CsrView<T> &M, const Gathers<T, NV> &g, const Epi &epi, cudaStream_t s) {
    if (M.ntiles <= 0) return;
    tile_kernel<T, A, NV, EXACT, Epi><<<M.ntiles, kTileThreads, 0, s>>>(M, g, epi);
    VK_LAUNCH_CHECK();
}

// Epilogue base: one unused reduction slot, unit gather scale, zero start,
// never skipped.
template <class A>
struct EpiBase {
    static constexpr int NR = 1;
    __device__ A init(int, int) const { return A(0); }
    __device__ A gscale(int) const { return A(1); }
    __device__ bool skip() const { return false; }
    __device__ void finish(double (&)[1], double *, int) const {}
};

// ---- setup (vk_csr.cu) ------------------------------------------------------

// Uploads an int64 CSR pattern, converts it to int32 on the device and builds
// the tile schedule. The pattern must already be validated.
void upload_pattern(int64_t rows, int64_t cols, const int64_t *h_ro, const int64_t *h_ci, CsrPattern32 &out,
                    cudaStream_t s);
// Builds the tile schedule of an int32 pattern already on the device.
void build_tiles(CsrPattern32 &p, cudaStream_t s);
// Transposes `a` on the device by a stable radix sort of the column indices
// (rows ascend within each column). perm[t] = source position of entry t.
void transpose_pattern(const CsrPattern32 &a, CsrPattern32 &at, DevBuf<int> &perm, cudaStream_t s);
// dst[t] = src[perm[t]] (optionally converting the value type).
template <class TD, class TS>
void gather_values(const int *perm, const TS *src, TD *dst, int64_t nnz, cudaStream_t s);
// Expands row offsets to a row index per nonzero.
void expand_rows(const CsrPattern32 &p, int *rowidx, cudaStream_t s);

} // namespace vk
