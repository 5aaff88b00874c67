// Many independent problems laid out as one block-diagonal problem: rows,
// columns and nonzeros concatenated in instance order, with the warp-tiles of
// the sparse passes broken at every instance start (no tile spans two
// instances), so per-tile sums can be reduced per instance in a fixed order and
// the tiles of a finished instance can be skipped.
#pragma once

#include "vk_solver.h"

#include <vector>

namespace vk {

struct BlockDiag {
    int count = 0, m = 0, n = 0;
    int64_t nnz = 0;
    std::vector<int> row_off, col_off;  // [count+1] first row / column of every instance
    std::vector<int> rinst, cinst;      // instance of every row / column
    std::vector<int64_t> nnz_off;       // [count+1]
    std::vector<int64_t> ro, ci;        // concatenated CSR (global column indices)
    std::vector<double> v, c, vl, vu, rl, ru, offset;
};

// Host concatenation of validated problems (their Q is ignored).
void concat_instances(const vk_problem *probs, int count, BlockDiag &out);

struct DeviceBlockDiag {
    CsrPattern32 a, at;              // A and A' with instance-aligned tiles
    DevBuf<int> perm;                // transposed position -> CSR position
    DevBuf<double> a_val, at_val;    // original values, both orders (padded)
    DevBuf<int> rinst, cinst;        // instance of every row / column
    DevBuf<int> tinst_a, tinst_at;   // instance of every tile of A / A'
    DevBuf<int> tbeg_a, tbeg_at;     // [count+1] first tile of every instance
};

// Uploads the block-diagonal matrix and builds both tile schedules;
// `autotune` times the kernel variants on A and A'.
void upload_block_diag(const BlockDiag &h, DeviceBlockDiag &d, cudaStream_t s, bool autotune);

} // namespace vk
