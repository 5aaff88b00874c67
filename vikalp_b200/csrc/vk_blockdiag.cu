#include "vk_blockdiag.cuh"
#include "vk_stage.cuh"

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

namespace vk {

namespace {

// Instance b's rows, columns and nonzeros at its offsets in the concatenation.
void fill_instance(const vk_problem &p, int b, BlockDiag &out) {
    const int r0 = out.row_off[b], c0 = out.col_off[b];
    const int64_t k0 = out.nnz_off[b];
    for (int64_t i = 0; i < p.A.rows; ++i) {
        out.ro[r0 + i + 1] = k0 + p.A.row_offsets[i + 1];
        out.rinst[r0 + i] = b;
        out.rl[r0 + i] = p.row_lower[i];
        out.ru[r0 + i] = p.row_upper[i];
    }
    const int64_t nz = out.nnz_off[b + 1] - k0;
    for (int64_t k = 0; k < nz; ++k) {
        out.ci[k0 + k] = c0 + p.A.col_indices[k];
        out.v[k0 + k] = p.A.values[k];
    }
    for (int64_t j = 0; j < p.A.cols; ++j) {
        out.c[c0 + j] = p.c[j];
        out.vl[c0 + j] = p.var_lower[j];
        out.vu[c0 + j] = p.var_upper[j];
        out.cinst[c0 + j] = b;
    }
    out.offset[b] = p.objective_offset;
}

} // namespace

void concat_instances(const vk_problem *probs, int count, BlockDiag &out) {
    out.count = count;
    out.row_off.assign(count + 1, 0);
    out.col_off.assign(count + 1, 0);
    out.nnz_off.assign(count + 1, 0);
    for (int b = 0; b < count; ++b) {
        const vk_problem &p = probs[b];
        out.row_off[b + 1] = out.row_off[b] + static_cast<int>(p.A.rows);
        out.col_off[b + 1] = out.col_off[b] + static_cast<int>(p.A.cols);
        out.nnz_off[b + 1] = out.nnz_off[b] + (p.A.rows > 0 ? p.A.row_offsets[p.A.rows] : 0);
    }
    const int m = out.row_off[count], n = out.col_off[count];
    const int64_t nnz = out.nnz_off[count];
    out.m = m;
    out.n = n;
    out.nnz = nnz;
    out.ro.assign(m + 1, 0);
    out.ci.resize(nnz);
    out.v.resize(nnz);
    out.c.resize(n);
    out.vl.resize(n);
    out.vu.resize(n);
    out.rl.resize(m);
    out.ru.resize(m);
    out.offset.resize(count);
    out.rinst.resize(m);
    out.cinst.resize(n);
    // instances write disjoint ranges: large batches fill them over host threads
    std::atomic<int> next{0};
    auto fill = [&] {
        for (int b = next++; b < count; b = next++) fill_instance(probs[b], b, out);
    };
    const unsigned hw = std::thread::hardware_concurrency();
    const int T = nnz < (int64_t(1) << 20) || count < 2 ? 1 : std::min<int>({count, 16, static_cast<int>(hw == 0 ? 1 : hw)});
    std::vector<std::thread> pool;
    for (int t = 1; t < T; ++t) pool.emplace_back(fill);
    fill();
    for (std::thread &th : pool) th.join();
}

namespace {

template <class V>
void upload(DevBuf<V> &d, const std::vector<V> &h, cudaStream_t s) {
    d.reset(h.empty() ? 1 : h.size());
    if (!h.empty()) VK_CUDA(cudaMemcpyAsync(d.get(), h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice, s));
}

// Instance of every tile (its first row's) and the first tile of every instance.
void tile_instances(const CsrPattern32 &p, const std::vector<int> &inst, int count, DevBuf<int> &tinst,
                    DevBuf<int> &tbeg, cudaStream_t s) {
    std::vector<int> tiles(p.ntiles + 1);
    VK_CUDA(cudaMemcpyAsync(tiles.data(), p.tiles.get(), tiles.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    VK_CUDA(cudaStreamSynchronize(s));
    std::vector<int> ti(std::max(p.ntiles, 1), 0), beg(count + 1, p.ntiles);
    for (int t = p.ntiles - 1; t >= 0; --t) {
        ti[t] = inst[tiles[t]];
        beg[ti[t]] = t;
    }
    // an instance without tiles starts where the next one does
    for (int b = count - 1; b >= 0; --b)
        if (beg[b] > beg[b + 1]) beg[b] = beg[b + 1];
    upload(tinst, ti, s);
    upload(tbeg, beg, s);
}

} // namespace

void upload_block_diag(const BlockDiag &h, DeviceBlockDiag &d, cudaStream_t s, bool autotune) {
    std::vector<unsigned char> rbreak(h.m + 1, 0), cbreak(h.n + 1, 0);
    for (int b = 0; b <= h.count; ++b) {
        rbreak[h.row_off[b]] = 1;
        cbreak[h.col_off[b]] = 1;
    }
    DevBuf<unsigned char> drb, dcb;
    upload(drb, rbreak, s);
    upload(dcb, cbreak, s);
    upload_pattern(h.m, h.n, h.ro.data(), h.ci.data(), d.a, s);
    build_tiles(d.a, s, drb.get());
    d.a_val.reset(padded(h.nnz));
    VK_CUDA(cudaMemsetAsync(d.a_val.get(), 0, padded(h.nnz) * sizeof(double), s));
    stage_h2d(d.a_val.get(), h.v.data(), h.nnz * sizeof(double), s);
    transpose_pattern(d.a, d.at, d.perm, s);
    build_tiles(d.at, s, dcb.get());
    d.at_val.reset(padded(h.nnz));
    VK_CUDA(cudaMemsetAsync(d.at_val.get(), 0, padded(h.nnz) * sizeof(double), s));
    gather_values<double, double>(d.perm.get(), d.a_val.get(), d.at_val.get(), h.nnz, s);
    if (autotune) {
        autotune_pattern<double>(d.a, d.a_val.get(), s);
        autotune_pattern<double>(d.at, d.at_val.get(), s);
    }
    upload(d.rinst, h.rinst, s);
    upload(d.cinst, h.cinst, s);
    tile_instances(d.a, h.rinst, h.count, d.tinst_a, d.tbeg_a, s);
    tile_instances(d.at, h.cinst, h.count, d.tinst_at, d.tbeg_at, s);
    VK_CUDA(cudaStreamSynchronize(s));
}

} // namespace vk
