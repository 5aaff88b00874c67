// Solver shell: model validation, upload, and the post-processing that turns
// final iterates into a SolveResult in original coordinates.
#include "vk_engine.cuh"
#include "vk_stage.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <system_error>
#include <thread>
#include <vector>

namespace vk {

namespace {
thread_local bool t_serial_host_work = false;
} // namespace

bool serial_host_work() { return t_serial_host_work; }
void set_serial_host_work(bool on) { t_serial_host_work = on; }

// ---------------------------------------------------------------------------
// Validation: Model::validate (Model.cpp:118-199) restricted to what a
// vk_problem can express, then the solve_lp / solve_qp gates
// (pdhg.cpp:274-291, pdqp.cpp:313-327). Same rules, same first-error message.
// ---------------------------------------------------------------------------
namespace {

// First failing index of [0, count) in order, or -1. check(b, e, &code)
// returns the first failing index of [b, e) (-1 if none) and its error code.
// When the scan touches at least 2^20 elements (`work`) the range is split
// over host threads; the failure of the lowest range wins, so the result is
// the sequential scan's.
template <class F>
int64_t first_failure(int64_t count, int64_t work, F check, int &code) {
    constexpr int64_t kSerial = int64_t(1) << 20;
    const unsigned hw = std::thread::hardware_concurrency();
    const int T = work < kSerial || count < 2 || serial_host_work()
                      ? 1
                      : static_cast<int>(std::min<unsigned>(hw == 0 ? 1 : hw, 16));
    if (T <= 1) return check(0, count, code);
    std::vector<int64_t> at(T, -1);
    std::vector<int> codes(T, 0);
    std::vector<std::thread> pool;
    pool.reserve(T - 1);
    auto part = [&](int t) {
        const int64_t b = count * t / T, e = count * (t + 1) / T;
        at[t] = check(b, e, codes[t]);
    };
    int started = 1;
    try {
        for (; started < T; ++started) pool.emplace_back(part, started);
    } catch (const std::system_error &) {
        // no more threads to be had: the parts not started run here
    }
    for (int t = started; t < T; ++t) part(t);
    part(0);
    for (auto &th : pool) th.join();
    for (int t = 0; t < T; ++t)
        if (at[t] >= 0) {
            code = codes[t];
            return at[t];
        }
    return -1;
}

std::string check_pattern(const vk_csr &a, const char *name) {
    const std::string nm(name);
    if (a.rows < 0 || a.cols < 0) return nm + " dimensions must be non-negative";
    if (a.rows > 0 && !a.row_offsets) return nm + " row_offsets must contain rows + 1 entries";
    const int64_t *ro = a.row_offsets;
    if (!ro) return "";
    if (ro[0] != 0) return nm + " row_offsets do not describe column_indices";
    const int64_t nnz = ro[a.rows];
    if (nnz < 0) return nm + " row_offsets must be ordered and in range";
    enum { kRange = 1, kColumn = 2, kOrder = 3 };
    auto rows = [&](int64_t r0, int64_t r1, int &code) -> int64_t {
        for (int64_t r = r0; r < r1; ++r) {
            const int64_t b = ro[r], e = ro[r + 1];
            if (b < 0 || b > e || e > nnz) {
                code = kRange;
                return r;
            }
            int64_t prev = -1;
            for (int64_t k = b; k < e; ++k) {
                const int64_t c = a.col_indices[k];
                if (c < 0 || c >= a.cols) {
                    code = kColumn;
                    return r;
                }
                if (c <= prev) {
                    code = kOrder;
                    return r;
                }
                prev = c;
            }
        }
        return -1;
    };
    // rows are split evenly; a thread's rows can hold many more nonzeros than
    // another's only for very skewed patterns, which then just run longer
    int code = 0;
    if (first_failure(a.rows, a.rows + nnz, rows, code) < 0) return "";
    return code == kRange    ? nm + " row_offsets must be ordered and in range"
           : code == kColumn ? nm + " contains an out-of-range column"
                             : nm + " columns must be strictly ordered per row";
}

int64_t nnz_of(const vk_csr &a) { return (a.rows >= 0 && a.row_offsets) ? a.row_offsets[a.rows] : 0; }

std::string check_matrix(const vk_csr &a, const char *name) {
    std::string e = check_pattern(a, name);
    if (!e.empty()) return e;
    auto finite = [&](int64_t b, int64_t e2, int &) -> int64_t {
        for (int64_t k = b; k < e2; ++k)
            if (!std::isfinite(a.values[k])) return k;
        return -1;
    };
    int code = 0;
    const int64_t nnz = nnz_of(a);
    if (first_failure(nnz, nnz, finite, code) >= 0) return std::string(name) + " coefficients must be finite";
    return "";
}

// Dense PSD test of continuous_common.hpp:242-275 (Cholesky with a 1e-10
// tolerance), used where n is small enough for a dense n x n copy.
bool dense_psd(const vk_csr &q) {
    const size_t n = static_cast<size_t>(q.rows);
    std::vector<double> a(n * n, 0.0);
    for (int64_t r = 0; r < q.rows; ++r)
        for (int64_t k = q.row_offsets[r]; k < q.row_offsets[r + 1]; ++k)
            a[static_cast<size_t>(r) * n + static_cast<size_t>(q.col_indices[k])] = q.values[k];
    const double tol = 1e-10;
    for (size_t k = 0; k < n; ++k) {
        double pivot = a[k * n + k];
        for (size_t j = 0; j < k; ++j) pivot -= a[k * n + j] * a[k * n + j];
        if (pivot < -tol * std::max(1.0, std::abs(a[k * n + k]))) return false;
        if (pivot <= tol) {
            for (size_t i = k + 1; i < n; ++i) {
                if (std::abs(a[i * n + k]) > tol) return false;
                a[i * n + k] = 0.0;
            }
            continue;
        }
        const double d = std::sqrt(pivot);
        a[k * n + k] = d;
        for (size_t i = k + 1; i < n; ++i) {
            double v = a[i * n + k];
            for (size_t j = 0; j < k; ++j) v -= a[i * n + j] * a[k * n + j];
            a[i * n + k] = v / d;
        }
    }
    return true;
}

} // namespace

// Largest n for which the dense PSD test runs (O(n^3) host work).
constexpr int64_t kDensePsdMax = 1500;
bool psd_check_large(const vk_csr &q); // vk_psd.cu

std::string validate_problem(const vk_problem &p, const vk_options &o, bool &unsupported) {
    unsupported = false;
    const int64_t m = p.A.rows, n = p.A.cols;
    if (m < 0 || n < 0) return "constraint matrix dimensions must be non-negative";
    if (!std::isfinite(p.objective_offset)) return "objective coefficients must be finite";
    for (int64_t j = 0; j < n; ++j)
        if (!std::isfinite(p.c[j])) return "objective coefficients must be finite";
    for (int64_t i = 0; i < m; ++i) {
        const double lo = p.row_lower[i], hi = p.row_upper[i];
        if (std::isnan(lo) || std::isnan(hi) || lo > hi)
            return "constraint bounds contains an invalid bound at index " + std::to_string(i);
    }
    for (int64_t j = 0; j < n; ++j) {
        const double lo = p.var_lower[j], hi = p.var_upper[j];
        if (std::isnan(lo) || std::isnan(hi) || lo > hi)
            return "variable bounds contains an invalid bound at index " + std::to_string(j);
    }
    std::string e = check_matrix(p.A, "constraint matrix");
    if (!e.empty()) return e;
    const vk_csr &q = p.Q;
    const bool q_absent = q.rows == 0 && q.cols == 0 && nnz_of(q) == 0;
    if (!q_absent) {
        e = check_matrix(q, "quadratic objective");
        if (!e.empty()) return e;
        if (q.rows != n || q.cols != n) return "quadratic objective must be square and match the variables";
        // symmetry (Model.cpp:157-180), each entry against its mirror
        for (int64_t r = 0; r < n; ++r) {
            for (int64_t k = q.row_offsets[r]; k < q.row_offsets[r + 1]; ++k) {
                const int64_t c = q.col_indices[k];
                const int64_t *b = q.col_indices + q.row_offsets[c];
                const int64_t *en = q.col_indices + q.row_offsets[c + 1];
                const int64_t *it = std::lower_bound(b, en, r);
                const double v = q.values[k];
                if (it == en || *it != r) return "quadratic objective must be stored symmetrically";
                const double w = q.values[it - q.col_indices];
                if (std::abs(v - w) > 1e-12 * std::max({1.0, std::abs(v), std::abs(w)}))
                    return "quadratic objective must be stored symmetrically";
            }
        }
    }
    const bool qp = nnz_of(q) > 0;
    if (n == 0) return qp ? "QP requires at least one variable" : "LP requires at least one variable";
    if (qp) {
        const bool psd = n <= kDensePsdMax ? dense_psd(q) : psd_check_large(q);
        if (!psd) {
            unsupported = true;
            return "QP objective matrix is not positive semidefinite";
        }
    }
    const bool opts_ok = o.iteration_limit >= 0 && std::isfinite(o.primal_tolerance) &&
                         std::isfinite(o.dual_tolerance) && o.primal_tolerance >= 0.0 && o.dual_tolerance >= 0.0 &&
                         (!std::isfinite(o.time_limit_seconds) || o.time_limit_seconds >= 0.0);
    if (!opts_ok) return "solver limits and tolerances must be non-negative";
    if (o.continuous_method != 0 && o.continuous_method != 1) {
        unsupported = true;
        return qp ? "requested continuous method is not implemented for QP"
                  : "requested continuous method is not implemented for LP";
    }
    if (m >= (int64_t(1) << 31) || n >= (int64_t(1) << 31) || nnz_of(p.A) >= (int64_t(1) << 31) ||
        nnz_of(q) >= (int64_t(1) << 31)) {
        unsupported = true;
        return "model exceeds the int32 index range of the device structures";
    }
    if (o.algorithm != VK_ALGO_REFERENCE && o.algorithm != VK_ALGO_HALPERN) return "unknown algorithm";
    if (o.precision != VK_PREC_FP64 && o.precision != VK_PREC_MIXED) return "unknown precision";
    return "";
}

void ensure_tuned(DeviceModel &dm, cudaStream_t s) {
    if (dm.tuned) return;
    autotune_pattern<double>(dm.a, dm.a_val.get(), s);
    autotune_pattern<double>(dm.at, dm.at_val.get(), s);
    if (dm.qp) autotune_pattern<double>(dm.q, dm.q_val.get(), s);
    dm.tuned = true;
}

std::unique_ptr<DeviceModel> upload_model(const vk_problem &p, cudaStream_t s, int verbose, bool reorder) {
    PhaseLog log(verbose, "upload", s);
    auto dm = std::make_unique<DeviceModel>();
    const int64_t m = p.A.rows, n = p.A.cols;
    dm->m = static_cast<int>(m);
    dm->n = static_cast<int>(n);
    dm->nnz = nnz_of(p.A);
    dm->q_nnz = nnz_of(p.Q);
    dm->qp = dm->q_nnz > 0;
    dm->offset = p.objective_offset;
    static const int64_t zero = 0;
    upload_pattern(m, n, m > 0 ? p.A.row_offsets : &zero, p.A.col_indices, dm->a, s);
    log.mark("pattern (int64 -> int32) + tiles");
    if (reorder && !dm->qp && order_columns_by_count(dm->a, column_order_mode(), dm->cperm, s))
        log.mark("column order (by nonzero count)");
    dm->a_val.reset(padded(dm->nnz));
    stage_h2d(dm->a_val.get(), p.A.values, dm->nnz * sizeof(double), s);
    log.mark("values");
    transpose_pattern(dm->a, dm->at, dm->perm, s);
    dm->at_val.reset(padded(dm->nnz));
    gather_values<double, double>(dm->perm.get(), dm->a_val.get(), dm->at_val.get(), dm->nnz, s);
    log.mark("transpose");
    if (dm->qp) {
        upload_pattern(n, n, p.Q.row_offsets, p.Q.col_indices, dm->q, s);
        dm->q_val.reset(padded(dm->q_nnz));
        stage_h2d(dm->q_val.get(), p.Q.values, dm->q_nnz * sizeof(double), s);
        dm->h_qro.assign(p.Q.row_offsets, p.Q.row_offsets + n + 1);
        dm->h_qci.assign(p.Q.col_indices, p.Q.col_indices + dm->q_nnz);
        dm->h_qv.assign(p.Q.values, p.Q.values + dm->q_nnz);
    }
    auto up = [&](DevBuf<double> &b, const double *h, int64_t k) {
        b.reset(k > 0 ? k : 1);
        if (k > 0) stage_h2d(b.get(), h, k * sizeof(double), s);
    };
    // column vectors into the device's column order (the caller's order lands
    // in `orig`, kept until the stream synchronises below)
    DevBuf<double> orig[3];
    int used = 0;
    auto upcol = [&](DevBuf<double> &b, const double *h) {
        if (!dm->reordered()) return up(b, h, n);
        up(orig[used], h, n);
        b.reset(n);
        gather_values<double, double>(dm->cperm.get(), orig[used].get(), b.get(), n, s);
        ++used;
    };
    upcol(dm->c, p.c);
    upcol(dm->vl, p.var_lower);
    upcol(dm->vu, p.var_upper);
    up(dm->rl, p.row_lower, m);
    up(dm->ru, p.row_upper, m);
    dm->h_c.assign(p.c, p.c + n);
    dm->h_vl.assign(p.var_lower, p.var_lower + n);
    dm->h_vu.assign(p.var_upper, p.var_upper + n);
    VK_CUDA(cudaStreamSynchronize(s));
    return dm;
}

// ---------------------------------------------------------------------------
// Deterministic partial-sum reduction (fixed assignment and tree).
// ---------------------------------------------------------------------------
namespace {
__global__ void reduce_partials_kernel(const double *__restrict__ p, int ntiles, int R, double *__restrict__ out) {
    __shared__ double scratch[32];
    for (int r = 0; r < R; ++r) {
        double v = 0.0;
        for (int t = threadIdx.x; t < ntiles; t += blockDim.x) v += p[(size_t)t * R + r];
        double a[1] = {v};
        block_sum<1>(a, scratch);
        if (threadIdx.x == 0) out[r] = a[0];
        __syncthreads();
    }
}
} // namespace

void reduce_partials(const double *partials, int ntiles, int R, double *out, cudaStream_t s) {
    reduce_partials_kernel<<<1, 1024, 0, s>>>(partials, ntiles, R, out);
    VK_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Post-processing in original coordinates (pdhg.cpp:153-264,
// pdqp.cpp:180-297), plus the relative KKT sums.
//   row pass over A (original values), gathering x:
//     row values, row box violation, row duals, row complementarity,
//     sum (Ax - clamp(Ax))^2, sum b_i^2, row terms of the dual objective,
//     sum of squared row-dual sign violations
//   column pass over A' (original values), gathering y, started at c (+Qx):
//     stationarity s = c + Qx + A'y (the reference's accumulation order),
//     its projected-gradient residual, variable duals within active_tol,
//     variable complementarity and box violation, sum (x - clamp x)^2,
//     sum c^2, dual residual sum, column dual-objective terms, c'x, x'Qx
// ---------------------------------------------------------------------------
namespace {

constexpr int kPostRowSums = 4; // rp2, b2, dobj_rows, viol2
constexpr int kPostColSums = 6; // box2, c2, rd2, dobj_cols, pobj, quad

struct PostRowEpi : EpiRow<double, PostRowEpi> {
    static constexpr int NR = 6; // [0] pr max [1] comp max, then sums
    const double *rl, *ru, *yo;
    double *ld, *ud;
    PostOut *out;
    double *partials;
    __device__ void row(int i, const double (&s)[1], double (&red)[6]) const {
        const double v = s[0], lo = rl[i], hi = ru[i], y = yo[i];
        const bool flo = isfinite(lo), fhi = isfinite(hi);
        if (flo) red[0] = smax(red[0], lo - v);
        if (fhi) red[0] = smax(red[0], v - hi);
        const double l = smax(0.0, -y), u = smax(0.0, y);
        if (ld) ld[i] = l;
        if (ud) ud[i] = u;
        if (flo) red[1] = smax(red[1], fabs((v - lo) * l));
        if (fhi) red[1] = smax(red[1], fabs((hi - v) * u));
        const double d = v - clampbox(v, lo, hi);
        red[2] += d * d;
        double b = 0.0;
        if (flo) b = smax(b, fabs(lo));
        if (fhi) b = smax(b, fabs(hi));
        red[3] += b * b;
        if (l > 0.0) {
            if (flo) red[4] += lo * l; else red[5] += l * l;
        }
        if (u > 0.0) {
            if (fhi) red[4] -= hi * u; else red[5] += u * u;
        }
    }
    __device__ void finish(double (&red)[6], double *scratch, int tile) const {
        const double a = block_max_nonneg(red[0], scratch);
        __syncthreads();
        const double b = block_max_nonneg(red[1], scratch);
        if (threadIdx.x == 0) {
            atomic_max_nonneg(&out->primal_res, a);
            atomic_max_nonneg(&out->comp_res, b);
        }
        __syncthreads();
        double sums[kPostRowSums] = {red[2], red[3], red[4], red[5]};
        block_sum<kPostRowSums>(sums, scratch);
        if (threadIdx.x == 0)
            for (int r = 0; r < kPostRowSums; ++r) partials[(size_t)tile * kPostRowSums + r] = sums[r];
    }
};

struct PostColEpi : EpiRow<double, PostColEpi> {
    static constexpr int NR = 10; // [0] stat max [1] comp max [2] box max [3] nonfinite, then sums
    const double *xo, *lo, *hi, *c, *qc;
    double atol;
    double *vld, *vud;
    PostOut *out;
    double *partials;
    __device__ double init_value(int j) const { return qc ? qc[j] : c[j]; }
    __device__ double gs() const { return 1.0; }
    __device__ void row(int j, const double (&s)[1], double (&red)[10]) const {
        const double st = s[0], x = xo[j], l = lo[j], u = hi[j];
        const bool fl = isfinite(l), fu = isfinite(u);
        // std::clamp(x - st, l, u) (pdhg.cpp:206-208)
        const double t = x - st;
        const double proj = (t < l) ? l : ((u < t) ? u : t);
        red[0] = smax(red[0], fabs(x - proj));
        double dl = 0.0, du = 0.0;
        if (fl && x - l <= atol) {
            dl = smax(0.0, st);
            red[1] = smax(red[1], fabs((x - l) * dl));
        }
        if (fu && u - x <= atol) {
            du = smax(0.0, -st);
            red[1] = smax(red[1], fabs((u - x) * du));
        }
        if (vld) vld[j] = dl;
        if (vud) vud[j] = du;
        if (fl) red[2] = smax(red[2], l - x);
        if (fu) red[2] = smax(red[2], x - u);
        if (!isfinite(x)) red[3] = 1.0;
        const double bx = x - clampbox(x, l, u);
        red[4] += bx * bx;
        red[5] += c[j] * c[j];
        const double pl = smax(0.0, st), pu = smax(0.0, -st);
        if (pl > 0.0) {
            if (fl) red[7] += l * pl; else red[6] += pl * pl;
        }
        if (pu > 0.0) {
            if (fu) red[7] -= u * pu; else red[6] += pu * pu;
        }
        red[8] += c[j] * x;
        if (qc) red[9] += x * (qc[j] - c[j]);
    }
    __device__ void finish(double (&red)[10], double *scratch, int tile) const {
        double mx[4];
        for (int r = 0; r < 4; ++r) {
            mx[r] = block_max_nonneg(red[r], scratch);
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            atomic_max_nonneg(&out->stat_res, mx[0]);
            atomic_max_nonneg(&out->comp_res, mx[1]);
            atomic_max_nonneg(&out->primal_res, mx[2]);
            if (mx[3] > 0.0) atomic_max_nonneg(&out->sums[11], 1.0);
        }
        double sums[kPostColSums] = {red[4], red[5], red[6], red[7], red[8], red[9]};
        block_sum<kPostColSums>(sums, scratch);
        if (threadIdx.x == 0)
            for (int r = 0; r < kPostColSums; ++r) partials[(size_t)tile * kPostColSums + r] = sums[r];
    }
};

// Column pass epilogue wrapper that starts every row at c_j or (c + Qx)_j.
struct PostColEpiInit : PostColEpi {
    __device__ double init(int j, int) const { return init_value(j); }
};

struct QcEpi : EpiRow<double, QcEpi> {
    const double *c;
    double *out;
    __device__ double init(int j, int) const { return c[j]; }
    __device__ void row(int j, const double (&s)[1], double (&)[1]) const { out[j] = s[0]; }
};

} // namespace

// ---------------------------------------------------------------------------
// Solver
// ---------------------------------------------------------------------------
Solver::Solver(const vk_problem &p, const vk_options &o) : opts_(o) {
    VK_CUDA(cudaSetDevice(o.device));
    device_error_flag(); // allocated here, never inside a graph capture
    VK_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    PhaseLog log(o.verbose, "create", stream_);
    dm_ = upload_model(p, stream_, o.verbose, o.spmv_order == VK_SPMV_FAST);
    log.mark("upload + transpose");
    // the Halpern passes (and the reference scheme's Q pass) run on the
    // patterns' tuned variants; the reference scheme tunes its fused passes itself
    if (o.algorithm == VK_ALGO_HALPERN || dm_->qp) {
        ensure_tuned(*dm_, stream_);
        log.mark("pattern autotune");
    }
    engine_ = o.algorithm == VK_ALGO_HALPERN ? make_halpern_engine(*dm_, o, stream_)
                                             : make_reference_engine(*dm_, o, stream_);
    log.mark("engine setup");
}

std::string Solver::set_options(const vk_options &o) {
    if (o.continuous_method != opts_.continuous_method || o.algorithm != opts_.algorithm ||
        o.precision != opts_.precision || o.spmv_order != opts_.spmv_order || o.check_every != opts_.check_every ||
        o.device != opts_.device)
        return "only limits and tolerances can change after vk_pdhg_create";
    const bool ok = o.iteration_limit >= 0 && std::isfinite(o.primal_tolerance) && std::isfinite(o.dual_tolerance) &&
                    o.primal_tolerance >= 0.0 && o.dual_tolerance >= 0.0 && !std::isnan(o.relative_tolerance) &&
                    o.relative_tolerance >= 0.0 &&
                    (!std::isfinite(o.time_limit_seconds) || o.time_limit_seconds >= 0.0);
    if (!ok) return "solver limits and tolerances must be non-negative";
    opts_ = o;
    engine_->set_limits(o);
    return "";
}

bool Solver::profile(long long iterations, vk_pass_profile *out) {
    VK_CUDA(cudaSetDevice(opts_.device));
    PassProfile pp;
    if (!engine_->profile(iterations, pp)) return false;
    *out = vk_pass_profile{};
    out->count = pp.count;
    for (int q = 0; q < pp.count && q < 8; ++q) {
        std::snprintf(out->name[q], sizeof(out->name[q]), "%s", pp.name[q] ? pp.name[q] : "");
        out->launches[q] = pp.launches[q];
        out->ms_per_launch[q] = pp.launches[q] ? pp.ms[q] / static_cast<double>(pp.launches[q]) : 0.0;
        out->bytes_per_launch[q] = pp.bytes[q];
    }
    return true;
}

Solver::~Solver() {
    engine_.reset();
    dm_.reset();
    if (stream_) cudaStreamDestroy(stream_);
}

namespace {
// out[j] = the override of device column j (the caller's column perm[j], or
// j without a column order), else the model's bound
__global__ void fill_override_kernel(const double *__restrict__ ov, const double *__restrict__ model,
                                     const int *__restrict__ perm, int n, double *__restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) out[j] = ov ? ov[perm ? perm[j] : j] : model[j];
}
} // namespace

void Solver::solve(const double *warm, const double *lo_ovr, const double *hi_ovr, vk_result *r) {
    const auto started = std::chrono::steady_clock::now();
    VK_CUDA(cudaSetDevice(opts_.device));
    const DeviceModel &dm = *dm_;
    const int m = dm.m, n = dm.n;
    const char *name = dm.qp ? "PDQP" : "PDHG";
    r->status = VK_STATUS_NOT_SOLVED;
    r->message[0] = '\0';
    r->iterations = 0;
    r->restarts = 0;
    r->fp32_iterations = 0;
    auto fail = [&](const char *msg) {
        r->status = VK_STATUS_INVALID_MODEL;
        std::snprintf(r->message, sizeof(r->message), "%s", msg);
    };
    // copy_bounds (continuous_common.hpp:80-110)
    for (const double *ov : {lo_ovr, hi_ovr}) {
        if (!ov) continue;
        for (int j = 0; j < n; ++j)
            if (std::isnan(ov[j])) return fail("variable bound overrides must be empty or sized and non-NaN");
    }
    for (int j = 0; j < n; ++j) {
        const double l = lo_ovr ? lo_ovr[j] : dm.h_vl[j];
        const double u = hi_ovr ? hi_ovr[j] : dm.h_vu[j];
        if (std::isnan(l) || std::isnan(u) || l > u) return fail("variable bound overrides contain an invalid interval");
    }
    // warm start (pdhg.cpp:29-33)
    if (warm)
        for (int j = 0; j < n; ++j)
            if (!std::isfinite(warm[j])) return fail("warm start must be empty or finite and sized to the model");

    cudaStream_t s = stream_;
    DevBuf<double> lo(n), hi(n), dwarm(warm ? n : 0), ov_lo(lo_ovr ? n : 0), ov_hi(hi_ovr ? n : 0);
    if (lo_ovr) VK_CUDA(cudaMemcpyAsync(ov_lo.get(), lo_ovr, n * sizeof(double), cudaMemcpyHostToDevice, s));
    if (hi_ovr) VK_CUDA(cudaMemcpyAsync(ov_hi.get(), hi_ovr, n * sizeof(double), cudaMemcpyHostToDevice, s));
    if (warm) VK_CUDA(cudaMemcpyAsync(dwarm.get(), warm, n * sizeof(double), cudaMemcpyHostToDevice, s));
    const int *cperm = dm.reordered() ? dm.cperm.get() : nullptr;
    fill_override_kernel<<<grid1d(n), 256, 0, s>>>(lo_ovr ? ov_lo.get() : nullptr, dm.vl.get(), cperm, n, lo.get());
    fill_override_kernel<<<grid1d(n), 256, 0, s>>>(hi_ovr ? ov_hi.get() : nullptr, dm.vu.get(), cperm, n, hi.get());
    VK_LAUNCH_CHECK();
    DevBuf<double> dwarm_dev(warm && cperm ? n : 0); // the warm start in the device's column order
    if (warm && cperm) gather_values<double, double>(cperm, dwarm.get(), dwarm_dev.get(), n, s);
    const double *warm_dev = !warm ? nullptr : cperm ? dwarm_dev.get() : dwarm.get();

    DevBuf<double> xo(n), yo(m > 0 ? m : 1);
    RunInfo info;
    PhaseLog log(opts_.verbose, "solve", s);
    log.mark("checks + overrides");
    engine_->run(warm_dev, lo.get(), hi.get(), xo.get(), yo.get(), info, started);
    log.mark("iterations");

    // post-processing
    const bool exact = opts_.spmv_order == VK_SPMV_SEQUENTIAL;
    DevBuf<PostOut> post(1);
    VK_CUDA(cudaMemsetAsync(post.get(), 0, sizeof(PostOut), s));
    DevBuf<double> ld(r->row_lower_dual && m ? m : 0), ud(r->row_upper_dual && m ? m : 0);
    DevBuf<double> vld(r->var_lower_dual ? n : 0), vud(r->var_upper_dual ? n : 0);
    DevBuf<double> prow(static_cast<size_t>(kMaxGrid) * kPostRowSums);
    DevBuf<double> pcol(static_cast<size_t>(kMaxGrid) * kPostColSums);
    DevBuf<double> sums(kPostRowSums + kPostColSums);
    VK_CUDA(cudaMemsetAsync(sums.get(), 0, sums.bytes(), s));
    if (m > 0) {
        PostRowEpi e;
        e.rl = dm.rl.get();
        e.ru = dm.ru.get();
        e.yo = yo.get();
        e.ld = ld.get();
        e.ud = ud.get();
        e.out = post.get();
        e.partials = prow.get();
        const int grid =
            exact ? launch_tiles<double, double, 1, true>(view(dm.a, dm.a_val.get()), Gathers<double, 1>{{xo.get()}}, e, s)
                  : launch_tiles<double, double, 1, false>(view(dm.a, dm.a_val.get()), Gathers<double, 1>{{xo.get()}}, e, s);
        reduce_partials(prow.get(), grid, kPostRowSums, sums.get(), s);
    }
    DevBuf<double> qc(dm.qp ? n : 0);
    if (dm.qp) {
        QcEpi q;
        q.c = dm.c.get();
        q.out = qc.get();
        if (exact)
            launch_tiles<double, double, 1, true>(view(dm.q, dm.q_val.get()), Gathers<double, 1>{{xo.get()}}, q, s);
        else
            launch_tiles<double, double, 1, false>(view(dm.q, dm.q_val.get()), Gathers<double, 1>{{xo.get()}}, q, s);
    }
    {
        PostColEpiInit e;
        e.xo = xo.get();
        e.lo = lo.get();
        e.hi = hi.get();
        e.c = dm.c.get();
        e.qc = dm.qp ? qc.get() : nullptr;
        e.atol = std::max(10.0 * opts_.primal_tolerance, 1e-8);
        e.vld = vld.get();
        e.vud = vud.get();
        e.out = post.get();
        e.partials = pcol.get();
        const double *ygather = m > 0 ? yo.get() : xo.get(); // never read when A has no entries
        const int grid =
            exact ? launch_tiles<double, double, 1, true>(view(dm.at, dm.at_val.get()), Gathers<double, 1>{{ygather}}, e, s)
                  : launch_tiles<double, double, 1, false>(view(dm.at, dm.at_val.get()), Gathers<double, 1>{{ygather}}, e, s);
        reduce_partials(pcol.get(), grid, kPostColSums, sums.get() + kPostRowSums, s);
    }
    PostOut hp;
    double hs[kPostRowSums + kPostColSums];
    VK_CUDA(cudaMemcpyAsync(&hp, post.get(), sizeof(hp), cudaMemcpyDeviceToHost, s));
    VK_CUDA(cudaMemcpyAsync(hs, sums.get(), sizeof(hs), cudaMemcpyDeviceToHost, s));
    // column-indexed results back into the caller's column order
    DevBuf<double> back(cperm ? 3 * static_cast<size_t>(n) : 0);
    const double *x_out = xo.get(), *vld_out = vld.get(), *vud_out = vud.get();
    if (cperm) {
        scatter_values(cperm, xo.get(), back.get(), n, s);
        x_out = back.get();
        if (r->var_lower_dual) {
            scatter_values(cperm, vld.get(), back.get() + n, n, s);
            vld_out = back.get() + n;
        }
        if (r->var_upper_dual) {
            scatter_values(cperm, vud.get(), back.get() + 2 * static_cast<size_t>(n), n, s);
            vud_out = back.get() + 2 * static_cast<size_t>(n);
        }
    }
    std::vector<double> hx(n);
    stage_d2h(hx.data(), x_out, n * sizeof(double), s);
    if (r->y && m > 0) stage_d2h(r->y, yo.get(), m * sizeof(double), s);
    if (r->row_lower_dual && m > 0) stage_d2h(r->row_lower_dual, ld.get(), m * sizeof(double), s);
    if (r->row_upper_dual && m > 0) stage_d2h(r->row_upper_dual, ud.get(), m * sizeof(double), s);
    if (r->var_lower_dual) stage_d2h(r->var_lower_dual, vld_out, n * sizeof(double), s);
    if (r->var_upper_dual) stage_d2h(r->var_upper_dual, vud_out, n * sizeof(double), s);
    VK_CUDA(cudaStreamSynchronize(s));
    if (r->x) std::memcpy(r->x, hx.data(), n * sizeof(double));

    // objective: offset + c'x (+ 0.5 x'Qx), the reference's order (continuous_common.hpp:284-300)
    double dot = 0.0;
    for (int j = 0; j < n; ++j) dot += dm.h_c[j] * hx[j];
    double obj = dm.offset + dot;
    if (dm.qp) {
        double quad = 0.0;
        for (int rr = 0; rr < n; ++rr)
            for (int64_t k = dm.h_qro[rr]; k < dm.h_qro[rr + 1]; ++k) quad += hx[rr] * dm.h_qv[k] * hx[dm.h_qci[k]];
        obj += 0.5 * quad;
    }
    r->objective = obj;
    r->primal_residual = hp.primal_res;
    r->stationarity_residual = hp.stat_res;
    r->complementarity_residual = hp.comp_res;
    // relative KKT
    const double rp2 = hs[0], b2 = hs[1], dobj_r = hs[2], viol2 = hs[3];
    const double box2 = hs[4], c2 = hs[5], rd2 = hs[6], dobj_c = hs[7], pobj = hs[8], quad = hs[9];
    const double pk = pobj + 0.5 * quad + dm.offset;
    const double dk = dobj_r + dobj_c - 0.5 * quad + dm.offset;
    r->rel_primal = (std::sqrt(rp2) + std::sqrt(box2)) / (1.0 + std::sqrt(b2));
    r->rel_dual = std::sqrt(rd2 + viol2) / (1.0 + std::sqrt(c2));
    r->rel_gap = std::abs(pk - dk) / (1.0 + std::abs(pk) + std::abs(dk));

    r->iterations = info.iterations;
    r->restarts = info.restarts;
    r->last_metric = info.last_metric;
    r->iterate_seconds = info.iterate_seconds;
    r->fp32_iterations = info.fp32_iterations;
    r->kernel_launches = info.kernel_launches;
    int status = info.status;
    if (!std::isfinite(obj)) {
        status = VK_STATUS_NUMERICAL_FAILURE;
        std::snprintf(r->message, sizeof(r->message), "%s produced a non-finite objective", name);
    }
    if (status == VK_STATUS_NOT_SOLVED) status = VK_STATUS_ITERATION_LIMIT;
    const bool nonfinite_x = hp.sums[11] > 0.0;
    if (nonfinite_x) {
        status = VK_STATUS_NUMERICAL_FAILURE;
        std::snprintf(r->message, sizeof(r->message), "%s produced a non-finite iterate", name);
    } else if (status == VK_STATUS_OPTIMAL && opts_.algorithm == VK_ALGO_REFERENCE &&
               (r->primal_residual > opts_.primal_tolerance || r->stationarity_residual > opts_.dual_tolerance)) {
        status = VK_STATUS_NUMERICAL_FAILURE;
        std::snprintf(r->message, sizeof(r->message),
                      "%s stopped without satisfying original-coordinate residual checks", name);
    }
    r->status = status;
    r->solve_seconds = seconds_since(started);
    log.mark("post-processing + results");
}

} // namespace vk
