// C-ABI shim over the reference VIKALP CPU path -- TEST / BASELINE INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles this file together with the reference's own
// sources (read in place from the reference tree, never copied) into
// oracle/_ref/libvkref.so. It lets the tests pin the C oracle against the real
// reference and lets bench.py time the reference's CPU implementation.
//
// Entry points:
//   vkref_solve_lp / vkref_solve_qp -> vikalp::solver::solve_lp / solve_qp with
//                                      make_cpu_backend() (continuous.hpp:10-22)
//   vkref_solve                     -> vikalp::solve(Model, SolverOptions) (Solver.hpp:19-21)
//   vkref_multiply                  -> ExecutionBackend::multiply on the CPU backend
//                                      (cpu_ops.cpp:393-460)
//   vkref_pdhg_replay_cuda          -> the same sequence on the reference's CUDA backend
//                                      (cuda/cuda_ops.cu), built into _ref/libvkref_cuda.so
//   vkref_mps_*                     -> vikalp::MpsReader::read (src/io/MpsReader.cpp:10-559),
//                                      the model and errors copied out
//   vkref_pdhg_replay               -> the per-iteration ExecutionBackend call sequence of
//                                      pdhg.cpp:92-130 on already-scaled data, for sizes where
//                                      the reference's own setup cannot finish (its column
//                                      scaling is O(n*nnz), continuous_common.hpp:160-176).
#include "vikalp/backend/CpuBackend.hpp"
#ifdef VKREF_CUDA
#include "vikalp/backend/CudaBackend.hpp"
#endif
#include "vikalp/contracts/ExecutionBackend.hpp"
#include "vikalp/contracts/Model.hpp"
#include "vikalp/contracts/SolveResult.hpp"
#include "vikalp/contracts/SolverOptions.hpp"
#include "vikalp/io/MpsReader.hpp"
#include "vikalp/solver/Solver.hpp"
#include "vikalp/solver/continuous.hpp"

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <limits>
#include <span>
#include <string>
#include <vector>

extern "C" {

typedef struct {
    int64_t m, n;
    const int64_t *ro, *ci;
    const double *v;
    int64_t q_nnz;
    const int64_t *qro, *qci;
    const double *qv;
    const double *c, *rl, *ru;
    double objective_offset;
    const double *l, *u;
} vkref_problem;

typedef struct {
    int64_t iteration_limit;
    double time_limit_seconds;
    double primal_tolerance, dual_tolerance;
    int32_t backend; // BackendPreference
    int32_t method;  // ContinuousMethod
} vkref_options;

typedef struct {
    double *x, *row_lower_dual, *row_upper_dual, *var_lower_dual, *var_upper_dual; // caller-allocated or NULL
    int32_t status;
    int64_t iterations;
    double objective, primal_residual, stationarity_residual, complementarity_residual;
    double dual_bound, solve_seconds;
    char solver[32];
    char backend[32];
    char message[256];
} vkref_result;
}

namespace {

vikalp::Model build_model(const vkref_problem *p) {
    vikalp::Model model;
    model.name = "vkref";
    const auto m = static_cast<std::size_t>(p->m), n = static_cast<std::size_t>(p->n);
    const auto nnz = static_cast<std::size_t>(p->ro[p->m]);
    model.linear_objective.assign(p->c, p->c + n);
    model.objective_offset = p->objective_offset;
    model.variable_lower.assign(p->l, p->l + n);
    model.variable_upper.assign(p->u, p->u + n);
    model.variable_types.assign(n, vikalp::VariableType::Continuous);
    model.constraint_lower.assign(p->rl, p->rl + m);
    model.constraint_upper.assign(p->ru, p->ru + m);
    model.constraint_matrix.pattern.rows = p->m;
    model.constraint_matrix.pattern.columns = p->n;
    model.constraint_matrix.pattern.row_offsets.assign(p->ro, p->ro + m + 1);
    model.constraint_matrix.pattern.column_indices.assign(p->ci, p->ci + nnz);
    model.constraint_matrix.values.assign(p->v, p->v + nnz);
    if (p->q_nnz > 0) {
        model.quadratic_objective.pattern.rows = p->n;
        model.quadratic_objective.pattern.columns = p->n;
        model.quadratic_objective.pattern.row_offsets.assign(p->qro, p->qro + n + 1);
        model.quadratic_objective.pattern.column_indices.assign(p->qci, p->qci + p->q_nnz);
        model.quadratic_objective.values.assign(p->qv, p->qv + p->q_nnz);
    }
    return model;
}

vikalp::SolverOptions build_options(const vkref_options *o) {
    vikalp::SolverOptions opts;
    opts.iteration_limit = o->iteration_limit;
    opts.time_limit_seconds = o->time_limit_seconds;
    opts.primal_tolerance = o->primal_tolerance;
    opts.dual_tolerance = o->dual_tolerance;
    opts.backend = static_cast<vikalp::BackendPreference>(o->backend);
    opts.continuous_method = static_cast<vikalp::ContinuousMethod>(o->method);
    return opts;
}

void copy_out(const std::vector<double> &src, double *dst) {
    if (dst && !src.empty()) std::memcpy(dst, src.data(), src.size() * sizeof(double));
}

void fill_result(const vikalp::SolveResult &r, vkref_result *out) {
    out->status = static_cast<int32_t>(r.status);
    out->iterations = r.iterations;
    out->objective = r.objective_value;
    out->primal_residual = r.primal_residual;
    out->stationarity_residual = r.stationarity_residual;
    out->complementarity_residual = r.complementarity_residual;
    out->dual_bound = r.dual_bound;
    out->solve_seconds = r.solve_seconds;
    copy_out(r.primal_solution, out->x);
    copy_out(r.constraint_lower_dual, out->row_lower_dual);
    copy_out(r.constraint_upper_dual, out->row_upper_dual);
    copy_out(r.variable_lower_dual, out->var_lower_dual);
    copy_out(r.variable_upper_dual, out->var_upper_dual);
    std::snprintf(out->solver, sizeof(out->solver), "%s", r.solver.c_str());
    std::snprintf(out->backend, sizeof(out->backend), "%s", r.backend.c_str());
    std::snprintf(out->message, sizeof(out->message), "%s", r.message.c_str());
}

std::span<const double> opt_span(const double *p, int64_t n) {
    return p ? std::span<const double>(p, static_cast<std::size_t>(n)) : std::span<const double>{};
}

} // namespace

extern "C" {

int vkref_solve_continuous(const vkref_problem *p, const vkref_options *o, const double *warm,
                           const double *lo, const double *hi, int qp, vkref_result *out) {
    try {
        const auto model = build_model(p);
        auto backend = vikalp::make_cpu_backend();
        const auto opts = build_options(o);
        const auto r = qp ? vikalp::solver::solve_qp(model, *backend, opts, opt_span(warm, p->n),
                                                     opt_span(lo, p->n), opt_span(hi, p->n))
                          : vikalp::solver::solve_lp(model, *backend, opts, opt_span(warm, p->n),
                                                     opt_span(lo, p->n), opt_span(hi, p->n));
        fill_result(r, out);
        return 0;
    } catch (const std::exception &e) {
        std::snprintf(out->message, sizeof(out->message), "%s", e.what());
        return -1;
    }
}

int vkref_solve(const vkref_problem *p, const vkref_options *o, vkref_result *out) {
    try {
        const auto model = build_model(p);
        const auto r = vikalp::solve(model, build_options(o));
        fill_result(r, out);
        return 0;
    } catch (const std::exception &e) {
        std::snprintf(out->message, sizeof(out->message), "%s", e.what());
        return -1;
    }
}

// y = alpha * op(A) * x + beta * y on the reference CPU backend. Returns 0, or
// -1 when the backend throws (dimension errors throw std::invalid_argument).
int vkref_multiply(int64_t m, int64_t n, const int64_t *ro, const int64_t *ci, const double *v,
                   double alpha, const double *x, int64_t x_len, double beta, double *y,
                   int64_t y_len, int transpose, char *err, int err_len) {
    try {
        auto be = vikalp::make_cpu_backend();
        vikalp::CsrPattern pat;
        pat.rows = m;
        pat.columns = n;
        pat.row_offsets.assign(ro, ro + m + 1);
        pat.column_indices.assign(ci, ci + ro[m]);
        auto mat = be->create_matrix(pat);
        be->set_values(std::span<const double>(v, static_cast<std::size_t>(ro[m])), *mat);
        auto xv = be->create_vector(x_len);
        auto yv = be->create_vector(y_len);
        be->upload(std::span<const double>(x, static_cast<std::size_t>(x_len)), *xv);
        be->upload(std::span<const double>(y, static_cast<std::size_t>(y_len)), *yv);
        be->multiply(alpha, *mat, *xv, beta, *yv,
                     transpose ? vikalp::Transpose::Yes : vikalp::Transpose::No);
        be->download(*yv, std::span<double>(y, static_cast<std::size_t>(y_len)));
        return 0;
    } catch (const std::exception &e) {
        if (err && err_len > 0) std::snprintf(err, static_cast<std::size_t>(err_len), "%s", e.what());
        return -1;
    }
}

// Runs `iterations` passes of the pdhg.cpp:92-130 backend-call sequence (fixed
// tau = sigma = step) on already-scaled data with the reference CPU backend.
// Returns seconds spent in the loop; x[n] and y[m] hold the final iterates.
} // extern "C"

namespace {
// The pdhg.cpp:92-130 call sequence on `bk`; seconds for `iterations` iterations.
double replay(vikalp::ExecutionBackend &bk, const vkref_problem *p, double step, int64_t iterations, double *x_out,
              double *y_out) {
    using vikalp::Transpose;
    vikalp::ExecutionBackend *be = &bk;
    const int64_t m = p->m, n = p->n;
    vikalp::CsrPattern pat;
    pat.rows = m;
    pat.columns = n;
    pat.row_offsets.assign(p->ro, p->ro + m + 1);
    pat.column_indices.assign(p->ci, p->ci + p->ro[m]);
    auto A = be->create_matrix(pat);
    be->set_values(std::span<const double>(p->v, static_cast<std::size_t>(p->ro[m])), *A);
    auto vec = [&](int64_t k) { return be->create_vector(k); };
    auto x = vec(n), xn = vec(n), xb = vec(n), aty = vec(n), g = vec(n), px = vec(n), res = vec(n);
    auto c = vec(n), l = vec(n), u = vec(n);
    auto y = vec(m), axb = vec(m), ya = vec(m), yp = vec(m), ax = vec(m), pax = vec(m), rl = vec(m), ru = vec(m);
    be->upload(std::span<const double>(p->c, static_cast<std::size_t>(n)), *c);
    be->upload(std::span<const double>(p->l, static_cast<std::size_t>(n)), *l);
    be->upload(std::span<const double>(p->u, static_cast<std::size_t>(n)), *u);
    be->upload(std::span<const double>(p->rl, static_cast<std::size_t>(m)), *rl);
    be->upload(std::span<const double>(p->ru, static_cast<std::size_t>(m)), *ru);
    be->fill(*x, 0.0);
    be->project_box(*x, *l, *u);
    be->fill(*y, 0.0);
    const double tau = step, sigma = step;
    double sink = 0.0;
    const auto t0 = std::chrono::steady_clock::now();
    for (int64_t it = 0; it < iterations; ++it) {
        be->multiply(1.0, *A, *y, 0.0, *aty, Transpose::Yes);
        be->copy(*x, *xn);
        be->axpby(-tau, *c, 1.0, *xn);
        be->axpby(-tau, *aty, 1.0, *xn);
        be->project_box(*xn, *l, *u);
        be->copy(*x, *xb);
        be->axpby(2.0, *xn, -1.0, *xb);
        be->multiply(1.0, *A, *xb, 0.0, *axb, Transpose::No);
        be->copy(*y, *ya);
        be->axpby(sigma, *axb, 1.0, *ya);
        be->copy(*ya, *yp);
        be->axpby(1.0 / sigma, *yp, 0.0, *yp);
        be->project_box(*yp, *rl, *ru);
        be->copy(*ya, *y);
        be->axpby(-sigma, *yp, 1.0, *y);
        be->copy(*xn, *x);
        be->multiply(1.0, *A, *x, 0.0, *ax, Transpose::No);
        be->copy(*ax, *pax);
        be->project_box(*pax, *rl, *ru);
        be->axpby(1.0, *pax, -1.0, *ax);
        sink += be->norm_inf(*ax);
        be->multiply(1.0, *A, *y, 0.0, *aty, Transpose::Yes);
        be->copy(*c, *g);
        be->axpby(1.0, *aty, 1.0, *g);
        be->copy(*x, *px);
        be->axpby(-1.0, *g, 1.0, *px);
        be->project_box(*px, *l, *u);
        be->copy(*x, *res);
        be->axpby(-1.0, *px, 1.0, *res);
        sink += be->norm_inf(*res);
    }
    be->synchronize();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (x_out) be->download(*x, std::span<double>(x_out, static_cast<std::size_t>(n)));
    if (y_out) be->download(*y, std::span<double>(y_out, static_cast<std::size_t>(m)));
    return secs + 0.0 * sink;
}
} // namespace

extern "C" {

double vkref_pdhg_replay(const vkref_problem *p, double step, int64_t iterations, double *x_out,
                         double *y_out) {
    auto be = vikalp::make_cpu_backend();
    return replay(*be, p, step, iterations, x_out, y_out);
}

#ifdef VKREF_CUDA
// The same sequence on the reference's CUDA backend (cuda/cuda_ops.cu:
// cuSPARSE SpMV, SIMT vector kernels, host-finished reductions), for the
// GPU-to-GPU comparison. Returns -1 when the backend throws.
double vkref_pdhg_replay_cuda(const vkref_problem *p, double step, int64_t iterations, double *x_out,
                              double *y_out) {
    try {
        auto be = vikalp::make_cuda_backend();
        return replay(*be, p, step, iterations, x_out, y_out);
    } catch (const std::exception &) {
        return -1.0;
    }
}
#endif

struct vkref_mps {
    vikalp::Model model;
    std::vector<vikalp::MpsError> errors;
    int ok = 0;
};

vkref_mps *vkref_mps_read(const char *path) {
    auto *h = new vkref_mps();
    vikalp::MpsReader r;
    h->ok = r.read(path, h->model) ? 1 : 0;
    h->errors = r.errors();
    return h;
}

int vkref_mps_ok(const vkref_mps *h) { return h->ok; }

void vkref_mps_sizes(const vkref_mps *h, int64_t *m, int64_t *n, int64_t *nnz) {
    const auto &A = h->model.constraint_matrix;
    *m = A.pattern.rows;
    *n = A.pattern.columns;
    *nnz = static_cast<int64_t>(A.pattern.column_indices.size());
}

// Arrays sized by vkref_mps_sizes: ro[m+1], ci[nnz], v[nnz], c/vl/vu/types[n], rl/ru[m].
void vkref_mps_arrays(const vkref_mps *h, int64_t *ro, int64_t *ci, double *v, double *c, double *vl, double *vu,
                      double *rl, double *ru, int32_t *types) {
    const vikalp::Model &md = h->model;
    const auto &A = md.constraint_matrix;
    std::copy(A.pattern.row_offsets.begin(), A.pattern.row_offsets.end(), ro);
    std::copy(A.pattern.column_indices.begin(), A.pattern.column_indices.end(), ci);
    std::copy(A.values.begin(), A.values.end(), v);
    std::copy(md.linear_objective.begin(), md.linear_objective.end(), c);
    std::copy(md.variable_lower.begin(), md.variable_lower.end(), vl);
    std::copy(md.variable_upper.begin(), md.variable_upper.end(), vu);
    std::copy(md.constraint_lower.begin(), md.constraint_lower.end(), rl);
    std::copy(md.constraint_upper.begin(), md.constraint_upper.end(), ru);
    for (std::size_t j = 0; j < md.variable_types.size(); ++j) types[j] = static_cast<int32_t>(md.variable_types[j]);
}

const char *vkref_mps_name(const vkref_mps *h) { return h->model.name.c_str(); }
int vkref_mps_error_count(const vkref_mps *h) { return static_cast<int>(h->errors.size()); }
const char *vkref_mps_error(const vkref_mps *h, int i, int64_t *line) {
    *line = static_cast<int64_t>(h->errors[static_cast<std::size_t>(i)].line);
    return h->errors[static_cast<std::size_t>(i)].message.c_str();
}
void vkref_mps_free(vkref_mps *h) { delete h; }

} // extern "C"
