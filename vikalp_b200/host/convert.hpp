#pragma once
// Conversions between the C++ contract types and the C ABI, shared by the
// relaxation oracles of this host layer (not installed).
#include "vikalp/contracts/Model.hpp"
#include "vikalp/contracts/SolveResult.hpp"
#include "vikalp/contracts/SolverOptions.hpp"

#include "vikalp_b200.h"

#include <string>

namespace vikalp::detail {

inline SolveResult status_result(SolveStatus s, const std::string &msg) {
    SolveResult r;
    r.status = s;
    r.message = msg;
    return r;
}

inline vk_csr to_csr(const CsrMatrix &m) {
    return vk_csr{m.pattern.rows, m.pattern.columns, m.pattern.row_offsets.data(),
                  m.pattern.column_indices.empty() ? nullptr : m.pattern.column_indices.data(),
                  m.values.empty() ? nullptr : m.values.data()};
}

inline vk_options to_options(const SolverOptions &o) {
    vk_options v;
    vk_default_options(&v);
    v.iteration_limit = o.iteration_limit;
    v.time_limit_seconds = o.time_limit_seconds;
    v.primal_tolerance = o.primal_tolerance;
    v.dual_tolerance = o.dual_tolerance;
    v.continuous_method = static_cast<int32_t>(o.continuous_method);
    v.algorithm = o.b200.scheme == B200Options::Scheme::Halpern ? VK_ALGO_HALPERN : VK_ALGO_REFERENCE;
    v.precision = o.b200.mixed_precision ? VK_PREC_MIXED : VK_PREC_FP64;
    v.spmv_order = o.b200.sequential_products ? VK_SPMV_SEQUENTIAL : VK_SPMV_FAST;
    v.relative_tolerance = o.b200.relative_tolerance;
    v.check_every = o.b200.check_every;
    v.device = o.b200.device;
    return v;
}

inline vk_problem to_problem(const Model &model) {
    vk_problem p{};
    p.A = to_csr(model.constraint_matrix);
    p.Q = to_csr(model.quadratic_objective);
    p.c = model.linear_objective.data();
    p.objective_offset = model.objective_offset;
    p.var_lower = model.variable_lower.data();
    p.var_upper = model.variable_upper.data();
    p.row_lower = model.constraint_lower.data();
    p.row_upper = model.constraint_upper.data();
    return p;
}

inline SolveStatus status_of_error(int rc) {
    if (rc == VK_ERR_INVALID) return SolveStatus::InvalidModel;
    if (rc == VK_ERR_UNSUPPORTED) return SolveStatus::UnsupportedModel;
    return SolveStatus::NumericalFailure; // backend failures, as Solver.cpp:81-86
}

// Sizes r's solution and dual vectors for a model and points `out` at them.
inline void bind_outputs(SolveResult &r, Index n, Index m, vk_result &out) {
    const auto nn = static_cast<std::size_t>(n), mm = static_cast<std::size_t>(m);
    r.primal_solution.resize(nn);
    r.constraint_lower_dual.resize(mm);
    r.constraint_upper_dual.resize(mm);
    r.variable_lower_dual.resize(nn);
    r.variable_upper_dual.resize(nn);
    out.x = r.primal_solution.data();
    out.row_lower_dual = r.constraint_lower_dual.data();
    out.row_upper_dual = r.constraint_upper_dual.data();
    out.var_lower_dual = r.variable_lower_dual.data();
    out.var_upper_dual = r.variable_upper_dual.data();
}

// The scalar fields of a finished solve (status, message, counts, objective,
// residuals; the bounds and gaps of an optimal answer, pdhg.cpp:256-261). A
// solve-time model error keeps no solution.
inline void finish_result(SolveResult &r, const vk_result &out) {
    r.status = static_cast<SolveStatus>(out.status);
    r.message = out.message;
    if (r.status == SolveStatus::InvalidModel) {
        r.primal_solution.clear();
        r.constraint_lower_dual.clear();
        r.constraint_upper_dual.clear();
        r.variable_lower_dual.clear();
        r.variable_upper_dual.clear();
        return;
    }
    r.iterations = out.iterations;
    r.objective_value = out.objective;
    r.primal_residual = out.primal_residual;
    r.stationarity_residual = out.stationarity_residual;
    r.complementarity_residual = out.complementarity_residual;
    if (r.status == SolveStatus::Optimal) {
        r.primal_bound = r.objective_value;
        r.dual_bound = r.objective_value;
        r.absolute_gap = 0.0;
        r.relative_gap = 0.0;
    }
}

} // namespace vikalp::detail
