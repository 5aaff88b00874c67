// vikalp::solve routed to the B200 PDHG / PDQP library through its C ABI.
//
// The reference's router (src/solver/Solver.cpp:92-146) validates the model,
// sends continuous classes to a RelaxationOracle, and its built-in oracle
// picks a backend (Solver.cpp:41-51) and runs solver::solve_lp / solve_qp.
// Here the continuous route is CudaRelaxationOracle: one vk_pdhg_create +
// vk_pdhg_solve pair per call, results mapped back to SolveResult in original
// coordinates. Backend preference Auto or CUDA uses it; CPU, nonlinear and
// discrete models are outside this library and return UnsupportedModel.
#include "vikalp/solver/Solver.hpp"

#include "vikalp_b200.h"

#include <chrono>
#include <exception>
#include <string>

namespace vikalp {
namespace {

SolveResult status_result(SolveStatus s, const std::string &msg) {
    SolveResult r;
    r.status = s;
    r.message = msg;
    return r;
}

vk_csr to_csr(const CsrMatrix &m) {
    return vk_csr{m.pattern.rows, m.pattern.columns, m.pattern.row_offsets.data(),
                  m.pattern.column_indices.empty() ? nullptr : m.pattern.column_indices.data(),
                  m.values.empty() ? nullptr : m.values.data()};
}

vk_options to_options(const SolverOptions &o) {
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

SolveStatus status_of_error(int rc) {
    if (rc == VK_ERR_INVALID) return SolveStatus::InvalidModel;
    if (rc == VK_ERR_UNSUPPORTED) return SolveStatus::UnsupportedModel;
    return SolveStatus::NumericalFailure; // backend failures, as Solver.cpp:81-86
}

} // namespace

SolveResult CudaRelaxationOracle::solve(const Model &model, std::span<const Scalar> lower,
                                        std::span<const Scalar> upper, std::span<const Scalar> warm,
                                        const SolverOptions &options) const {
    const auto started = std::chrono::steady_clock::now();
    try {
        if (options.backend == BackendPreference::CPU)
            return status_result(SolveStatus::UnsupportedModel,
                                 "the CPU backend is not part of this library; it runs the B200 CUDA path");
        const ProblemClass cls = model.has_quadratic_objective() ? ProblemClass::QP : ProblemClass::LP;
        if (model.nonlinear)
            return status_result(SolveStatus::UnsupportedModel, "No built-in continuous relaxation is available");
        const Index n = model.num_variables();
        const auto sized = [n](std::span<const Scalar> s) { return s.empty() || static_cast<Index>(s.size()) == n; };
        if (!sized(lower) || !sized(upper))
            return status_result(SolveStatus::InvalidModel,
                                 "variable bound overrides must be empty or sized and non-NaN");
        if (!sized(warm))
            return status_result(SolveStatus::InvalidModel, "warm start must be empty or finite and sized to the model");

        vk_problem p{};
        p.A = to_csr(model.constraint_matrix);
        p.Q = to_csr(model.quadratic_objective);
        p.c = model.linear_objective.data();
        p.objective_offset = model.objective_offset;
        p.var_lower = model.variable_lower.data();
        p.var_upper = model.variable_upper.data();
        p.row_lower = model.constraint_lower.data();
        p.row_upper = model.constraint_upper.data();
        const vk_options vo = to_options(options);
        vk_pdhg *h = nullptr;
        if (const int rc = vk_pdhg_create(&p, &vo, &h); rc != VK_OK) {
            SolveResult r = status_result(status_of_error(rc), vk_last_error());
            r.backend = "cuda";
            return r;
        }
        SolveResult r;
        const auto nn = static_cast<std::size_t>(n), mm = static_cast<std::size_t>(model.num_constraints());
        r.primal_solution.resize(nn);
        r.constraint_lower_dual.resize(mm);
        r.constraint_upper_dual.resize(mm);
        r.variable_lower_dual.resize(nn);
        r.variable_upper_dual.resize(nn);
        vk_result out{};
        out.x = r.primal_solution.data();
        out.row_lower_dual = r.constraint_lower_dual.data();
        out.row_upper_dual = r.constraint_upper_dual.data();
        out.var_lower_dual = r.variable_lower_dual.data();
        out.var_upper_dual = r.variable_upper_dual.data();
        const int rc = vk_pdhg_solve(h, warm.empty() ? nullptr : warm.data(), lower.empty() ? nullptr : lower.data(),
                                     upper.empty() ? nullptr : upper.data(), &out);
        const std::string err = rc == VK_OK ? std::string() : std::string(vk_last_error());
        vk_pdhg_destroy(h);
        r.backend = "cuda";
        r.solver = cls == ProblemClass::QP ? "PDQP" : "PDHG";
        if (rc != VK_OK) {
            r.status = SolveStatus::NumericalFailure;
            r.message = err;
            return r;
        }
        r.status = static_cast<SolveStatus>(out.status);
        r.message = out.message;
        if (r.status == SolveStatus::InvalidModel) { // a solve-time model error: no solution
            r.primal_solution.clear();
            r.constraint_lower_dual.clear();
            r.constraint_upper_dual.clear();
            r.variable_lower_dual.clear();
            r.variable_upper_dual.clear();
            return r;
        }
        r.iterations = out.iterations;
        r.objective_value = out.objective;
        r.primal_residual = out.primal_residual;
        r.stationarity_residual = out.stationarity_residual;
        r.complementarity_residual = out.complementarity_residual;
        if (r.status == SolveStatus::Optimal) { // pdhg.cpp:256-261
            r.primal_bound = r.objective_value;
            r.dual_bound = r.objective_value;
            r.absolute_gap = 0.0;
            r.relative_gap = 0.0;
        }
        r.solve_seconds = std::chrono::duration<Scalar>(std::chrono::steady_clock::now() - started).count();
        return r;
    } catch (const std::exception &e) {
        return status_result(SolveStatus::NumericalFailure, e.what());
    }
}

SolveResult solve(const Model &model, const SolverOptions &options) {
    CudaRelaxationOracle oracle;
    SolveResult r = solve(model, oracle, options);
    if (r.backend.empty() && r.status != SolveStatus::UnsupportedModel) r.backend = "cuda";
    return r;
}

SolveResult solve(const Model &model, const RelaxationOracle &oracle, const SolverOptions &options) {
    const auto errors = model.validate();
    if (!errors.empty()) return status_result(SolveStatus::InvalidModel, errors.front());
    switch (model.problem_class()) {
    case ProblemClass::LP:
    case ProblemClass::QP: {
        SolveResult r = oracle.solve(model, {}, {}, {}, options);
        r.solver = "vikalp-continuous";
        return r;
    }
    case ProblemClass::NLP:
        return status_result(SolveStatus::UnsupportedModel,
                             "nonlinear models are outside the B200 PDHG path (the reference's IPM is not built)");
    case ProblemClass::MILP:
    case ProblemClass::MIQP:
    case ProblemClass::MINLP:
        return status_result(SolveStatus::UnsupportedModel,
                             "mixed-integer models are outside the B200 PDHG path (branch-and-bound is not built)");
    }
    return status_result(SolveStatus::UnsupportedModel, "Unknown problem class");
}

} // namespace vikalp
