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

#include "convert.hpp"
#include "vikalp_b200.h"

#include <chrono>
#include <exception>
#include <string>

namespace vikalp {
using detail::finish_result;
using detail::status_of_error;
using detail::status_result;

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

        const vk_problem p = detail::to_problem(model);
        const vk_options vo = detail::to_options(options);
        vk_pdhg *h = nullptr;
        if (const int rc = vk_pdhg_create(&p, &vo, &h); rc != VK_OK) {
            SolveResult r = status_result(status_of_error(rc), vk_last_error());
            r.backend = "cuda";
            return r;
        }
        SolveResult r;
        vk_result out{};
        detail::bind_outputs(r, n, model.num_constraints(), out);
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
        finish_result(r, out);
        if (r.status == SolveStatus::InvalidModel) return r; // a solve-time model error: no solution
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
