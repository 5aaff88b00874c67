#pragma once
// Top-level entry points (the reference's include/vikalp/solver/Solver.hpp:19-30).
// Continuous LP / QP models go to the B200 PDHG / PDQP path
// (BackendPreference::CUDA or Auto). The reference's CPU backend and its
// discrete / nonlinear engines are not part of this library: those requests
// return UnsupportedModel with a message saying so.
#include "vikalp/contracts/Model.hpp"
#include "vikalp/contracts/RelaxationOracle.hpp"
#include "vikalp/contracts/SolveResult.hpp"
#include "vikalp/contracts/SolverOptions.hpp"

namespace vikalp {

[[nodiscard]] SolveResult solve(const Model &model, const SolverOptions &options = {});

[[nodiscard]] SolveResult solve(const Model &model, const RelaxationOracle &oracle, const SolverOptions &options);

// The relaxation oracle solve() uses for continuous models: every call runs
// one vk_pdhg_create / vk_pdhg_solve pair on the GPU.
class CudaRelaxationOracle final : public RelaxationOracle {
public:
    [[nodiscard]] SolveResult solve(const Model &model, std::span<const Scalar> variable_lower_override,
                                    std::span<const Scalar> variable_upper_override,
                                    std::span<const Scalar> warm_start,
                                    const SolverOptions &options) const override;
};

} // namespace vikalp
