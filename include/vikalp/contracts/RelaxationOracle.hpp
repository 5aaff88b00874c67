#pragma once
// Continuous-relaxation oracle (interface of the reference's
// include/vikalp/contracts/RelaxationOracle.hpp:11-23). Override and
// warm-start spans are empty or num_variables() long; empty overrides use the
// model's bounds, an empty warm start means a cold start.
#include "vikalp/contracts/Model.hpp"
#include "vikalp/contracts/SolveResult.hpp"
#include "vikalp/contracts/SolverOptions.hpp"

#include <span>

namespace vikalp {

class RelaxationOracle {
public:
    virtual ~RelaxationOracle() = default;
    [[nodiscard]] virtual SolveResult solve(const Model &model, std::span<const Scalar> variable_lower_override,
                                            std::span<const Scalar> variable_upper_override,
                                            std::span<const Scalar> warm_start,
                                            const SolverOptions &options) const = 0;
};

} // namespace vikalp
