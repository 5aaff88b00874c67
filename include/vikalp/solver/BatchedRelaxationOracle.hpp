#pragma once
// A relaxation oracle that solves many branch-and-bound nodes of one model in
// one device batch.
//
// The reference's branch-and-bound loop pops one node at a time and calls
// RelaxationOracle::solve(working_model, lower, upper, node.relaxation_solution,
// options) for it (src/solver/mip/BranchAndBound.cpp:272-297). A caller that
// pops k nodes instead hands them to solve_batch: the k relaxations share every
// read of the constraint matrix on the GPU (vk_batch_solve_shared) and come
// back in node order, each a full SolveResult -- primal solution, the four
// split dual vectors, the reference's three residuals, objective, bounds and
// status -- as CudaRelaxationOracle returns it for that node alone (up to
// rounding: each node keeps its own primal weight, restarts and stopping).
//
// Determinism: the same nodes in the same order give the same results, bit
// for bit, every time (the sparse passes' variant picks are fixed per matrix
// for the process and every reduction runs in a fixed order).
//
// Batches run the restarted Halpern scheme (stop: SolverOptions::b200.
// relative_tolerance, relative KKT in original units) whatever
// SolverOptions::b200.scheme says: the reference's fixed-rule scheme has no
// batched form. Nodes whose overrides or warm start fail the single-node
// checks get InvalidModel with the single-node message; the others are
// solved. What the batch cannot take (a quadratic objective, a nonlinear
// model, sequential products, the CPU backend) goes node by node through
// CudaRelaxationOracle with the options as given, so solve_batch always
// answers.
#include "vikalp/contracts/RelaxationOracle.hpp"
#include "vikalp/solver/Solver.hpp"

#include <span>
#include <vector>

namespace vikalp {

// One node relaxation: bound overrides and warm start, each empty or
// num_variables() long (RelaxationOracle.hpp's conventions).
struct NodeRelaxation {
    std::span<const Scalar> variable_lower_override;
    std::span<const Scalar> variable_upper_override;
    std::span<const Scalar> warm_start;
};

class BatchedRelaxationOracle final : public RelaxationOracle {
public:
    // One node: a batch of one.
    [[nodiscard]] SolveResult solve(const Model &model, std::span<const Scalar> variable_lower_override,
                                    std::span<const Scalar> variable_upper_override,
                                    std::span<const Scalar> warm_start,
                                    const SolverOptions &options) const override;

    // nodes.size() relaxations of `model` in one batch; results[i] answers nodes[i].
    [[nodiscard]] std::vector<SolveResult> solve_batch(const Model &model, std::span<const NodeRelaxation> nodes,
                                                       const SolverOptions &options) const;
};

} // namespace vikalp
