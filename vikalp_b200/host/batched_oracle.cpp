// BatchedRelaxationOracle: branch-and-bound node relaxations of one model in
// one vk_batch_solve_shared call (the data-parallel form of the node loop of
// src/solver/mip/BranchAndBound.cpp:272-297, which calls the oracle once per
// node).
#include "vikalp/solver/BatchedRelaxationOracle.hpp"

#include "convert.hpp"
#include "vikalp_b200.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <exception>
#include <string>
#include <vector>

namespace vikalp {

SolveResult BatchedRelaxationOracle::solve(const Model &model, std::span<const Scalar> lower,
                                           std::span<const Scalar> upper, std::span<const Scalar> warm,
                                           const SolverOptions &options) const {
    const NodeRelaxation node{lower, upper, warm};
    return solve_batch(model, std::span<const NodeRelaxation>(&node, 1), options).front();
}

std::vector<SolveResult> BatchedRelaxationOracle::solve_batch(const Model &model,
                                                              std::span<const NodeRelaxation> nodes,
                                                              const SolverOptions &options) const {
    using detail::status_result;
    const auto started = std::chrono::steady_clock::now();
    const std::size_t k = nodes.size();
    std::vector<SolveResult> out(k);
    if (k == 0) return out;
    // what the batch cannot take goes node by node through the one-node oracle
    const bool per_node = options.backend == BackendPreference::CPU || model.nonlinear ||
                          model.has_quadratic_objective() || options.b200.sequential_products;
    if (per_node) {
        CudaRelaxationOracle one;
        for (std::size_t i = 0; i < k; ++i)
            out[i] = one.solve(model, nodes[i].variable_lower_override, nodes[i].variable_upper_override,
                               nodes[i].warm_start, options);
        return out;
    }
    try {
        const Index n = model.num_variables(), m = model.num_constraints();
        const auto nn = static_cast<std::size_t>(n);
        // node arrays, node i at offset i * n; a node that fails the size
        // checks of the one-node oracle gets its answer now and the model's
        // bounds in the batch (its result is replaced below)
        std::vector<Scalar> lo(k * nn), hi(k * nn), ws;
        std::vector<char> bad(k, 0);
        bool any_warm = false;
        for (const NodeRelaxation &nd : nodes) any_warm = any_warm || !nd.warm_start.empty();
        if (any_warm) ws.assign(k * nn, 0.0); // a cold start is x = 0 (clamped), as an absent warm start
        const auto sized = [n](std::span<const Scalar> s) { return s.empty() || static_cast<Index>(s.size()) == n; };
        for (std::size_t i = 0; i < k; ++i) {
            const NodeRelaxation &nd = nodes[i];
            Scalar *l = lo.data() + i * nn, *u = hi.data() + i * nn;
            if (!sized(nd.variable_lower_override) || !sized(nd.variable_upper_override)) {
                out[i] = status_result(SolveStatus::InvalidModel,
                                       "variable bound overrides must be empty or sized and non-NaN");
                bad[i] = 1;
            } else if (!sized(nd.warm_start)) {
                out[i] = status_result(SolveStatus::InvalidModel,
                                       "warm start must be empty or finite and sized to the model");
                bad[i] = 1;
            }
            const bool ol = !bad[i] && !nd.variable_lower_override.empty();
            const bool ou = !bad[i] && !nd.variable_upper_override.empty();
            for (std::size_t j = 0; j < nn; ++j) {
                l[j] = ol ? nd.variable_lower_override[j] : model.variable_lower[j];
                u[j] = ou ? nd.variable_upper_override[j] : model.variable_upper[j];
            }
            if (any_warm && !bad[i] && !nd.warm_start.empty())
                std::copy(nd.warm_start.begin(), nd.warm_start.end(), ws.begin() + static_cast<std::ptrdiff_t>(i * nn));
        }
        const vk_problem p = detail::to_problem(model);
        vk_options vo = detail::to_options(options);
        vo.algorithm = VK_ALGO_HALPERN; // the reference scheme has no batched form
        std::vector<vk_result> res(k);
        for (std::size_t i = 0; i < k; ++i) {
            res[i] = vk_result{};
            if (!bad[i]) detail::bind_outputs(out[i], n, m, res[i]);
        }
        // y: the row multipliers, needed for the split duals (kept per node)
        std::vector<std::vector<Scalar>> ys(k);
        for (std::size_t i = 0; i < k; ++i)
            if (!bad[i]) {
                ys[i].resize(static_cast<std::size_t>(m));
                res[i].y = ys[i].data();
            }
        const int rc = vk_batch_solve_shared(&p, static_cast<int32_t>(k), lo.data(), hi.data(),
                                             any_warm ? ws.data() : nullptr, &vo, res.data());
        if (rc != VK_OK) {
            const std::string err = vk_last_error();
            for (std::size_t i = 0; i < k; ++i) {
                out[i] = status_result(detail::status_of_error(rc), err);
                out[i].backend = "cuda";
            }
            return out;
        }
        const Scalar secs = std::chrono::duration<Scalar>(std::chrono::steady_clock::now() - started).count();
        for (std::size_t i = 0; i < k; ++i) {
            SolveResult &r = out[i];
            r.backend = "cuda";
            r.solver = "PDHG";
            if (bad[i]) continue;
            detail::finish_result(r, res[i]);
            r.solve_seconds = secs;
        }
        return out;
    } catch (const std::exception &e) {
        for (SolveResult &r : out) r = status_result(SolveStatus::NumericalFailure, e.what());
        return out;
    }
}

} // namespace vikalp
