// BatchedRelaxationOracle, written the way the reference's branch-and-bound
// tests are (tests/solver/integer/test_mip.cpp: expect counters, exit code 0 or
// 1). The node loop below pops k nodes at a time in best-bound order with ties
// broken by node id, the batched form of BranchAndBound.cpp:272-297.
//
//   test_batched_oracle cpu   routes that never reach the GPU
//   test_batched_oracle gpu   batches against one-node solves, node order,
//                             split duals and residuals, determinism (needs a GPU)
#include "vikalp/solver/BatchedRelaxationOracle.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <queue>
#include <vector>

namespace {

int failures = 0;

void expect(bool c, const char *what) {
    if (!c) {
        std::cerr << "FAIL: " << what << '\n';
        ++failures;
    }
}

void expect_near(double a, double b, double tol, const char *what) {
    const bool ok = std::isfinite(a) && std::abs(a - b) <= tol;
    expect(ok, what);
    if (!ok) std::cerr << "  got " << a << " want " << b << '\n';
}

// Small seeded LP of the workloads' kind: 4 distinct rows per column, values
// in [-1, 1], a feasible x0 in [0, 10] fixes the rows (even rows equalities,
// odd rows <= A x0 + slack), c in [-1, 1], x in [0, 10].
struct Lcg {
    uint64_t s;
    double next() {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        return static_cast<double>(s >> 11) / 9007199254740992.0;
    }
};

vikalp::Model small_lp(int m, int n, uint64_t seed) {
    Lcg g{seed};
    std::vector<std::vector<std::pair<int, double>>> rows(m);
    for (int j = 0; j < n; ++j) {
        std::vector<int> picked;
        while (picked.size() < 4) {
            const int r = static_cast<int>(g.next() * m);
            if (std::find(picked.begin(), picked.end(), r) == picked.end()) picked.push_back(r);
        }
        for (int r : picked) rows[r].push_back({j, 2.0 * g.next() - 1.0});
    }
    vikalp::Model md;
    md.constraint_matrix.pattern.rows = m;
    md.constraint_matrix.pattern.columns = n;
    md.constraint_matrix.pattern.row_offsets.assign(1, 0); // CsrPattern starts as {0}
    for (auto &row : rows) {
        std::sort(row.begin(), row.end());
        for (auto &[c, v] : row) {
            md.constraint_matrix.pattern.column_indices.push_back(c);
            md.constraint_matrix.values.push_back(v);
        }
        md.constraint_matrix.pattern.row_offsets.push_back(
            static_cast<vikalp::Index>(md.constraint_matrix.pattern.column_indices.size()));
    }
    std::vector<double> x0(n);
    for (double &v : x0) v = 10.0 * g.next();
    for (int i = 0; i < m; ++i) {
        double r = 0.0;
        for (auto &[c, v] : rows[i]) r += v * x0[c];
        if (i % 2 == 0) {
            md.constraint_lower.push_back(r);
            md.constraint_upper.push_back(r);
        } else {
            md.constraint_lower.push_back(-vikalp::Model::infinity());
            md.constraint_upper.push_back(r + g.next());
        }
    }
    for (int j = 0; j < n; ++j) md.linear_objective.push_back(2.0 * g.next() - 1.0);
    md.variable_lower.assign(n, 0.0);
    md.variable_upper.assign(n, 10.0);
    md.variable_types.assign(n, vikalp::VariableType::Continuous);
    return md;
}

vikalp::SolverOptions options() {
    vikalp::SolverOptions o;
    o.iteration_limit = 200'000;
    o.time_limit_seconds = 60.0;
    o.b200.scheme = vikalp::B200Options::Scheme::Halpern;
    o.b200.relative_tolerance = 1e-7;
    return o;
}

void cpu_routes() {
    const auto model = small_lp(20, 40, 3);
    expect(model.validate().empty(), "test model valid");
    vikalp::BatchedRelaxationOracle oracle;
    expect(oracle.solve_batch(model, {}, options()).empty(), "empty batch: no results");
    // the CPU backend is not in this library: every node says so, in order
    auto o = options();
    o.backend = vikalp::BackendPreference::CPU;
    std::vector<double> lo(40, 1.0);
    std::vector<vikalp::NodeRelaxation> nodes(3);
    nodes[1].variable_lower_override = lo;
    const auto rs = oracle.solve_batch(model, nodes, o);
    expect(rs.size() == 3, "cpu backend: one result per node");
    for (const auto &r : rs) expect(r.status == vikalp::SolveStatus::UnsupportedModel, "cpu backend: unsupported");
}

struct Node {
    int id;
    double bound;
    std::vector<double> lo, hi, warm;
};

struct ByBound {
    bool operator()(const Node &a, const Node &b) const {
        return a.bound != b.bound ? a.bound > b.bound : a.id > b.id; // best bound first, then lower id
    }
};

// A few rounds of a batched best-bound loop on the LP's variables treated as
// integers: pop up to k nodes, solve them in one batch, branch on the most
// fractional variable of each. Returns the processed (id, objective, branch
// variable) sequence.
std::vector<std::tuple<int, double, int>> batched_loop(const vikalp::Model &model, int rounds, int k) {
    vikalp::BatchedRelaxationOracle oracle;
    const int n = static_cast<int>(model.num_variables());
    std::priority_queue<Node, std::vector<Node>, ByBound> queue;
    queue.push(Node{0, -1e300, model.variable_lower, model.variable_upper, {}});
    int next_id = 1;
    std::vector<std::tuple<int, double, int>> seq;
    for (int round = 0; round < rounds && !queue.empty(); ++round) {
        std::vector<Node> pop;
        while (!queue.empty() && static_cast<int>(pop.size()) < k) {
            pop.push_back(queue.top());
            queue.pop();
        }
        std::vector<vikalp::NodeRelaxation> nodes;
        for (const Node &nd : pop) nodes.push_back({nd.lo, nd.hi, nd.warm});
        const auto rs = oracle.solve_batch(model, nodes, options());
        for (std::size_t i = 0; i < pop.size(); ++i) {
            const auto &r = rs[i];
            if (r.status != vikalp::SolveStatus::Optimal) {
                seq.push_back({pop[i].id, NAN, -1});
                continue;
            }
            int best = -1;
            double frac = 1e-6;
            for (int j = 0; j < n; ++j) {
                const double f = std::abs(r.primal_solution[j] - std::round(r.primal_solution[j]));
                if (f > frac) {
                    frac = f;
                    best = j;
                }
            }
            seq.push_back({pop[i].id, r.objective_value, best});
            if (best < 0) continue;
            Node down{next_id++, r.objective_value, pop[i].lo, pop[i].hi, r.primal_solution};
            down.hi[best] = std::floor(r.primal_solution[best]);
            Node up{next_id++, r.objective_value, pop[i].lo, pop[i].hi, r.primal_solution};
            up.lo[best] = std::ceil(r.primal_solution[best]);
            queue.push(down);
            queue.push(up);
        }
    }
    return seq;
}

void gpu_batches() {
    const int m = 40, n = 100;
    const auto model = small_lp(m, n, 11);
    expect(model.validate().empty(), "test model valid");
    vikalp::BatchedRelaxationOracle batched;
    vikalp::CudaRelaxationOracle one;
    // 10 nodes: tightened bounds, a warm start, a wrong-size override, a crossed interval
    std::vector<std::vector<double>> los, his;
    Lcg g{5};
    for (int b = 0; b < 10; ++b) {
        std::vector<double> lo(model.variable_lower), hi(model.variable_upper);
        for (int t = 0; t <= b % 4; ++t) {
            const int j = static_cast<int>(g.next() * n);
            if (g.next() < 0.5)
                hi[j] = std::floor(6.0 * g.next());
            else
                lo[j] = std::ceil(4.0 + 5.0 * g.next());
        }
        los.push_back(lo);
        his.push_back(hi);
    }
    his[7][3] = -1.0; // lower 0 > upper -1: the device checks reject it
    const std::vector<double> short_override(n - 1, 0.0);
    std::vector<vikalp::NodeRelaxation> nodes;
    for (int b = 0; b < 10; ++b) nodes.push_back({los[b], his[b], {}});
    nodes[4].variable_lower_override = short_override;
    auto opts = options();
    const auto rs = batched.solve_batch(model, nodes, opts);
    expect(rs.size() == nodes.size(), "one result per node");
    expect(rs[4].status == vikalp::SolveStatus::InvalidModel, "wrong-size override: InvalidModel");
    expect(rs[4].message == "variable bound overrides must be empty or sized and non-NaN", "wrong-size message");
    expect(rs[7].status == vikalp::SolveStatus::InvalidModel, "crossed interval: InvalidModel");
    expect(rs[7].message == "variable bound overrides contain an invalid interval", "crossed interval message");
    for (int b = 0; b < 10; ++b) {
        if (b == 4 || b == 7) continue;
        const auto &r = rs[b];
        expect(r.status == vikalp::SolveStatus::Optimal, "node optimal");
        expect(r.backend == "cuda", "backend cuda");
        expect(r.primal_solution.size() == static_cast<std::size_t>(n), "x sized");
        expect(r.constraint_lower_dual.size() == static_cast<std::size_t>(m) &&
                   r.constraint_upper_dual.size() == static_cast<std::size_t>(m) &&
                   r.variable_lower_dual.size() == static_cast<std::size_t>(n) &&
                   r.variable_upper_dual.size() == static_cast<std::size_t>(n),
               "duals sized");
        bool nonneg = true, split = true;
        for (int i = 0; i < m; ++i) {
            nonneg = nonneg && r.constraint_lower_dual[i] >= 0.0 && r.constraint_upper_dual[i] >= 0.0;
            split = split && (r.constraint_lower_dual[i] == 0.0 || r.constraint_upper_dual[i] == 0.0);
        }
        for (int j = 0; j < n; ++j) nonneg = nonneg && r.variable_lower_dual[j] >= 0.0 && r.variable_upper_dual[j] >= 0.0;
        expect(nonneg, "duals non-negative");
        expect(split, "row duals split into one side");
        expect(std::isfinite(r.primal_residual) && r.primal_residual <= 1e-4, "primal residual reported and small");
        expect(std::isfinite(r.stationarity_residual), "stationarity residual reported");
        expect(std::isfinite(r.complementarity_residual), "complementarity residual reported");
        for (int j = 0; j < n; ++j)
            expect(r.primal_solution[j] >= los[b][j] - 1e-9 && r.primal_solution[j] <= his[b][j] + 1e-9,
                   "x within the node's bounds");
        // the same node alone through the one-node oracle
        const auto single = one.solve(model, los[b], his[b], {}, opts);
        expect(single.status == vikalp::SolveStatus::Optimal, "one-node solve optimal");
        expect_near(r.objective_value, single.objective_value, 1e-5 * (1.0 + std::abs(single.objective_value)),
                    "batch objective = one-node objective");
        expect_near(r.dual_bound, r.objective_value, 0.0, "optimal: dual bound = objective");
    }
    // the same nodes again: the same bits
    const auto again = batched.solve_batch(model, nodes, opts);
    bool same = true;
    for (std::size_t b = 0; b < nodes.size(); ++b) {
        same = same && again[b].status == rs[b].status && again[b].primal_solution == rs[b].primal_solution &&
               again[b].constraint_upper_dual == rs[b].constraint_upper_dual &&
               again[b].variable_lower_dual == rs[b].variable_lower_dual &&
               (std::isnan(rs[b].objective_value) || again[b].objective_value == rs[b].objective_value);
    }
    expect(same, "determinism: identical results on a second call");
    // warm starts from the first answers: optimal again, no more iterations
    std::vector<vikalp::NodeRelaxation> warm_nodes;
    for (int b = 0; b < 10; ++b)
        if (b != 4 && b != 7) warm_nodes.push_back({los[b], his[b], rs[b].primal_solution});
    const auto warm = batched.solve_batch(model, warm_nodes, opts);
    int wi = 0;
    for (int b = 0; b < 10; ++b) {
        if (b == 4 || b == 7) continue;
        expect(warm[wi].status == vikalp::SolveStatus::Optimal, "warm node optimal");
        expect_near(warm[wi].objective_value, rs[b].objective_value, 1e-5 * (1.0 + std::abs(rs[b].objective_value)),
                    "warm node objective");
        ++wi;
    }
    // one node through the RelaxationOracle interface (a batch of one)
    const vikalp::RelaxationOracle &as_oracle = batched;
    const auto r0 = as_oracle.solve(model, los[0], his[0], {}, opts);
    expect_near(r0.objective_value, rs[0].objective_value, 1e-5 * (1.0 + std::abs(rs[0].objective_value)),
                "batch of one = batch member");
    // deterministic node order (test_mip.cpp:534): two runs of the batched loop agree exactly
    const auto s1 = batched_loop(model, 4, 4), s2 = batched_loop(model, 4, 4);
    expect(s1.size() == s2.size() && s1.size() >= 4, "batched loop processed nodes");
    bool same_order = s1.size() == s2.size();
    for (std::size_t i = 0; same_order && i < s1.size(); ++i) {
        const auto &[ia, oa, ba] = s1[i];
        const auto &[ib, ob, bb] = s2[i];
        same_order = ia == ib && ba == bb && (oa == ob || (std::isnan(oa) && std::isnan(ob)));
    }
    expect(same_order, "deterministic node order and answers across runs");
}

} // namespace

int main(int argc, char **argv) {
    const bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
    cpu_routes();
    if (gpu) gpu_batches();
    if (failures == 0) std::cout << "ALL CHECKS PASSED\n";
    return failures == 0 ? 0 : 1;
}
