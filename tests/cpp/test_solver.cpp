// vikalp::solve on the B200 path, written the way the reference's own tests
// are (tests/solver/integration/test_solver.cpp, tests/solver/continuous/
// test_pdhg.cpp): expect / expect_near counters, exit code 0 or 1.
//
//   test_solver cpu   routes that never reach the GPU (validation, unsupported
//                     classes and backends)
//   test_solver gpu   the LP / QP known answers through vikalp::solve and the
//                     CUDA relaxation oracle (needs a GPU)
#include "vikalp/contracts/NonlinearOracle.hpp"
#include "vikalp/solver/Solver.hpp"

#include <cmath>
#include <cstring>
#include <iostream>
#include <memory>
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
    expect(std::isfinite(a) && std::abs(a - b) <= tol, what);
    if (!(std::isfinite(a) && std::abs(a - b) <= tol)) std::cerr << "  got " << a << " want " << b << '\n';
}

vikalp::SolverOptions options() {
    vikalp::SolverOptions o;
    o.iteration_limit = 10'000;
    o.time_limit_seconds = 10.0;
    o.primal_tolerance = 1e-5;
    o.dual_tolerance = 1e-5;
    return o;
}

vikalp::Model one_variable(vikalp::VariableType t) {
    vikalp::Model m;
    m.linear_objective = {-1.0};
    m.variable_lower = {0.0};
    m.variable_upper = {10.0};
    m.variable_types = {t};
    m.constraint_matrix.pattern = {0, 1, {0}, {}};
    return m;
}

class Quadratic final : public vikalp::NonlinearOracle {
public:
    vikalp::Index variables() const noexcept override { return 1; }
    vikalp::Index constraints() const noexcept override { return 0; }
    vikalp::Scalar objective(std::span<const vikalp::Scalar> x) const override { return (x[0] - 0.6) * (x[0] - 0.6); }
    void objective_gradient(std::span<const vikalp::Scalar> x, std::span<vikalp::Scalar> g) const override {
        g[0] = 2.0 * (x[0] - 0.6);
    }
    void constraint_values(std::span<const vikalp::Scalar>, std::span<vikalp::Scalar>) const override {}
    const vikalp::CsrPattern &jacobian_pattern() const noexcept override { return jac_; }
    void jacobian_values(std::span<const vikalp::Scalar>, std::span<vikalp::Scalar>) const override {}
    const vikalp::CsrPattern &hessian_pattern() const noexcept override { return hes_; }
    void hessian_values(std::span<const vikalp::Scalar>, vikalp::Scalar s, std::span<const vikalp::Scalar>,
                        std::span<vikalp::Scalar> v) const override {
        v[0] = 2.0 * s;
    }

private:
    vikalp::CsrPattern jac_{0, 1, {0}, {}};
    vikalp::CsrPattern hes_{1, 1, {0, 1}, {0}};
};

void cpu_routes() {
    // invalid bounds (test_pdhg.cpp:193-196)
    auto bad = one_variable(vikalp::VariableType::Continuous);
    bad.variable_lower = {3.0};
    bad.variable_upper = {2.0};
    const auto r1 = vikalp::solve(bad, options());
    expect(r1.status == vikalp::SolveStatus::InvalidModel, "invalid bounds are rejected");
    expect(r1.message == "variable bounds contains an invalid bound at index 0", "invalid-bound message");
    // a model whose metadata sizes disagree
    auto sizes = one_variable(vikalp::VariableType::Continuous);
    sizes.variable_types.clear();
    expect(vikalp::solve(sizes, options()).status == vikalp::SolveStatus::InvalidModel, "metadata sizes");
    // discrete and nonlinear classes are outside this path
    const auto milp = vikalp::solve(one_variable(vikalp::VariableType::Integer), options());
    expect(milp.status == vikalp::SolveStatus::UnsupportedModel, "MILP is unsupported here");
    auto nlp = one_variable(vikalp::VariableType::Continuous);
    nlp.nonlinear = std::make_shared<Quadratic>();
    expect(vikalp::solve(nlp, options()).status == vikalp::SolveStatus::UnsupportedModel, "NLP is unsupported here");
    // the CPU backend is not part of this library
    auto cpu = options();
    cpu.backend = vikalp::BackendPreference::CPU;
    const auto r2 = vikalp::solve(one_variable(vikalp::VariableType::Continuous), cpu);
    expect(r2.status == vikalp::SolveStatus::UnsupportedModel, "CPU backend request is unsupported");
    // non-convex QP (test_pdhg.cpp:161-164) is rejected before any device work
    auto nc = one_variable(vikalp::VariableType::Continuous);
    nc.linear_objective = {-10.0};
    nc.quadratic_objective.pattern = {1, 1, {0, 1}, {0}};
    nc.quadratic_objective.values = {-2.0};
    auto o = options();
    o.backend = vikalp::BackendPreference::CUDA;
    expect(vikalp::solve(nc, o).status == vikalp::SolveStatus::UnsupportedModel, "non-convex QP is rejected");
    // negative iteration limit (test_pdhg.cpp:212-216)
    auto neg = options();
    neg.iteration_limit = -1;
    neg.backend = vikalp::BackendPreference::CUDA;
    expect(vikalp::solve(one_variable(vikalp::VariableType::Continuous), neg).status ==
               vikalp::SolveStatus::InvalidModel,
           "negative iteration limits are rejected");
}

void gpu_routes() {
    auto o = options();
    o.backend = vikalp::BackendPreference::CUDA;
    // test_solver.cpp:81-87: LP x = 10
    const auto lp = vikalp::solve(one_variable(vikalp::VariableType::Continuous), o);
    expect(lp.status == vikalp::SolveStatus::Optimal, "LP integrated route");
    expect(!lp.primal_solution.empty(), "LP returns a solution");
    if (!lp.primal_solution.empty()) expect_near(lp.primal_solution[0], 10.0, 1e-4, "LP solution");
    expect(lp.backend == "cuda", "LP backend label");
    expect(lp.solver == "vikalp-continuous", "continuous solver label");
    expect_near(lp.dual_bound, lp.objective_value, 0.0, "optimal dual bound equals objective");
    // test_solver.cpp:98-109: QP min x^2 - 1.2x on [0, 2] -> 0.6
    auto qp = one_variable(vikalp::VariableType::Continuous);
    qp.linear_objective = {-1.2};
    qp.variable_upper = {2.0};
    qp.quadratic_objective.pattern = {1, 1, {0, 1}, {0}};
    qp.quadratic_objective.values = {2.0};
    const auto q = vikalp::solve(qp, o);
    expect(q.status == vikalp::SolveStatus::Optimal, "QP integrated route");
    if (!q.primal_solution.empty()) expect_near(q.primal_solution[0], 0.6, 1e-4, "QP solution");
    // the MPS fixture tests/io/simple_lp.mps: min x1, x1 <= 5, 0 <= x1 <= 10 -> 0
    vikalp::Model mps;
    mps.linear_objective = {1.0};
    mps.variable_lower = {0.0};
    mps.variable_upper = {10.0};
    mps.variable_types = {vikalp::VariableType::Continuous};
    mps.constraint_matrix.pattern = {1, 1, {0, 1}, {0}};
    mps.constraint_matrix.values = {1.0};
    mps.constraint_lower = {-vikalp::Model::infinity()};
    mps.constraint_upper = {5.0};
    const auto r = vikalp::solve(mps, o);
    expect(r.status == vikalp::SolveStatus::Optimal, "MPS model route");
    if (!r.primal_solution.empty()) expect_near(r.primal_solution[0], 0.0, 1e-5, "MPS model solution");
    // test_pdhg.cpp:118-136 through the oracle: x <= 3 row, warm start 2, upper override 4 -> 3
    auto row = one_variable(vikalp::VariableType::Continuous);
    row.variable_upper = {20.0};
    row.constraint_matrix.pattern = {1, 1, {0, 1}, {0}};
    row.constraint_matrix.values = {1.0};
    row.constraint_lower = {-vikalp::Model::infinity()};
    row.constraint_upper = {3.0};
    vikalp::CudaRelaxationOracle oracle;
    const std::vector<double> warm = {2.0}, upper = {4.0};
    auto po = o;
    po.iteration_limit = 5000;
    const auto rel = oracle.solve(row, {}, upper, warm, po);
    expect(rel.status == vikalp::SolveStatus::Optimal, "oracle with warm start and override");
    if (!rel.primal_solution.empty()) expect_near(rel.primal_solution[0], 3.0, 1e-4, "oracle solution");
    // the Halpern scheme through the same route
    auto ho = o;
    ho.b200.scheme = vikalp::B200Options::Scheme::Halpern;
    ho.b200.relative_tolerance = 1e-7;
    const auto h = vikalp::solve(row, ho);
    expect(h.status == vikalp::SolveStatus::Optimal, "Halpern scheme route");
    if (!h.primal_solution.empty()) expect_near(h.primal_solution[0], 3.0, 1e-5, "Halpern solution");
    // a bad override length is an InvalidModel result, not a crash
    const std::vector<double> two = {1.0, 2.0};
    expect(oracle.solve(row, two, {}, {}, po).status == vikalp::SolveStatus::InvalidModel, "override size check");
}

} // namespace

int main(int argc, char **argv) {
    const bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
    if (gpu)
        gpu_routes();
    else
        cpu_routes();
    if (failures) {
        std::cerr << failures << " checks failed\n";
        return 1;
    }
    std::cout << "ALL CHECKS PASSED (" << (gpu ? "gpu" : "cpu") << ")\n";
    return 0;
}
