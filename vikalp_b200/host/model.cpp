// vikalp::Model methods: sizes, problem class and validation with the rules
// and messages of the reference (src/contracts/Model.cpp:13-199), so callers
// see the same InvalidModel messages on this path.
#include "vikalp/contracts/Model.hpp"
#include "vikalp/contracts/NonlinearOracle.hpp"

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

namespace vikalp {
namespace {

bool check_pattern(const CsrPattern &p, const std::string &name, std::vector<std::string> &errors) {
    if (p.rows < 0 || p.columns < 0) {
        errors.push_back(name + " dimensions must be non-negative");
        return false;
    }
    if (p.row_offsets.size() != static_cast<std::size_t>(p.rows + 1)) {
        errors.push_back(name + " row_offsets must contain rows + 1 entries");
        return false;
    }
    const auto nnz = static_cast<Index>(p.column_indices.size());
    if (p.row_offsets.empty() || p.row_offsets.front() != 0 || p.row_offsets.back() != nnz) {
        errors.push_back(name + " row_offsets do not describe column_indices");
        return false;
    }
    for (Index r = 0; r < p.rows; ++r) {
        const Index b = p.row_offsets[static_cast<std::size_t>(r)];
        const Index e = p.row_offsets[static_cast<std::size_t>(r + 1)];
        if (b < 0 || b > e || e > nnz) {
            errors.push_back(name + " row_offsets must be ordered and in range");
            return false;
        }
        Index prev = -1;
        for (Index k = b; k < e; ++k) {
            const Index c = p.column_indices[static_cast<std::size_t>(k)];
            if (c < 0 || c >= p.columns) {
                errors.push_back(name + " contains an out-of-range column");
                return false;
            }
            if (c <= prev) {
                errors.push_back(name + " columns must be strictly ordered per row");
                return false;
            }
            prev = c;
        }
    }
    return true;
}

bool check_matrix(const CsrMatrix &m, const std::string &name, std::vector<std::string> &errors) {
    bool ok = check_pattern(m.pattern, name, errors);
    if (m.values.size() != m.pattern.column_indices.size()) {
        errors.push_back(name + " values and column_indices sizes differ");
        ok = false;
    }
    if (std::any_of(m.values.begin(), m.values.end(), [](Scalar v) { return !std::isfinite(v); })) {
        errors.push_back(name + " coefficients must be finite");
        ok = false;
    }
    return ok;
}

void check_bounds(const std::vector<Scalar> &lo, const std::vector<Scalar> &hi, const std::string &name,
                  std::vector<std::string> &errors) {
    if (lo.size() != hi.size()) {
        errors.push_back(name + " lower and upper sizes differ");
        return;
    }
    for (std::size_t i = 0; i < lo.size(); ++i)
        if (std::isnan(lo[i]) || std::isnan(hi[i]) || lo[i] > hi[i])
            errors.push_back(name + " contains an invalid bound at index " + std::to_string(i));
}

} // namespace

Index Model::num_variables() const noexcept { return static_cast<Index>(linear_objective.size()); }

Index Model::num_constraints() const noexcept { return static_cast<Index>(constraint_lower.size()); }

bool Model::has_quadratic_objective() const noexcept { return !quadratic_objective.values.empty(); }

bool Model::has_integer_variables() const noexcept {
    return std::any_of(variable_types.begin(), variable_types.end(),
                       [](VariableType t) { return t != VariableType::Continuous; });
}

ProblemClass Model::problem_class() const noexcept {
    const bool integer = has_integer_variables();
    if (nonlinear) return integer ? ProblemClass::MINLP : ProblemClass::NLP;
    if (has_quadratic_objective()) return integer ? ProblemClass::MIQP : ProblemClass::QP;
    return integer ? ProblemClass::MILP : ProblemClass::LP;
}

std::vector<std::string> Model::validate() const {
    std::vector<std::string> errors;
    const Index n = num_variables(), m = num_constraints();
    if (!std::isfinite(objective_offset) ||
        std::any_of(linear_objective.begin(), linear_objective.end(), [](Scalar v) { return !std::isfinite(v); }))
        errors.push_back("objective coefficients must be finite");
    if (constraint_upper.size() != constraint_lower.size())
        errors.push_back("constraint lower and upper sizes differ");
    if (variable_lower.size() != static_cast<std::size_t>(n) || variable_upper.size() != static_cast<std::size_t>(n) ||
        variable_types.size() != static_cast<std::size_t>(n))
        errors.push_back("variable metadata sizes must equal the objective size");
    check_bounds(constraint_lower, constraint_upper, "constraint bounds", errors);
    check_bounds(variable_lower, variable_upper, "variable bounds", errors);
    check_matrix(constraint_matrix, "constraint matrix", errors);
    if (constraint_matrix.pattern.rows != m || constraint_matrix.pattern.columns != n)
        errors.push_back("constraint matrix dimensions do not match the model");
    const auto &q = quadratic_objective;
    const bool q_absent = q.pattern.rows == 0 && q.pattern.columns == 0 && q.pattern.column_indices.empty() &&
                          q.values.empty();
    const bool q_ok = check_matrix(q, "quadratic objective", errors);
    const bool q_square = q.pattern.rows == n && q.pattern.columns == n;
    if (!q_absent && !q_square) errors.push_back("quadratic objective must be square and match the variables");
    if (!q_absent && q_ok && q_square) {
        // every entry must have an equal mirror (1e-12 relative)
        for (Index r = 0; r < n; ++r) {
            bool bad = false;
            for (Index k = q.pattern.row_offsets[static_cast<std::size_t>(r)];
                 k < q.pattern.row_offsets[static_cast<std::size_t>(r + 1)]; ++k) {
                const Index c = q.pattern.column_indices[static_cast<std::size_t>(k)];
                const auto b = q.pattern.column_indices.begin() + q.pattern.row_offsets[static_cast<std::size_t>(c)];
                const auto e = q.pattern.column_indices.begin() + q.pattern.row_offsets[static_cast<std::size_t>(c + 1)];
                const auto it = std::lower_bound(b, e, r);
                const Scalar v = q.values[static_cast<std::size_t>(k)];
                if (it == e || *it != r) {
                    bad = true;
                    break;
                }
                const Scalar w = q.values[static_cast<std::size_t>(it - q.pattern.column_indices.begin())];
                if (std::abs(v - w) > 1e-12 * std::max({1.0, std::abs(v), std::abs(w)})) {
                    bad = true;
                    break;
                }
            }
            if (bad) {
                errors.push_back("quadratic objective must be stored symmetrically");
                break;
            }
        }
    }
    if (nonlinear) {
        if (nonlinear->variables() != n || nonlinear->constraints() != m)
            errors.push_back("nonlinear oracle dimensions do not match the model");
        const auto &j = nonlinear->jacobian_pattern();
        check_pattern(j, "nonlinear Jacobian", errors);
        if (j.rows != m || j.columns != n) errors.push_back("nonlinear Jacobian dimensions do not match the model");
        const auto &h = nonlinear->hessian_pattern();
        check_pattern(h, "nonlinear Hessian", errors);
        if (h.rows != n || h.columns != n) errors.push_back("nonlinear Hessian dimensions do not match the model");
    }
    return errors;
}

} // namespace vikalp
