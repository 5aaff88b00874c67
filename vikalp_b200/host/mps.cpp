// The MPS ingest path: vikalp::MpsReader (VIKALP src/io/MpsReader.cpp:10-559
// gives the format rules, messages and error order kept here) and a small C
// entry point so a file can go straight into vk_pdhg_create. Tokens are read
// with the same stream extraction as the reference, so malformed numbers,
// blank-looking lines and second entries are taken the same way; the matrix
// is assembled by sorting (row, variable) keys rather than by scanning every
// row against every variable.
#include "vikalp/io/MpsReader.hpp"
#include "vikalp_b200.h"

#include <algorithm>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <unordered_map>
#include <unordered_set>

namespace vikalp {

namespace {

enum class Section { None, Rows, Columns, Rhs, Bounds };

struct Entry {
    std::string variable, row;
    Scalar value;
};

struct Bound {
    std::string type, variable;
    Scalar value;
};

} // namespace

bool MpsReader::read(const std::string &path, Model &model) {
    errors_.clear();
    std::ifstream in(path);
    if (!in) {
        errors_.push_back({0, "unable to open MPS file: " + path});
        return false;
    }
    model = Model{};
    auto fail = [&](std::size_t line, std::string msg) { errors_.push_back({line, std::move(msg)}); };

    bool saw_name = false, saw_rows = false, saw_columns = false, saw_rhs = false, saw_end = false;
    Section sec = Section::None;
    std::string objective_row;
    std::vector<std::string> rows;
    std::vector<char> row_type;
    std::vector<std::string> first_seen; // variable names in order of appearance (repeats kept)
    std::vector<Entry> entries;
    std::map<std::string, Scalar> rhs;
    std::vector<Bound> bounds;

    std::string line;
    std::size_t ln = 0;
    while (std::getline(in, line)) {
        ++ln;
        if (line.empty()) continue;
        std::istringstream ss(line);
        std::string head;
        ss >> head;
        if (head == "NAME") {
            saw_name = true;
            ss >> model.name;
            sec = Section::None;
        } else if (head == "ROWS") {
            saw_rows = true;
            sec = Section::Rows;
        } else if (head == "COLUMNS") {
            saw_columns = true;
            sec = Section::Columns;
        } else if (head == "RHS") {
            saw_rhs = true;
            sec = Section::Rhs;
        } else if (head == "BOUNDS") {
            sec = Section::Bounds;
        } else if (head == "ENDATA") {
            saw_end = true;
            break;
        } else if (sec == Section::Rows) {
            std::string name;
            ss >> name;
            if (name.empty()) {
                fail(ln, "missing row name");
            } else if (head == "N") {
                objective_row = name;
            } else if (head == "L" || head == "G" || head == "E") {
                rows.push_back(name);
                row_type.push_back(head[0]);
            } else {
                fail(ln, "unsupported ROWS type '" + head + "'");
            }
        } else if (sec == Section::Columns) {
            std::string r;
            double v = 0.0;
            ss >> r >> v;
            if (head.empty() || r.empty() || ss.fail()) {
                fail(ln, "invalid COLUMNS entry");
                continue;
            }
            first_seen.push_back(head);
            entries.push_back({head, r, v});
            std::string r2;
            double v2 = 0.0;
            if (ss >> r2 >> v2) entries.push_back({head, r2, v2});
        } else if (sec == Section::Rhs) {
            std::string r;
            double v = 0.0;
            ss >> r >> v;
            if (head.empty() || r.empty() || ss.fail()) {
                fail(ln, "invalid RHS entry");
                continue;
            }
            rhs[r] = v;
            std::string r2;
            double v2 = 0.0;
            if (ss >> r2 >> v2) rhs[r2] = v2;
        } else if (sec == Section::Bounds) {
            std::string set, var;
            double v = 0.0;
            ss >> set >> var;
            if (head.empty() || set.empty() || var.empty()) {
                fail(ln, "invalid BOUNDS entry");
                continue;
            }
            if (head == "LO" || head == "UP" || head == "FX") {
                if (!(ss >> v)) {
                    fail(ln, "missing bound value");
                    continue;
                }
                bounds.push_back({head, var, v});
            } else if (head == "BV") {
                bounds.push_back({head, var, 1.0});
            } else if (head == "FR") {
                bounds.push_back({head, var, 0.0});
            } else {
                fail(ln, "unsupported BOUNDS type '" + head + "'");
            }
        }
    }
    if (!saw_name) fail(0, "missing NAME section");
    if (!saw_rows) fail(0, "missing ROWS section");
    if (!saw_columns) fail(0, "missing COLUMNS section");
    if (!saw_rhs) fail(0, "missing RHS section");
    if (!saw_end) fail(ln, "missing ENDATA section");
    if (!errors_.empty()) return false;

    // variables in order of first appearance
    std::unordered_map<std::string, Index> var;
    std::vector<std::string> names;
    for (const auto &v : first_seen)
        if (var.emplace(v, static_cast<Index>(names.size())).second) names.push_back(v);
    const Index n = static_cast<Index>(names.size()), m = static_cast<Index>(rows.size());
    std::unordered_map<std::string, Index> row;
    for (Index i = 0; i < m; ++i) row.emplace(rows[static_cast<std::size_t>(i)], i);

    model.linear_objective.assign(static_cast<std::size_t>(n), 0.0);
    model.variable_lower.assign(static_cast<std::size_t>(n), 0.0);
    model.variable_upper.assign(static_cast<std::size_t>(n), Model::infinity());
    model.variable_types.assign(static_cast<std::size_t>(n), VariableType::Continuous);
    model.constraint_lower.assign(static_cast<std::size_t>(m), -Model::infinity());
    model.constraint_upper.assign(static_cast<std::size_t>(m), Model::infinity());

    // (row, variable) -> value, the last entry winning
    std::vector<std::pair<std::pair<Index, Index>, std::pair<std::size_t, Scalar>>> coo;
    coo.reserve(entries.size());
    for (std::size_t k = 0; k < entries.size(); ++k) {
        const Entry &e = entries[k];
        const auto vi = var.find(e.variable);
        if (vi == var.end()) {
            fail(0, "unknown variable in COLUMNS: " + e.variable);
            continue;
        }
        if (e.row == objective_row) {
            model.linear_objective[static_cast<std::size_t>(vi->second)] = e.value;
            continue;
        }
        const auto ri = row.find(e.row);
        if (ri == row.end()) {
            fail(0, "unknown row in COLUMNS: " + e.row);
            continue;
        }
        coo.push_back({{ri->second, vi->second}, {k, e.value}});
    }
    if (!errors_.empty()) return false;

    for (Index i = 0; i < m; ++i) {
        const auto it = rhs.find(rows[static_cast<std::size_t>(i)]);
        const Scalar b = it == rhs.end() ? 0.0 : it->second;
        const auto u = static_cast<std::size_t>(i);
        switch (row_type[u]) {
        case 'L': model.constraint_upper[u] = b; break;
        case 'G': model.constraint_lower[u] = b; break;
        default: model.constraint_lower[u] = model.constraint_upper[u] = b; break;
        }
    }
    for (const Bound &b : bounds) {
        const auto vi = var.find(b.variable);
        if (vi == var.end()) {
            fail(0, "unknown variable in BOUNDS: " + b.variable);
            continue;
        }
        const auto j = static_cast<std::size_t>(vi->second);
        if (b.type == "LO") {
            model.variable_lower[j] = b.value;
        } else if (b.type == "UP") {
            model.variable_upper[j] = b.value;
        } else if (b.type == "FX") {
            model.variable_lower[j] = model.variable_upper[j] = b.value;
        } else if (b.type == "FR") {
            model.variable_lower[j] = -Model::infinity();
            model.variable_upper[j] = Model::infinity();
        } else { // BV
            model.variable_lower[j] = 0.0;
            model.variable_upper[j] = 1.0;
            model.variable_types[j] = VariableType::Binary;
        }
    }
    if (!errors_.empty()) return false;

    // CSR: sort by (row, variable), keep the last entry of each key
    std::stable_sort(coo.begin(), coo.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
    auto &A = model.constraint_matrix;
    A.pattern.rows = m;
    A.pattern.columns = n;
    A.pattern.row_offsets.assign(static_cast<std::size_t>(m) + 1, 0);
    A.pattern.column_indices.clear();
    A.values.clear();
    for (std::size_t k = 0; k < coo.size(); ++k) {
        if (k + 1 < coo.size() && coo[k + 1].first == coo[k].first) continue; // a later entry wins
        A.pattern.column_indices.push_back(coo[k].first.second);
        A.values.push_back(coo[k].second.second);
        ++A.pattern.row_offsets[static_cast<std::size_t>(coo[k].first.first) + 1];
    }
    for (Index i = 0; i < m; ++i)
        A.pattern.row_offsets[static_cast<std::size_t>(i) + 1] += A.pattern.row_offsets[static_cast<std::size_t>(i)];
    return model.validate().empty();
}

const std::vector<MpsError> &MpsReader::errors() const noexcept { return errors_; }

} // namespace vikalp

// ---- C entry points (vk_mps_*, include/vikalp_mps.h) -------------------------

struct vk_mps {
    vikalp::Model model;
    std::vector<vikalp::MpsError> errors;
    bool ok = false;
};

extern "C" {

int vk_mps_read(const char *path, vk_mps **out) {
    if (!path || !out) return VK_ERR_INVALID;
    try {
        auto h = std::make_unique<vk_mps>();
        vikalp::MpsReader reader;
        h->ok = reader.read(path, h->model);
        h->errors = reader.errors(); // empty when only Model::validate() failed, as in the reference
        const int rc = h->ok ? VK_OK : VK_ERR_INVALID;
        *out = h.release();
        return rc;
    } catch (...) {
        return VK_ERR_INTERNAL;
    }
}

int vk_mps_problem(const vk_mps *h, vk_problem *p, int64_t *m, int64_t *n, int64_t *nnz) {
    if (!h || !p) return VK_ERR_INVALID;
    const vikalp::Model &md = h->model;
    std::memset(p, 0, sizeof(*p));
    const auto &A = md.constraint_matrix;
    p->A = vk_csr{A.pattern.rows, A.pattern.columns, A.pattern.row_offsets.data(), A.pattern.column_indices.data(),
                  A.values.data()};
    static const int64_t zero = 0;
    p->Q = vk_csr{0, 0, &zero, nullptr, nullptr};
    p->c = md.linear_objective.data();
    p->objective_offset = md.objective_offset;
    p->var_lower = md.variable_lower.data();
    p->var_upper = md.variable_upper.data();
    p->row_lower = md.constraint_lower.data();
    p->row_upper = md.constraint_upper.data();
    if (m) *m = A.pattern.rows;
    if (n) *n = A.pattern.columns;
    if (nnz) *nnz = static_cast<int64_t>(A.pattern.column_indices.size());
    return VK_OK;
}

const char *vk_mps_name(const vk_mps *h) { return h ? h->model.name.c_str() : ""; }

int32_t vk_mps_binary_count(const vk_mps *h) {
    if (!h) return 0;
    return static_cast<int32_t>(std::count(h->model.variable_types.begin(), h->model.variable_types.end(),
                                           vikalp::VariableType::Binary));
}

int32_t vk_mps_error_count(const vk_mps *h) { return h ? static_cast<int32_t>(h->errors.size()) : 0; }

const char *vk_mps_error(const vk_mps *h, int32_t i, int64_t *line) {
    if (!h || i < 0 || i >= static_cast<int32_t>(h->errors.size())) return nullptr;
    if (line) *line = static_cast<int64_t>(h->errors[static_cast<std::size_t>(i)].line);
    return h->errors[static_cast<std::size_t>(i)].message.c_str();
}

void vk_mps_free(vk_mps *h) { delete h; }

} // extern "C"
