// make_cuda_backend(): the ExecutionBackend contract on the B200, checked the
// way the reference checks its backends (tests/test_backend.cpp known answers,
// tests/test_cuda_consistency.cpp's GPU-vs-CPU agreement): expect counters,
// exit code 0 or 1. The CPU side of the consistency checks is a plain loop in
// this file with the CPU backend's arithmetic (src/backend/cpu_ops.cpp).
//
//   test_backend gpu   every check (needs a GPU)
#include "vikalp/backend/CudaBackend.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <iostream>
#include <limits>
#include <random>
#include <stdexcept>
#include <vector>

using namespace vikalp;

namespace {

int failures = 0;

void expect(bool c, const char *what) {
    if (!c) {
        std::cerr << "FAIL: " << what << '\n';
        ++failures;
    }
}

bool same(const std::vector<double> &a, const std::vector<double> &b) {
    if (a.size() != b.size()) return false;
    for (std::size_t i = 0; i < a.size(); ++i)
        if (!(a[i] == b[i] || (std::isnan(a[i]) && std::isnan(b[i])))) return false;
    return true;
}

double max_diff(const std::vector<double> &a, const std::vector<double> &b) {
    double d = 0.0;
    for (std::size_t i = 0; i < a.size(); ++i) d = std::max(d, std::abs(a[i] - b[i]));
    return d;
}

template <class F>
bool throws_invalid(F &&f) {
    try {
        f();
    } catch (const std::invalid_argument &) {
        return true;
    } catch (...) {
        return false;
    }
    return false;
}

std::vector<double> get(ExecutionBackend &be, const BackendVector &v) {
    std::vector<double> h(static_cast<std::size_t>(v.size()));
    be.download(v, h);
    return h;
}

std::unique_ptr<BackendVector> put(ExecutionBackend &be, const std::vector<double> &h) {
    auto v = be.create_vector(static_cast<Index>(h.size()));
    be.upload(h, *v);
    return v;
}

// A = [1 2 0; 0 3 4]
CsrPattern small_pattern() { return CsrPattern{2, 3, {0, 2, 4}, {0, 1, 1, 2}}; }
const std::vector<double> small_values = {1.0, 2.0, 3.0, 4.0};

// CPU-backend arithmetic: y = alpha A x + beta y, rows left to right; the
// transpose scales y by beta, then scatters v * (alpha x_row) in row order.
void cpu_multiply(const CsrPattern &p, const std::vector<double> &v, double alpha, const std::vector<double> &x,
                  double beta, std::vector<double> &y, bool transpose) {
    if (!transpose) {
        for (Index r = 0; r < p.rows; ++r) {
            double acc = 0.0;
            for (Index k = p.row_offsets[r]; k < p.row_offsets[r + 1]; ++k) acc += v[k] * x[p.column_indices[k]];
            y[r] = alpha * acc + beta * y[r];
        }
    } else {
        for (auto &e : y) e *= beta;
        for (Index r = 0; r < p.rows; ++r) {
            const double sx = alpha * x[r];
            for (Index k = p.row_offsets[r]; k < p.row_offsets[r + 1]; ++k) y[p.column_indices[k]] += v[k] * sx;
        }
    }
}

void known_answers(ExecutionBackend &be) {
    auto A = be.create_matrix(small_pattern());
    expect(A->rows() == 2 && A->columns() == 3, "matrix dimensions");
    be.set_values(small_values, *A);
    auto x = put(be, {2.0, 1.0, 3.0});
    auto y = be.create_vector(2);
    be.multiply(1.0, *A, *x, 0.0, *y, Transpose::No);
    expect(same(get(be, *y), {4.0, 15.0}), "A x = [4, 15]");
    auto yt = be.create_vector(3);
    auto w = put(be, {2.0, 1.0});
    be.multiply(1.0, *A, *w, 0.0, *yt, Transpose::Yes);
    expect(same(get(be, *yt), {2.0, 7.0, 4.0}), "A' [2, 1] = [2, 7, 4]");
    // alpha / beta
    auto y2 = put(be, {1.0, -1.0});
    be.multiply(2.0, *A, *x, 0.5, *y2, Transpose::No);
    expect(same(get(be, *y2), {8.5, 29.5}), "2 A x + 0.5 y");
    auto y3 = put(be, {1.0, 1.0, 1.0});
    be.multiply(-1.0, *A, *w, 3.0, *y3, Transpose::Yes);
    expect(same(get(be, *y3), {1.0, -4.0, -1.0}), "-A' w + 3 y");
    // zero x
    auto z = be.create_vector(3);
    auto y4 = put(be, {5.0, 6.0});
    be.multiply(1.0, *A, *z, 0.0, *y4, Transpose::No);
    expect(same(get(be, *y4), {0.0, 0.0}), "A 0 = 0");
    // 1x1
    auto B = be.create_matrix(CsrPattern{1, 1, {0, 1}, {0}});
    be.set_values(std::vector<double>{-3.0}, *B);
    auto b1 = put(be, {2.0});
    auto o1 = be.create_vector(1);
    be.multiply(1.0, *B, *b1, 0.0, *o1, Transpose::No);
    expect(same(get(be, *o1), {-6.0}), "1x1 product");
    // an empty row
    auto E = be.create_matrix(CsrPattern{3, 2, {0, 1, 1, 2}, {0, 1}});
    be.set_values(std::vector<double>{2.0, 5.0}, *E);
    auto ex = put(be, {1.0, 1.0});
    auto ey = put(be, {9.0, 9.0, 9.0});
    be.multiply(1.0, *E, *ex, 0.0, *ey, Transpose::No);
    expect(same(get(be, *ey), {2.0, 0.0, 5.0}), "empty row gives 0");
}

void vector_ops(ExecutionBackend &be) {
    auto v = be.create_vector(4);
    expect(v->size() == 4, "size");
    expect(same(get(be, *v), {0.0, 0.0, 0.0, 0.0}), "new vector is zero");
    be.fill(*v, 2.5);
    expect(same(get(be, *v), {2.5, 2.5, 2.5, 2.5}), "fill");
    auto a = put(be, {1.0, -2.0, 3.0, 0.1});
    auto c = be.create_vector(4);
    be.copy(*a, *c);
    expect(same(get(be, *c), {1.0, -2.0, 3.0, 0.1}), "copy");
    be.axpby(0.3, *a, -1.7, *c);
    std::vector<double> want = {1.0, -2.0, 3.0, 0.1}, av = want;
    for (std::size_t i = 0; i < 4; ++i) want[i] = 0.3 * av[i] + -1.7 * want[i];
    expect(same(get(be, *c), want), "axpby bit-identical to the CPU loop");
    expect(be.dot(*a, *a) == 1.0 + 4.0 + 9.0 + 0.1 * 0.1, "dot");
    auto n = put(be, {1.0, -7.0, std::numeric_limits<double>::quiet_NaN(), 3.0});
    expect(be.norm_inf(*n) == 7.0, "norm_inf ignores NaN");
    auto e = be.create_vector(0);
    expect(be.norm_inf(*e) == 0.0 && be.dot(*e, *e) == 0.0, "empty reductions are 0");
    auto x = put(be, {-5.0, 0.5, 5.0, std::numeric_limits<double>::quiet_NaN()});
    auto lo = put(be, {-1.0, -1.0, -1.0, -1.0});
    auto hi = put(be, {1.0, 1.0, 1.0, 1.0});
    be.project_box(*x, *lo, *hi);
    const auto px = get(be, *x);
    expect(px[0] == -1.0 && px[1] == 0.5 && px[2] == 1.0 && std::isnan(px[3]), "project_box (NaN passes)");
    be.synchronize();
}

void dimension_errors(ExecutionBackend &be) {
    auto A = be.create_matrix(small_pattern());
    auto v2 = be.create_vector(2), v3 = be.create_vector(3);
    expect(throws_invalid([&] { be.upload(std::vector<double>{1.0}, *v2); }), "upload size");
    expect(throws_invalid([&] {
               std::vector<double> h(5);
               be.download(*v2, h);
           }),
           "download size");
    expect(throws_invalid([&] { be.copy(*v2, *v3); }), "copy size");
    expect(throws_invalid([&] { be.axpby(1.0, *v2, 1.0, *v3); }), "axpby size");
    expect(throws_invalid([&] { (void)be.dot(*v2, *v3); }), "dot size");
    expect(throws_invalid([&] { be.project_box(*v2, *v3, *v2); }), "project_box size");
    expect(throws_invalid([&] { be.multiply(1.0, *A, *v2, 0.0, *v2, Transpose::No); }), "multiply x size");
    expect(throws_invalid([&] { be.multiply(1.0, *A, *v3, 0.0, *v3, Transpose::No); }), "multiply y size");
    expect(throws_invalid([&] { be.multiply(1.0, *A, *v3, 0.0, *v3, Transpose::Yes); }), "multiply T x size");
    expect(throws_invalid([&] { be.set_values(std::vector<double>{1.0, 2.0}, *A); }), "set_values size");
    expect(throws_invalid([&] { (void)be.create_vector(-1); }), "negative size");
    expect(throws_invalid([&] { (void)be.create_matrix(CsrPattern{2, 3, {0, 2, 1}, {0, 1}}); }), "bad pattern");
    expect(throws_invalid([&] { (void)be.create_matrix(CsrPattern{1, 3, {0, 2}, {2, 1}}); }), "unsorted columns");
    auto b = be.create_vector(2), s = be.create_vector(2);
    expect(throws_invalid([&] { (void)be.solve_linear_system(*A, *b, *s, MatrixProperty::General, 1e-9, 10); }),
           "solve needs a square matrix");
}

// tests/test_cuda_consistency.cpp: the GPU against the CPU backend's
// arithmetic on a random matrix, within 1e-10 (FAST) or bit for bit (SEQUENTIAL).
void consistency(ExecutionBackend &be, bool exact) {
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    const Index m = 300, n = 500;
    CsrPattern p{m, n, {0}, {}};
    std::vector<double> vals;
    for (Index r = 0; r < m; ++r) {
        const int len = static_cast<int>(rng() % 40);
        std::vector<Index> cols;
        for (int k = 0; k < len; ++k) cols.push_back(static_cast<Index>(rng() % n));
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        for (Index c : cols) {
            p.column_indices.push_back(c);
            vals.push_back(U(rng));
        }
        p.row_offsets.push_back(static_cast<Index>(p.column_indices.size()));
    }
    auto A = be.create_matrix(p);
    be.set_values(vals, *A);
    std::vector<double> x(n), y(m), xt(m), yt(n);
    for (auto &e : x) e = U(rng);
    for (auto &e : y) e = U(rng);
    for (auto &e : xt) e = U(rng);
    for (auto &e : yt) e = U(rng);
    auto dx = put(be, x), dy = put(be, y), dxt = put(be, xt), dyt = put(be, yt);
    be.multiply(0.75, *A, *dx, -1.25, *dy, Transpose::No);
    be.multiply(-0.5, *A, *dxt, 2.0, *dyt, Transpose::Yes);
    cpu_multiply(p, vals, 0.75, x, -1.25, y, false);
    cpu_multiply(p, vals, -0.5, xt, 2.0, yt, true);
    if (exact) {
        expect(same(get(be, *dy), y), "sequential A x bit-identical to the CPU backend");
        expect(same(get(be, *dyt), yt), "sequential A'x bit-identical to the CPU backend");
    } else {
        expect(max_diff(get(be, *dy), y) <= 1e-10, "fast A x within 1e-10 of the CPU backend");
        expect(max_diff(get(be, *dyt), yt) <= 1e-10, "fast A'x within 1e-10 of the CPU backend");
    }
    double d = 0.0;
    for (Index i = 0; i < n; ++i) d += x[i] * yt[i];
    expect(std::abs(be.dot(*dx, *dyt) - d) <= 1e-10 * (1.0 + std::abs(d)), "dot within 1e-10");
}

void linear_solve(ExecutionBackend &be) {
    // diagonally dominant tridiagonal system, n = 200
    const Index n = 200;
    CsrPattern p{n, n, {0}, {}};
    std::vector<double> vals;
    for (Index i = 0; i < n; ++i) {
        for (Index j = std::max<Index>(0, i - 1); j <= std::min<Index>(n - 1, i + 1); ++j) {
            p.column_indices.push_back(j);
            vals.push_back(i == j ? 4.0 + 0.01 * i : (j < i ? -1.0 : -0.5));
        }
        p.row_offsets.push_back(static_cast<Index>(p.column_indices.size()));
    }
    auto A = be.create_matrix(p);
    be.set_values(vals, *A);
    std::vector<double> xs(n);
    for (Index i = 0; i < n; ++i) xs[i] = std::sin(0.1 * i);
    std::vector<double> b(n, 0.0);
    cpu_multiply(p, vals, 1.0, xs, 0.0, b, false);
    auto db = put(be, b), sol = be.create_vector(n);
    const auto r = be.solve_linear_system(*A, *db, *sol, MatrixProperty::General, 1e-11, 500);
    expect(r.converged && r.iterations > 0 && r.residual <= 1e-11, "BiCGSTAB converges");
    expect(max_diff(get(be, *sol), xs) <= 1e-9, "BiCGSTAB solution");
    // zero right-hand side: converged before the first iteration
    auto zb = be.create_vector(n);
    const auto r0 = be.solve_linear_system(*A, *zb, *sol, MatrixProperty::General, 1e-12, 50);
    expect(r0.converged && r0.iterations == 0 && r0.residual == 0.0, "zero rhs");
    // breakdown: A = [0], b = [1] -> r_hat'v = 0 in the first iteration
    auto Z = be.create_matrix(CsrPattern{1, 1, {0, 1}, {0}});
    be.set_values(std::vector<double>{0.0}, *Z);
    auto one = put(be, {1.0}), s1 = be.create_vector(1);
    const auto rb = be.solve_linear_system(*Z, *one, *s1, MatrixProperty::General, 1e-12, 20);
    expect(!rb.converged && rb.iterations == 1 && rb.residual == 1.0, "breakdown reported, residual |b|");
    expect(throws_invalid([&] { (void)be.solve_linear_system(*A, *db, *sol, MatrixProperty::General, -1.0, 5); }),
           "negative tolerance");
}

} // namespace

int main(int argc, char **argv) {
    if (argc < 2 || std::strcmp(argv[1], "gpu") != 0) {
        std::cerr << "usage: test_backend gpu\n";
        return 2;
    }
    for (const bool exact : {false, true}) {
        auto be = make_cuda_backend(exact ? CudaProductOrder::Sequential : CudaProductOrder::Fast);
        known_answers(*be);
        vector_ops(*be);
        dimension_errors(*be);
        consistency(*be, exact);
        linear_solve(*be);
    }
    if (failures == 0) std::cout << "ALL CHECKS PASSED\n";
    return failures == 0 ? 0 : 1;
}
