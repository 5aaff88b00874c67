// Positive-semidefiniteness gate for large Q.
//
// The reference rejects a non-convex QP with a dense Cholesky test
// (continuous_common.hpp:242-275, called at pdqp.cpp:318). That needs an n x n
// dense copy, so the library uses it only up to a few thousand variables;
// above that this file estimates the smallest eigenvalue of the sparse Q with
// a Lanczos run (no reorthogonalisation; its Ritz values stay inside Q's
// spectrum) and rejects Q when that estimate is clearly negative relative to
// the largest one.
#include "vikalp_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>

namespace vk {

namespace {

void spmv(const vk_csr &q, const std::vector<double> &x, std::vector<double> &y) {
    for (int64_t r = 0; r < q.rows; ++r) {
        double s = 0.0;
        for (int64_t k = q.row_offsets[r]; k < q.row_offsets[r + 1]; ++k) s += q.values[k] * x[q.col_indices[k]];
        y[r] = s;
    }
}

// Extreme eigenvalues of the symmetric tridiagonal matrix (alpha, beta) by
// bisection on the Sturm sequence.
double tridiag_eig(const std::vector<double> &a, const std::vector<double> &b, bool smallest) {
    const int k = static_cast<int>(a.size());
    double lo = 0.0, hi = 0.0;
    for (int i = 0; i < k; ++i) {
        const double r = (i > 0 ? std::abs(b[i - 1]) : 0.0) + (i + 1 < k ? std::abs(b[i]) : 0.0);
        lo = std::min(lo, a[i] - r);
        hi = std::max(hi, a[i] + r);
    }
    auto count_below = [&](double x) {
        int c = 0;
        double d = 1.0;
        for (int i = 0; i < k; ++i) {
            d = a[i] - x - (i > 0 ? b[i - 1] * b[i - 1] / d : 0.0);
            if (d == 0.0) d = 1e-300;
            if (d < 0.0) ++c;
        }
        return c;
    };
    const int target = smallest ? 1 : k;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (count_below(mid) >= target)
            hi = mid;
        else
            lo = mid;
    }
    return 0.5 * (lo + hi);
}

} // namespace

bool psd_check_large(const vk_csr &q) {
    const int64_t n = q.rows;
    // Quick accept: symmetric, non-negative diagonal, diagonally dominant.
    bool dominant = true;
    for (int64_t r = 0; r < n && dominant; ++r) {
        double diag = 0.0, off = 0.0;
        for (int64_t k = q.row_offsets[r]; k < q.row_offsets[r + 1]; ++k) {
            if (q.col_indices[k] == r) diag = q.values[k];
            else off += std::abs(q.values[k]);
        }
        if (diag < 0.0 || diag < off) dominant = false;
    }
    if (dominant) return true;
    const int steps = static_cast<int>(std::min<int64_t>(n, 80));
    std::vector<double> v(n), w(n), vprev(n, 0.0);
    std::mt19937_64 rng(0x5eedULL);
    std::normal_distribution<double> nd;
    double nrm = 0.0;
    for (auto &e : v) {
        e = nd(rng);
        nrm += e * e;
    }
    nrm = std::sqrt(nrm);
    for (auto &e : v) e /= nrm;
    std::vector<double> alpha, beta;
    double bprev = 0.0;
    for (int it = 0; it < steps; ++it) {
        spmv(q, v, w);
        double a = 0.0;
        for (int64_t i = 0; i < n; ++i) a += w[i] * v[i];
        for (int64_t i = 0; i < n; ++i) w[i] -= a * v[i] + bprev * vprev[i];
        double b = 0.0;
        for (int64_t i = 0; i < n; ++i) b += w[i] * w[i];
        b = std::sqrt(b);
        alpha.push_back(a);
        if (b < 1e-12 || it + 1 == steps) break;
        beta.push_back(b);
        vprev.swap(v);
        for (int64_t i = 0; i < n; ++i) v[i] = w[i] / b;
        bprev = b;
    }
    beta.resize(alpha.size() > 0 ? alpha.size() - 1 : 0);
    const double lmin = tridiag_eig(alpha, beta, true);
    const double lmax = tridiag_eig(alpha, beta, false);
    return lmin >= -1e-8 * std::max(1.0, std::abs(lmax));
}

} // namespace vk
