/*
 * CPU oracle for the PDHG LP / PDQP hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker the parity tests, smoke() and the bench's CPU
 * baseline leg compare the CUDA library against. The product (libvikalp_b200)
 * never links, loads or calls it.
 *
 * It restates, in plain C99 FP64, the reference's algorithm for this path in
 * the reference's exact floating-point operation order, so that its iterates
 * equal the reference's bit for bit on x86-64 (no FMA contraction: build with
 * -ffp-contract=off). Each function names the reference lines it follows
 * (paths inside the VIKALP project). Parity of this restatement is pinned
 * against the reference itself (compiled from its own sources by
 * oracle/Makefile into oracle/_ref/) and against the reference's own
 * known-answer tests (tests/golden/).
 *
 * Functions with no reference counterpart (CSR transpose, relative KKT) say so.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "pdhg_oracle.h"

/* std::max(a, b) == (a < b) ? b : a ; std::min(a, b) == (b < a) ? b : a */
static double smax(double a, double b) { return (a < b) ? b : a; }
static double smin(double a, double b) { return (b < a) ? b : a; }
/* x = std::min(std::max(x, lo), hi)  -- cpu_ops.cpp:382 (NaN passes through) */
static double clampbox(double x, double lo, double hi) { return smin(smax(x, lo), hi); }
/* std::clamp(v, lo, hi) -- pdhg.cpp:206-208 */
static double sclamp(double v, double lo, double hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

/* y = alpha*A*x + beta*y, row-sequential -- cpu_ops.cpp:418-427 */
void or_spmv(int64_t m, const int64_t *ro, const int64_t *ci, const double *v, double alpha,
             const double *x, double beta, double *y) {
    for (int64_t r = 0; r < m; ++r) {
        double acc = 0.0;
        for (int64_t k = ro[r]; k < ro[r + 1]; ++k) acc += v[k] * x[ci[k]];
        y[r] = alpha * acc + beta * y[r];
    }
}

/* y = alpha*A'*x + beta*y, row-order scatter -- cpu_ops.cpp:444-458 */
void or_spmv_t(int64_t m, int64_t n, const int64_t *ro, const int64_t *ci, const double *v,
               double alpha, const double *x, double beta, double *y) {
    for (int64_t j = 0; j < n; ++j) y[j] *= beta;
    for (int64_t r = 0; r < m; ++r) {
        const double sx = alpha * x[r];
        for (int64_t k = ro[r]; k < ro[r + 1]; ++k) y[ci[k]] += v[k] * sx;
    }
}

/*
 * CSR transpose by a stable counting sort on the column index (no reference
 * counterpart; it makes explicit the order the reference's transposed product
 * accumulates in, cpu_ops.cpp:449-458: within each column, rows ascend).
 * perm[t] = position in the original CSR of transposed entry t.
 */
void or_csr_transpose(int64_t m, int64_t n, const int64_t *ro, const int64_t *ci, const double *v,
                      int64_t *tro, int64_t *trow, double *tv, int64_t *perm) {
    memset(tro, 0, sizeof(int64_t) * (size_t)(n + 1));
    const int64_t nnz = ro[m];
    for (int64_t k = 0; k < nnz; ++k) tro[ci[k] + 1]++;
    for (int64_t j = 0; j < n; ++j) tro[j + 1] += tro[j];
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    for (int64_t j = 0; j < n; ++j) fill[j] = tro[j];
    for (int64_t r = 0; r < m; ++r) {
        for (int64_t k = ro[r]; k < ro[r + 1]; ++k) {
            const int64_t t = fill[ci[k]]++;
            trow[t] = r;
            if (tv) tv[t] = v[k];
            if (perm) perm[t] = k;
        }
    }
    free(fill);
}

/*
 * Single-pass infinity-norm equilibration -- continuous_common.hpp:133-205.
 * Rows and columns are scaled only where their max |a| exceeds 1. The column
 * max is taken over the ORIGINAL values, as the reference does; max is
 * order-independent, so walking the columns through a transposed index gives
 * the same factors as the reference's O(n*nnz) scan.
 */
void or_scale(const or_problem *p, const double *lower, const double *upper, or_scaled *s) {
    const int64_t m = p->m, n = p->n;
    for (int64_t r = 0; r < m; ++r) {
        double mx = 0.0;
        for (int64_t k = p->ro[r]; k < p->ro[r + 1]; ++k) mx = smax(mx, fabs(p->v[k]));
        s->row_scale[r] = (mx > 1.0) ? 1.0 / mx : 1.0;
    }
    double *colmax = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    for (int64_t r = 0; r < m; ++r)
        for (int64_t k = p->ro[r]; k < p->ro[r + 1]; ++k)
            colmax[p->ci[k]] = smax(colmax[p->ci[k]], fabs(p->v[k]));
    for (int64_t j = 0; j < n; ++j) s->col_scale[j] = (colmax[j] > 1.0) ? 1.0 / colmax[j] : 1.0;
    free(colmax);
    for (int64_t r = 0; r < m; ++r)
        for (int64_t k = p->ro[r]; k < p->ro[r + 1]; ++k)
            s->v[k] = p->v[k] * (s->row_scale[r] * s->col_scale[p->ci[k]]);
    for (int64_t j = 0; j < n; ++j) {
        const double sc = s->col_scale[j];
        s->c[j] = p->c[j] * sc;
        s->l[j] = isfinite(lower[j]) ? lower[j] / sc : lower[j];
        s->u[j] = isfinite(upper[j]) ? upper[j] / sc : upper[j];
    }
    for (int64_t r = 0; r < m; ++r) {
        const double sc = s->row_scale[r];
        s->rl[r] = isfinite(p->rl[r]) ? p->rl[r] * sc : p->rl[r];
        s->ru[r] = isfinite(p->ru[r]) ? p->ru[r] * sc : p->ru[r];
    }
}

/* sqrt(max row abs-sum * max column abs-sum) -- continuous_common.hpp:207-225 */
double or_operator_bound(int64_t m, int64_t n, const int64_t *ro, const int64_t *ci, const double *v) {
    double max_row = 0.0;
    double *cols = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    for (int64_t r = 0; r < m; ++r) {
        double rs = 0.0;
        for (int64_t k = ro[r]; k < ro[r + 1]; ++k) {
            rs += fabs(v[k]);
            cols[ci[k]] += fabs(v[k]);
        }
        max_row = smax(max_row, rs);
    }
    double max_col = 0.0;
    for (int64_t j = 0; j < n; ++j) max_col = smax(max_col, cols[j]);
    free(cols);
    return sqrt(max_row * max_col);
}

static double norm_inf(const double *a, int64_t n) {
    double r = 0.0;
    for (int64_t i = 0; i < n; ++i) r = smax(r, fabs(a[i]));
    return r;
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/*
 * box_violation -- continuous_common.hpp:317-326
 */
static double box_violation(const double *val, const double *lo, const double *hi, int64_t k) {
    double r = 0.0;
    for (int64_t i = 0; i < k; ++i) {
        if (isfinite(lo[i])) r = smax(r, lo[i] - val[i]);
        if (isfinite(hi[i])) r = smax(r, val[i] - hi[i]);
    }
    return smax(0.0, r);
}

/*
 * Restarted PDHG (LP) or PDQP (when p->q_nnz > 0), in the reference's exact
 * operation order:
 *   scaling            pdhg.cpp:25 / pdqp.cpp:25,35-45
 *   step size          pdhg.cpp:75-78 / pdqp.cpp:89-99
 *   iteration          pdhg.cpp:87-151 / pdqp.cpp:110-178
 *   post-processing    pdhg.cpp:153-264 / pdqp.cpp:180-297
 * Returns 0, or -1 on an invalid warm start (pdhg.cpp:29-33).
 * The caller has already validated the model and bounds (pdhg.cpp:274-291).
 */
int or_pdhg_solve(const or_problem *p, const or_options *o, const double *warm, const double *lower,
                  const double *upper, or_result *res) {
    const double t0 = now_s();
    const int64_t m = p->m, n = p->n;
    const int qp = p->q_nnz > 0;
    if (warm) {
        for (int64_t j = 0; j < n; ++j)
            if (!isfinite(warm[j])) return -1;
    }
    or_scaled s;
    s.v = (double *)malloc(sizeof(double) * (size_t)(p->ro[m] > 0 ? p->ro[m] : 1));
    s.c = (double *)malloc(sizeof(double) * (size_t)(n + 1));
    s.l = (double *)malloc(sizeof(double) * (size_t)(n + 1));
    s.u = (double *)malloc(sizeof(double) * (size_t)(n + 1));
    s.col_scale = (double *)malloc(sizeof(double) * (size_t)(n + 1));
    s.rl = (double *)malloc(sizeof(double) * (size_t)(m + 1));
    s.ru = (double *)malloc(sizeof(double) * (size_t)(m + 1));
    s.row_scale = (double *)malloc(sizeof(double) * (size_t)(m + 1));
    or_scale(p, lower, upper, &s);

    double *qv = NULL;
    if (qp) { /* pdqp.cpp:35-45 */
        qv = (double *)malloc(sizeof(double) * (size_t)p->q_nnz);
        for (int64_t r = 0; r < n; ++r)
            for (int64_t k = p->qro[r]; k < p->qro[r + 1]; ++k)
                qv[k] = p->qv[k] * (s.col_scale[r] * s.col_scale[p->qci[k]]);
    }

    double *x = (double *)calloc((size_t)(n + 1), sizeof(double));
    double *xn = (double *)calloc((size_t)(n + 1), sizeof(double));
    double *xb = (double *)calloc((size_t)(n + 1), sizeof(double));
    double *aty = (double *)calloc((size_t)(n + 1), sizeof(double));
    double *qx = (double *)calloc((size_t)(n + 1), sizeof(double));
    double *g = (double *)calloc((size_t)(n + 1), sizeof(double));
    double *px = (double *)calloc((size_t)(n + 1), sizeof(double));
    double *y = (double *)calloc((size_t)(m + 1), sizeof(double));
    double *axb = (double *)calloc((size_t)(m + 1), sizeof(double));
    double *yarg = (double *)calloc((size_t)(m + 1), sizeof(double));
    double *yproj = (double *)calloc((size_t)(m + 1), sizeof(double));
    double *ax = (double *)calloc((size_t)(m + 1), sizeof(double));
    double *pax = (double *)calloc((size_t)(m + 1), sizeof(double));

    /* warm start / projection -- pdhg.cpp:61-72 */
    for (int64_t j = 0; j < n; ++j) x[j] = warm ? warm[j] / s.col_scale[j] : 0.0;
    for (int64_t j = 0; j < n; ++j) x[j] = clampbox(x[j], s.l[j], s.u[j]);

    const double matrix_norm = or_operator_bound(m, n, p->ro, p->ci, s.v);
    double max_step;
    if (qp) { /* pdqp.cpp:89-99 */
        double q_norm = 0.0;
        for (int64_t r = 0; r < n; ++r) {
            double rs = 0.0;
            for (int64_t k = p->qro[r]; k < p->qro[r + 1]; ++k) rs += fabs(qv[k]);
            q_norm = smax(q_norm, rs);
        }
        max_step = 0.99 / smax(1.0, matrix_norm * matrix_norm + q_norm);
    } else {
        max_step = 0.99 / smax(1.0, matrix_norm);
    }
    double tau = max_step, sigma = max_step;
    double previous = INFINITY;
    int restart = 0;
    res->status = OR_NOT_SOLVED;
    res->iterations = 0;
    res->restarts = 0;
    const double tol = smax(o->primal_tolerance, o->dual_tolerance);

    for (int64_t it = 0; it < o->iteration_limit; ++it) {
        if (isfinite(o->time_limit_seconds) && now_s() - t0 >= o->time_limit_seconds) {
            res->status = OR_TIME_LIMIT;
            break;
        }
        or_spmv_t(m, n, p->ro, p->ci, s.v, 1.0, y, 0.0, aty);
        if (qp) {
            or_spmv(n, p->qro, p->qci, qv, 1.0, x, 0.0, qx);
            for (int64_t j = 0; j < n; ++j) g[j] = qx[j];
            for (int64_t j = 0; j < n; ++j) g[j] = 1.0 * s.c[j] + 1.0 * g[j];
            for (int64_t j = 0; j < n; ++j) g[j] = 1.0 * aty[j] + 1.0 * g[j];
            for (int64_t j = 0; j < n; ++j) xn[j] = x[j];
            for (int64_t j = 0; j < n; ++j) xn[j] = -tau * g[j] + 1.0 * xn[j];
        } else {
            for (int64_t j = 0; j < n; ++j) xn[j] = x[j];
            for (int64_t j = 0; j < n; ++j) xn[j] = -tau * s.c[j] + 1.0 * xn[j];
            for (int64_t j = 0; j < n; ++j) xn[j] = -tau * aty[j] + 1.0 * xn[j];
        }
        for (int64_t j = 0; j < n; ++j) xn[j] = clampbox(xn[j], s.l[j], s.u[j]);
        if (restart) {
            for (int64_t j = 0; j < n; ++j) xb[j] = xn[j];
            restart = 0;
        } else {
            for (int64_t j = 0; j < n; ++j) xb[j] = x[j];
            for (int64_t j = 0; j < n; ++j) xb[j] = 2.0 * xn[j] + -1.0 * xb[j];
        }
        or_spmv(m, p->ro, p->ci, s.v, 1.0, xb, 0.0, axb);
        const double inv_sigma = 1.0 / sigma;
        for (int64_t r = 0; r < m; ++r) yarg[r] = y[r];
        for (int64_t r = 0; r < m; ++r) yarg[r] = sigma * axb[r] + 1.0 * yarg[r];
        for (int64_t r = 0; r < m; ++r) yproj[r] = yarg[r];
        for (int64_t r = 0; r < m; ++r) yproj[r] = inv_sigma * yproj[r] + 0.0 * yproj[r];
        for (int64_t r = 0; r < m; ++r) yproj[r] = clampbox(yproj[r], s.rl[r], s.ru[r]);
        for (int64_t r = 0; r < m; ++r) y[r] = yarg[r];
        for (int64_t r = 0; r < m; ++r) y[r] = -sigma * yproj[r] + 1.0 * y[r];
        for (int64_t j = 0; j < n; ++j) x[j] = xn[j];
        res->iterations = it + 1;

        or_spmv(m, p->ro, p->ci, s.v, 1.0, x, 0.0, ax);
        for (int64_t r = 0; r < m; ++r) pax[r] = clampbox(ax[r], s.rl[r], s.ru[r]);
        for (int64_t r = 0; r < m; ++r) ax[r] = 1.0 * pax[r] + -1.0 * ax[r];
        const double primal = norm_inf(ax, m);

        or_spmv_t(m, n, p->ro, p->ci, s.v, 1.0, y, 0.0, aty);
        if (qp) {
            or_spmv(n, p->qro, p->qci, qv, 1.0, x, 0.0, qx);
            for (int64_t j = 0; j < n; ++j) g[j] = qx[j];
            for (int64_t j = 0; j < n; ++j) g[j] = 1.0 * s.c[j] + 1.0 * g[j];
            for (int64_t j = 0; j < n; ++j) g[j] = 1.0 * aty[j] + 1.0 * g[j];
        } else {
            for (int64_t j = 0; j < n; ++j) g[j] = s.c[j];
            for (int64_t j = 0; j < n; ++j) g[j] = 1.0 * aty[j] + 1.0 * g[j];
        }
        for (int64_t j = 0; j < n; ++j) px[j] = -1.0 * g[j] + 1.0 * x[j];
        for (int64_t j = 0; j < n; ++j) px[j] = clampbox(px[j], s.l[j], s.u[j]);
        double stat = 0.0;
        for (int64_t j = 0; j < n; ++j) stat = smax(stat, fabs(1.0 * x[j] + -1.0 * px[j]));
        const double metric = smax(primal, stat);
        res->last_metric = metric;

        /* step / restart rule -- pdhg.cpp:133-145 */
        if (it > 0 && it % 50 == 0) {
            if (metric > previous * 1.25) {
                tau *= 0.5;
                sigma *= 0.5;
                restart = 1;
                res->restarts++;
            } else if (metric < previous * 0.1) {
                tau = smin(tau * 1.05, max_step);
                sigma = tau;
            }
            previous = metric;
        } else if (it == 0) {
            previous = metric;
        }
        if (metric <= tol) {
            res->status = OR_OPTIMAL;
            break;
        }
    }
    res->tau = tau;

    /* post-processing in original coordinates -- pdhg.cpp:153-264 */
    for (int64_t j = 0; j < n; ++j) res->x[j] = x[j] * s.col_scale[j];
    if (res->scaled_x)
        for (int64_t j = 0; j < n; ++j) res->scaled_x[j] = x[j];
    if (res->scaled_y)
        for (int64_t r = 0; r < m; ++r) res->scaled_y[r] = y[r];
    const double *sol = res->x;
    double dot = 0.0;
    for (int64_t j = 0; j < n; ++j) dot += p->c[j] * sol[j];
    double obj = p->objective_offset + dot;
    if (qp) { /* continuous_common.hpp:284-300 (dense sum; zero entries add nothing) */
        double quad = 0.0;
        for (int64_t r = 0; r < n; ++r)
            for (int64_t k = p->qro[r]; k < p->qro[r + 1]; ++k) quad += sol[r] * p->qv[k] * sol[p->qci[k]];
        obj += 0.5 * quad;
    }
    res->objective = obj;
    int nonfinite_obj = !isfinite(obj);
    double *rowv = ax;
    or_spmv(m, p->ro, p->ci, p->v, 1.0, sol, 0.0, rowv);
    res->primal_residual = box_violation(rowv, p->rl, p->ru, m);
    res->primal_residual = smax(res->primal_residual, box_violation(sol, lower, upper, n));

    for (int64_t r = 0; r < m; ++r) {
        const double d = y[r] * s.row_scale[r];
        res->y[r] = d;
        res->row_lower_dual[r] = smax(0.0, -d);
        res->row_upper_dual[r] = smax(0.0, d);
    }
    double *st = g;
    for (int64_t j = 0; j < n; ++j) st[j] = p->c[j];
    if (qp) { /* pdqp.cpp:216-225 */
        for (int64_t r = 0; r < n; ++r)
            for (int64_t k = p->qro[r]; k < p->qro[r + 1]; ++k) st[r] += p->qv[k] * sol[p->qci[k]];
    }
    for (int64_t r = 0; r < m; ++r) {
        const double mult = res->y[r];
        for (int64_t k = p->ro[r]; k < p->ro[r + 1]; ++k) st[p->ci[k]] += mult * p->v[k];
    }
    double stat_res = 0.0, comp = 0.0;
    const double active_tol = smax(10.0 * o->primal_tolerance, 1e-8);
    for (int64_t j = 0; j < n; ++j) {
        const double proj = sclamp(sol[j] - st[j], lower[j], upper[j]);
        stat_res = smax(stat_res, fabs(sol[j] - proj));
        res->var_lower_dual[j] = 0.0;
        res->var_upper_dual[j] = 0.0;
        if (isfinite(lower[j]) && sol[j] - lower[j] <= active_tol) {
            res->var_lower_dual[j] = smax(0.0, st[j]);
            comp = smax(comp, fabs((sol[j] - lower[j]) * res->var_lower_dual[j]));
        }
        if (isfinite(upper[j]) && upper[j] - sol[j] <= active_tol) {
            res->var_upper_dual[j] = smax(0.0, -st[j]);
            comp = smax(comp, fabs((upper[j] - sol[j]) * res->var_upper_dual[j]));
        }
    }
    for (int64_t r = 0; r < m; ++r) {
        if (isfinite(p->rl[r])) comp = smax(comp, fabs((rowv[r] - p->rl[r]) * res->row_lower_dual[r]));
        if (isfinite(p->ru[r])) comp = smax(comp, fabs((p->ru[r] - rowv[r]) * res->row_upper_dual[r]));
    }
    res->stationarity_residual = stat_res;
    res->complementarity_residual = comp;
    if (nonfinite_obj) res->status = OR_NUMERICAL_FAILURE;
    if (res->status == OR_NOT_SOLVED) res->status = OR_ITERATION_LIMIT;
    int finite = 1;
    for (int64_t j = 0; j < n; ++j)
        if (!isfinite(sol[j])) finite = 0;
    if (!finite) {
        res->status = OR_NUMERICAL_FAILURE;
    } else if (res->status == OR_OPTIMAL &&
               (res->primal_residual > o->primal_tolerance || stat_res > o->dual_tolerance)) {
        res->status = OR_NUMERICAL_FAILURE;
    }
    res->solve_seconds = now_s() - t0;

    free(x); free(xn); free(xb); free(aty); free(qx); free(g); free(px);
    free(y); free(axb); free(yarg); free(yproj); free(ax); free(pax); free(qv);
    free(s.v); free(s.c); free(s.l); free(s.u); free(s.col_scale); free(s.rl); free(s.ru); free(s.row_scale);
    return 0;
}

/*
 * Relative KKT error of (x, y) in original coordinates (no reference
 * counterpart: the reference stops on an absolute infinity norm in scaled
 * coordinates, pdhg.cpp:147). Sign convention as SolveResult.hpp:31-33:
 * c + Qx + A'y - lambda = 0, y > 0 <=> upper row bound active.
 *   primal  = ||Ax - clamp(Ax, rl, ru)||_2 + ||x - clamp(x, l, u)||_2
 *   dual    = ||lambda - proj_Lambda(lambda)||_2 (+ row-dual sign violations)
 *   gap     = |p - d|
 * and the scales 1 + ||b||_2 (b_i = largest finite |row bound|), 1 + ||c||_2,
 * 1 + |p| + |d|.
 */
void or_rel_kkt(const or_problem *p, const double *lower, const double *upper, const double *x,
                const double *y, or_kkt *out) {
    const int64_t m = p->m, n = p->n;
    double *ax = (double *)calloc((size_t)(m + 1), sizeof(double));
    double *lam = (double *)calloc((size_t)(n + 1), sizeof(double));
    double *qx = (double *)calloc((size_t)(n + 1), sizeof(double));
    or_spmv(m, p->ro, p->ci, p->v, 1.0, x, 0.0, ax);
    if (p->q_nnz > 0) or_spmv(n, p->qro, p->qci, p->qv, 1.0, x, 0.0, qx);
    double rp_rows = 0.0, rp_box = 0.0, bnorm = 0.0, cnorm = 0.0;
    for (int64_t r = 0; r < m; ++r) {
        const double pr = clampbox(ax[r], p->rl[r], p->ru[r]);
        rp_rows += (ax[r] - pr) * (ax[r] - pr);
        double b = 0.0;
        if (isfinite(p->rl[r])) b = smax(b, fabs(p->rl[r]));
        if (isfinite(p->ru[r])) b = smax(b, fabs(p->ru[r]));
        bnorm += b * b;
    }
    for (int64_t j = 0; j < n; ++j) {
        const double pj = clampbox(x[j], lower[j], upper[j]);
        rp_box += (x[j] - pj) * (x[j] - pj);
        cnorm += p->c[j] * p->c[j];
        lam[j] = p->c[j] + qx[j];
    }
    or_spmv_t(m, n, p->ro, p->ci, p->v, 1.0, y, 1.0, lam);
    double rd = 0.0, dual_obj = 0.0, primal_obj = 0.0, quad = 0.0;
    for (int64_t r = 0; r < m; ++r) {
        const double yl = smax(0.0, -y[r]), yu = smax(0.0, y[r]);
        if (yl > 0.0) {
            if (isfinite(p->rl[r])) dual_obj += p->rl[r] * yl; else rd += yl * yl;
        }
        if (yu > 0.0) {
            if (isfinite(p->ru[r])) dual_obj -= p->ru[r] * yu; else rd += yu * yu;
        }
    }
    for (int64_t j = 0; j < n; ++j) {
        const double vl = smax(0.0, lam[j]), vu = smax(0.0, -lam[j]);
        if (vl > 0.0) {
            if (isfinite(lower[j])) dual_obj += lower[j] * vl; else rd += vl * vl;
        }
        if (vu > 0.0) {
            if (isfinite(upper[j])) dual_obj -= upper[j] * vu; else rd += vu * vu;
        }
        primal_obj += p->c[j] * x[j];
        quad += x[j] * qx[j];
    }
    primal_obj += 0.5 * quad + p->objective_offset;
    dual_obj += -0.5 * quad + p->objective_offset;
    out->primal_residual = sqrt(rp_rows) + sqrt(rp_box);
    out->dual_residual = sqrt(rd);
    out->primal_objective = primal_obj;
    out->dual_objective = dual_obj;
    out->gap = fabs(primal_obj - dual_obj);
    out->rel_primal = out->primal_residual / (1.0 + sqrt(bnorm));
    out->rel_dual = out->dual_residual / (1.0 + sqrt(cnorm));
    out->rel_gap = out->gap / (1.0 + fabs(primal_obj) + fabs(dual_obj));
    free(ax); free(lam); free(qx);
}
