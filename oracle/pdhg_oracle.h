/* CPU oracle for the PDHG LP / PDQP path -- test infrastructure only (see pdhg_oracle.c). */
#ifndef VIKALP_PDHG_ORACLE_H
#define VIKALP_PDHG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_NOT_SOLVED = 0, OR_OPTIMAL = 1, OR_ITERATION_LIMIT = 6, OR_TIME_LIMIT = 8, OR_NUMERICAL_FAILURE = 9 };

typedef struct {
    int64_t m, n;
    const int64_t *ro, *ci; /* A: CSR, m x n */
    const double *v;
    int64_t q_nnz; /* 0 for an LP */
    const int64_t *qro, *qci;
    const double *qv;
    const double *c, *rl, *ru;
    double objective_offset;
} or_problem;

typedef struct {
    int64_t iteration_limit;
    double time_limit_seconds;
    double primal_tolerance, dual_tolerance;
} or_options;

typedef struct {
    double *v, *c, *l, *u, *rl, *ru, *row_scale, *col_scale;
} or_scaled;

typedef struct {
    /* caller-allocated outputs */
    double *x;              /* [n] original coordinates */
    double *y;              /* [m] unscaled row multipliers (y > 0: upper row active) */
    double *row_lower_dual; /* [m] */
    double *row_upper_dual; /* [m] */
    double *var_lower_dual; /* [n] */
    double *var_upper_dual; /* [n] */
    double *scaled_x;       /* [n] or NULL: final iterate in scaled coordinates */
    double *scaled_y;       /* [m] or NULL */
    int status;
    int64_t iterations, restarts;
    double objective, primal_residual, stationarity_residual, complementarity_residual;
    double last_metric, tau, solve_seconds;
} or_result;

typedef struct {
    double primal_residual, dual_residual, gap;
    double primal_objective, dual_objective;
    double rel_primal, rel_dual, rel_gap;
} or_kkt;

void or_spmv(int64_t m, const int64_t *ro, const int64_t *ci, const double *v, double alpha,
             const double *x, double beta, double *y);
void or_spmv_t(int64_t m, int64_t n, const int64_t *ro, const int64_t *ci, const double *v,
               double alpha, const double *x, double beta, double *y);
void or_csr_transpose(int64_t m, int64_t n, const int64_t *ro, const int64_t *ci, const double *v,
                      int64_t *tro, int64_t *trow, double *tv, int64_t *perm);
void or_scale(const or_problem *p, const double *lower, const double *upper, or_scaled *s);
double or_operator_bound(int64_t m, int64_t n, const int64_t *ro, const int64_t *ci, const double *v);
int or_pdhg_solve(const or_problem *p, const or_options *o, const double *warm, const double *lower,
                  const double *upper, or_result *res);
void or_rel_kkt(const or_problem *p, const double *lower, const double *upper, const double *x,
                const double *y, or_kkt *out);

#ifdef __cplusplus
}
#endif
#endif
