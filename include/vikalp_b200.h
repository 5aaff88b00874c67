/*
 * vikalp_b200.h -- C ABI of the B200 (sm_100a) PDHG LP / PDQP library.
 *
 * This is the boundary VIKALP's CUDA route binds to. It replaces, for LP and
 * convex QP, the reference's CUDA ExecutionBackend
 * (include/vikalp/backend/CudaBackend.hpp:18-20, cuda/cuda_ops.cu) plus the
 * backend-driven PDHG / PDQP loops that run on it
 * (src/solver/lp/pdhg.cpp:20-265, src/solver/qp/pdqp.cpp:20-298). The C++
 * router (vikalp::solve, include/vikalp/solver/Solver.hpp) calls these entry
 * points when SolverOptions::backend == BackendPreference::CUDA.
 *
 * Conventions
 *   - Plain pointers and sizes only; all matrices are CSR with int64 offsets
 *     and indices and float64 values, exactly the reference's CsrPattern /
 *     CsrMatrix (include/vikalp/contracts/Model.hpp:16-26).
 *   - Every function returns VK_OK (0) or a negative status; nothing throws
 *     across the ABI. vk_last_error() gives the message of the calling
 *     thread's most recent failure.
 *   - Host pointers unless the name says _device. Device pointers are
 *     addresses on the current CUDA device.
 *   - A handle is owned by one thread at a time and owns one CUDA stream
 *     ("create one backend per thread", CudaBackend.hpp:17).
 */
#ifndef VIKALP_B200_H
#define VIKALP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define VK_OK 0
#define VK_ERR_INVALID (-1)     /* invalid input: SolveStatus::InvalidModel      */
#define VK_ERR_UNSUPPORTED (-2) /* unsupported model/method: UnsupportedModel     */
#define VK_ERR_CUDA (-3)        /* CUDA runtime failure: NumericalFailure         */
#define VK_ERR_INTERNAL (-4)    /* any other failure: NumericalFailure            */

/* SolveStatus values (include/vikalp/contracts/SolveResult.hpp:11-24). */
enum {
    VK_STATUS_NOT_SOLVED = 0,
    VK_STATUS_OPTIMAL = 1,
    VK_STATUS_ITERATION_LIMIT = 6,
    VK_STATUS_TIME_LIMIT = 8,
    VK_STATUS_NUMERICAL_FAILURE = 9,
    VK_STATUS_UNSUPPORTED_MODEL = 10,
    VK_STATUS_INVALID_MODEL = 11
};

/* Iteration schemes. */
enum {
    /* The reference's restarted PDHG / PDQP, iterate for iterate
     * (pdhg.cpp:87-151, pdqp.cpp:110-178): single-pass infinity-norm scaling,
     * tau = sigma, step halving / growth every 50 iterations, absolute
     * infinity-norm stop in scaled coordinates. */
    VK_ALGO_REFERENCE = 0,
    /* Restarted reflected-Halpern PDHG: Ruiz + Pock-Chambolle scaling, power
     * iteration step size, primal weight, fixed-point-residual restarts and a
     * relative-KKT stop in original coordinates. */
    VK_ALGO_HALPERN = 1
};

enum { VK_PREC_FP64 = 0, VK_PREC_MIXED = 1 };

/* Sparse products: FAST uses warp-cooperative sums for long rows;
 * SEQUENTIAL sums every row left to right in CSR order, which is the order the
 * reference's CPU backend uses (cpu_ops.cpp:418-427, 444-458), so results
 * are bit-identical to it. */
enum { VK_SPMV_FAST = 0, VK_SPMV_SEQUENTIAL = 1 };

typedef struct {
    int64_t rows, cols;
    const int64_t *row_offsets; /* [rows + 1], row_offsets[0] == 0 */
    const int64_t *col_indices; /* [nnz], strictly increasing per row */
    const double *values;       /* [nnz] */
} vk_csr;

/* Canonical model (Model.hpp:38-44): min c'x + 0.5 x'Qx + offset
 * s.t. row_lower <= A x <= row_upper, var_lower <= x <= var_upper. */
typedef struct {
    vk_csr A;        /* m x n */
    vk_csr Q;        /* n x n full symmetric CSR, or rows == cols == 0 for an LP */
    const double *c; /* [n] */
    double objective_offset;
    const double *var_lower, *var_upper; /* [n], -inf / +inf allowed */
    const double *row_lower, *row_upper; /* [m], -inf / +inf allowed */
} vk_problem;

/* Mirrors vikalp::SolverOptions (SolverOptions.hpp:15-28) plus the B200
 * extensions. Fill with vk_default_options() first. */
typedef struct {
    int64_t iteration_limit;   /* SolverOptions::iteration_limit (100000)       */
    double time_limit_seconds; /* SolverOptions::time_limit_seconds (+inf)      */
    double primal_tolerance;   /* SolverOptions::primal_tolerance (1e-7)        */
    double dual_tolerance;     /* SolverOptions::dual_tolerance (1e-7)          */
    int32_t continuous_method; /* SolverOptions::continuous_method: 0 Auto,     */
                               /* 1 PDHG, 2 RevisedSimplex, 3 InteriorPoint (0) */
    int32_t algorithm;         /* VK_ALGO_*                    (REFERENCE)      */
    int32_t precision;         /* VK_PREC_*                    (FP64)           */
    int32_t spmv_order;        /* VK_SPMV_*                    (FAST)           */
    int32_t check_every;       /* iterations per device-side check (64)         */
    double relative_tolerance; /* HALPERN stop: relative KKT (1e-6)             */
    int32_t device;            /* CUDA device ordinal (0)                       */
    int32_t verbose;           /* 0: silent                                      */
} vk_options;

/* Outputs. Array pointers are caller-allocated host buffers or NULL. */
typedef struct {
    double *x;              /* [n] primal solution, original coordinates      */
    double *y;              /* [m] row multipliers (y > 0: upper row active)   */
    double *row_lower_dual; /* [m] SolveResult::constraint_lower_dual          */
    double *row_upper_dual; /* [m] SolveResult::constraint_upper_dual          */
    double *var_lower_dual; /* [n] SolveResult::variable_lower_dual            */
    double *var_upper_dual; /* [n] SolveResult::variable_upper_dual            */
    int32_t status;         /* VK_STATUS_*                                      */
    int64_t iterations;
    int64_t restarts;
    double objective;
    double primal_residual, stationarity_residual, complementarity_residual;
    double rel_primal, rel_dual, rel_gap; /* relative KKT of the returned point  */
    double last_metric;                   /* the reference's scaled max(inf-norms) */
    double solve_seconds;
    double iterate_seconds; /* device time of the iteration loop alone */
    int64_t fp32_iterations; /* MIXED: iterations done in FP32 */
    int64_t kernel_launches; /* kernels this library launched in the iteration loop */
    char message[256];
} vk_result;

typedef struct vk_pdhg vk_pdhg;

void vk_default_options(vk_options *opts);
const char *vk_last_error(void);
const char *vk_version(void);

/* Validates the model as Model::validate + solve_lp/solve_qp do
 * (Model.cpp:118-199, continuous_common.hpp:80-126), copies it to the GPU and
 * builds every device-side structure (int32 CSR, transposed CSR, scaling,
 * tile schedules). Replaces the setup half of solve_scaled_lp / qp
 * (pdhg.cpp:20-80, pdqp.cpp:20-103). With VK_SPMV_FAST an LP whose column
 * nonzero counts are skewed gets its columns renamed internally in order of
 * decreasing count (environment VIKALP_B200_COLUMN_ORDER = auto | keep |
 * count, read here; any other value fails with VK_ERR_INVALID); overrides,
 * warm starts and results stay in the caller's column order. */
int vk_pdhg_create(const vk_problem *problem, const vk_options *opts, vk_pdhg **out);

/* Runs the solve. warm_start, var_lower_override and var_upper_override are
 * NULL or n long (RelaxationOracle.hpp:15-16, continuous_common.hpp:80-110).
 * Replaces the loop and post-processing of solve_scaled_lp / qp
 * (pdhg.cpp:87-264, pdqp.cpp:110-297). Model errors (bad overrides, a
 * non-finite warm start) return VK_OK with result->status INVALID_MODEL, as the
 * reference returns a SolveResult rather than throwing. */
int vk_pdhg_solve(vk_pdhg *h, const double *warm_start, const double *var_lower_override,
                  const double *var_upper_override, vk_result *result);

/* Changes the per-solve options of a handle for its next solves: the limits
 * and tolerances (iteration_limit, time_limit_seconds, primal_tolerance,
 * dual_tolerance, relative_tolerance, verbose), as the reference passes
 * SolverOptions to every RelaxationOracle::solve call
 * (RelaxationOracle.hpp:17-22). Every other field must equal the one the
 * handle was created with (VK_ERR_INVALID otherwise); invalid limits are
 * rejected with the reference's message (continuous_common.hpp:50-56). */
int vk_pdhg_set_options(vk_pdhg *h, const vk_options *opts);

void vk_pdhg_destroy(vk_pdhg *h);

/* Device time of each kernel kind of a handle's iteration loop: runs
 * `iterations` iterations of the handle's scheme from a cold start with the
 * model's bounds (no tolerance stop), launched one by one instead of as a
 * CUDA graph, with CUDA events around every kernel kind on the handle's
 * stream. For measurement only (no counterpart in the reference, whose
 * backend calls are timed by nothing). VK_ALGO_REFERENCE handles report
 * three kinds: the column pass, the control (+ primal) kernels and the row
 * pass; other schemes return VK_ERR_UNSUPPORTED. */
typedef struct {
    int32_t count;             /* kernel kinds reported (<= 8)                  */
    char name[8][48];
    double ms_per_launch[8];   /* mean device time per launch                   */
    int64_t launches[8];
    double bytes_per_launch[8]; /* algorithmic bytes one launch moves (0: none) */
} vk_pass_profile;
int vk_pdhg_profile(vk_pdhg *h, int64_t iterations, vk_pass_profile *out);

/* ---- primitives (ExecutionBackend-level, ExecutionBackend.hpp:36-64) ------ */

/* CSR transpose on the GPU by a stable counting sort on the column index, so
 * that rows ascend within each column (the accumulation order of the
 * reference's transposed product, cpu_ops.cpp:449-458). Host arrays:
 * t_row_offsets[cols+1], t_col_indices[nnz] (= source rows), t_values[nnz]
 * (may be NULL), perm[nnz] (source position of each entry; may be NULL). */
int vk_csr_transpose(const vk_csr *a, int64_t *t_row_offsets, int64_t *t_col_indices,
                     double *t_values, int64_t *perm);

/* y = alpha * op(A) * x + beta * y with host arrays
 * (ExecutionBackend::multiply, cpu_ops.cpp:393-460 / cuda_ops.cu:473-528).
 * transpose != 0 computes A' * x through a transposed CSR built on the GPU. */
int vk_spmv(const vk_csr *a, double alpha, const double *x, double beta, double *y, int transpose,
            int spmv_order);

/* A reusable sparse operator resident on the GPU, for repeated products on
 * device vectors (the bench's SpMV bandwidth figure uses it). */
typedef struct vk_spmat vk_spmat;
/* precision: VK_PREC_FP64 stores float64 values, VK_PREC_MIXED float32. */
int vk_spmat_create(const vk_csr *a, int32_t precision, vk_spmat **out);
/* y = A x (transpose == 0) or A' x (transpose != 0) on device arrays of the
 * matrix's precision, on `stream` (a cudaStream_t, NULL = default stream). */
int vk_spmat_apply_device(vk_spmat *m, const void *x_device, void *y_device, int transpose,
                          void *stream);
/* Algorithmic bytes one vk_spmat_apply_device call moves (values, int32
 * indices, int32 offsets, x once, y once). */
int64_t vk_spmat_bytes(const vk_spmat *m, int transpose);
/* Kernel variant the setup autotuner picked for A (transpose == 0) or A'
 * (timing each candidate on this matrix), and a way to pin one
 * (0 <= variant < 18). Results agree to rounding across variants. */
int vk_spmat_variant(const vk_spmat *m, int transpose);
int vk_spmat_set_variant(vk_spmat *m, int transpose, int variant);
void vk_spmat_destroy(vk_spmat *m);

/* Replaces the operator's values (nnz doubles, host array, the CSR order it was
 * created with): ExecutionBackend::set_values (cpu_ops.cpp set_values,
 * cuda_ops.cu:362-372). Float64 operators only. */
int vk_spmat_set_values(vk_spmat *m, const double *values, int64_t nnz);

/* ---- device vectors (ExecutionBackend.hpp:36-64) ------------------------------
 * The vector side of the reference's ExecutionBackend contract, for its CUDA
 * route (make_cuda_backend, include/vikalp/backend/CudaBackend.hpp in this
 * repository, built on these). A vk_dvec is n doubles on the device that was
 * current when it was created; every operation runs on that thread's legacy
 * default stream, in call order. Semantics are the CPU backend's
 * (cpu_ops.cpp): axpby rounds alpha*x and beta*y separately (bit-identical to
 * the CPU loop), project_box is min(max(x, lo), hi) with NaN in x passing
 * through, norm_inf ignores NaN, dot is a fixed-order tree sum. Size
 * mismatches return VK_ERR_INVALID naming the operation (the reference throws
 * std::invalid_argument there). */
typedef struct vk_dvec vk_dvec;
int vk_device_select(int32_t device); /* makes `device` current for this thread */
int vk_device_synchronize(void);     /* waits for the current device's work */
int vk_dvec_create(int64_t n, vk_dvec **out); /* zero-filled */
void vk_dvec_destroy(vk_dvec *v);
int64_t vk_dvec_size(const vk_dvec *v);
int vk_dvec_upload(vk_dvec *v, const double *host, int64_t n);
int vk_dvec_download(const vk_dvec *v, double *host, int64_t n); /* returns when the copy is done */
int vk_dvec_fill(vk_dvec *v, double value);
int vk_dvec_copy(const vk_dvec *src, vk_dvec *dst);
int vk_dvec_axpby(double alpha, const vk_dvec *x, double beta, vk_dvec *y); /* y = alpha x + beta y */
int vk_dvec_dot(const vk_dvec *x, const vk_dvec *y, double *result);
int vk_dvec_norm_inf(const vk_dvec *x, double *result);
int vk_dvec_project_box(vk_dvec *x, const vk_dvec *lower, const vk_dvec *upper);
/* y = alpha * op(A) x + beta * y on device vectors (ExecutionBackend::multiply,
 * cpu_ops.cpp:393-460, cuda_ops.cu:473-528): x and y distinct, op(A) = A' when
 * transpose != 0 (the pre-built transposed CSR). VK_SPMV_SEQUENTIAL sums in
 * the CPU backend's order (bit-identical); VK_SPMV_FAST uses the autotuned
 * kernels. */
int vk_spmat_multiply(vk_spmat *m, double alpha, const vk_dvec *x, double beta, vk_dvec *y, int transpose,
                      int spmv_order);

/* ExecutionBackend::dot and ::norm_inf on device arrays of n doubles
 * (ExecutionBackend.hpp:49-51; cuda_ops.cu:407-451), written to
 * *result_device on `stream` (a cudaStream_t, NULL = default stream). Block
 * partials go to a per-device scratch buffer this library allocates on first
 * use (cudaMalloc) and grows as needed; the final sum / max runs on the device
 * in a fixed order, so results are deterministic. norm_inf ignores NaN
 * entries, as std::max does in the reference (cpu_ops.cpp:358-364). */
int vk_vec_dot_device(const double *x_device, const double *y_device, int64_t n, double *result_device,
                      void *stream);
int vk_vec_norm_inf_device(const double *x_device, int64_t n, double *result_device, void *stream);

/* vk_vec_dot_device for callers that cannot allocate device memory (a
 * framework allocator or memory pool owns every byte, or the process has a
 * fixed memory budget): the same kernels and the same result, with the block
 * partials in a 32 KB array compiled into the library instead of a buffer
 * allocated by cudaMalloc. No counterpart in the reference. It never calls
 * cudaMalloc or cudaFree. Limits and caveats:
 *   - n <= 8388608 (4096 block partials); larger n returns VK_ERR_INVALID;
 *   - every GPU that loads the library holds the array until the process
 *     exits, and all calls share it: calls that overlap on the GPU (other
 *     streams or host threads) race and may return wrong sums;
 *   - the first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress); make that call before any stream capture. */
int vk_vec_dot_device_noalloc(const double *x_device, const double *y_device, int64_t n, double *result_device,
                              void *stream);

/* ---- diagnostics ------------------------------------------------------------ */

/* Runs the library's failure path for a device wait that never completes,
 * without a fault: one kernel polls an mbarrier that nothing arrives on,
 * `polls` times at most (1..1048576; each poll may suspend the thread
 * briefly), the way the pipelined sparse passes wait for their staged copies.
 * When the limit runs out the kernel records the barrier-timeout code in the
 * per-device error flag and returns; the host reads and clears the flag as
 * after every solve chunk. Expected result: VK_ERR_CUDA with the timeout
 * message (vk_last_error), and the device stays usable for the next call.
 * No counterpart in the reference (its CUDA backend has no device-side waits;
 * failures there are exceptions, cuda_ops.cu:35-46). */
int vk_diag_bounded_wait(int32_t polls);

/* ---- batches ---------------------------------------------------------------- */

/* Solves `count` independent LPs (any sizes) together with VK_ALGO_HALPERN
 * (opts->algorithm must be VK_ALGO_HALPERN; NULL opts = defaults with that
 * algorithm). Replaces a loop of vikalp::solve calls, one per model
 * (Solver.hpp:19-21; the reference has no batch entry point). Every problem is
 * validated with vk_pdhg_create's rules (an invalid one fails the whole call
 * with its index in the message); quadratic objectives are VK_ERR_UNSUPPORTED.
 * The instances share the device passes (one launch advances all of them) but
 * keep their own step sizes, primal weights, restarts and stopping, so each
 * result[b] equals, up to rounding, what one VK_ALGO_HALPERN solve of
 * problem b returns. results[b] receives x, y, status, iterations, restarts,
 * objective and the relative KKT figures. When results[b] also carries any of
 * the four dual arrays (and x, y), those arrays and the reference's three
 * absolute residuals are filled as vk_pdhg_solve fills them (pdhg.cpp:153-264;
 * host threads, after the device loop); otherwise the residuals are NaN.
 * iterate_seconds and kernel_launches cover the whole batch. */
int vk_batch_solve(const vk_problem *problems, int32_t count, const vk_options *opts, vk_result *results);

/* Solves `count` relaxations of ONE LP that differ only in their variable
 * bounds and warm start -- the node LPs of a branch-and-bound tree -- together
 * with VK_ALGO_HALPERN. Replaces a loop of RelaxationOracle::solve(model,
 * lower_override, upper_override, warm_start, options) calls on one model
 * (RelaxationOracle.hpp:17-22). lower, upper and warm are NULL (the model's
 * bounds / a cold start) or count * n doubles, instance b at offset b * n.
 * An instance whose overrides or warm start fail the checks of vk_pdhg_solve
 * gets status INVALID_MODEL and its message; the others are solved. The
 * instances share every read of the constraint matrix (the vectors of all
 * instances are interleaved on the device); each keeps its own primal weight,
 * restarts and stopping, so results[b] equals, up to rounding, one
 * VK_ALGO_HALPERN solve with those overrides. Result fields as in
 * vk_batch_solve. */
int vk_batch_solve_shared(const vk_problem *problem, int32_t count, const double *lower, const double *upper,
                          const double *warm, const vk_options *opts, vk_result *results);

/* vk_batch_solve_shared(problem, node_count, lower, upper, warm, ...) and
 * vk_batch_solve(problems, count, ...) in one call, the two device loops in
 * flight together: both batches are set up first, then each iterates on its
 * own stream from its own host thread, so neither waits for the other's
 * iterations and the GPU is shared between them. node_results[b] and
 * results[b] are what the two calls would return (each member keeps its own
 * primal weight, restarts and stopping). The mixed workload of a
 * branch-and-bound run that also solves independent LPs; no counterpart in the
 * reference (it solves one LP at a time, BranchAndBound.cpp:296-297). */
int vk_batch_solve_together(const vk_problem *problem, int32_t node_count, const double *lower,
                            const double *upper, const double *warm, const vk_problem *problems, int32_t count,
                            const vk_options *opts, vk_result *node_results, vk_result *results);

/* ---- differentiation ---------------------------------------------------------- */

typedef struct {
    double active_tolerance; /* row / bound activity: within tol * (1 + |bound|) (1e-6) */
    double solve_tolerance;  /* LSQR stop: relative residual / normal residual (1e-10)  */
    int64_t iteration_limit; /* LSQR iterations per instance (20000)                    */
    int32_t device;          /* CUDA device ordinal (0)                                 */
} vk_adjoint_options;

typedef struct {
    int64_t rows_active; /* |R|: equality rows and rows at a bound          */
    int64_t cols_free;   /* |F|: variables strictly inside their bounds     */
    int64_t iterations;  /* LSQR iterations                                 */
    int32_t status;      /* VK_STATUS_OPTIMAL or VK_STATUS_ITERATION_LIMIT  */
    double residual;     /* |A_RF' w - g_F| / |g_F|                         */
    double normal_residual; /* |A_RF (A_RF' w - g_F)| / (|A_RF|_F |A_RF' w - g_F|) */
} vk_adjoint_info;

void vk_default_adjoint_options(vk_adjoint_options *opts);

/* Gradients of L = dL_dx' x* + dL_dobj * c'x* for `count` solved LPs with
 * respect to c, the row bounds and the stored values of A, through the
 * active-set KKT system of each optimum (no counterpart in the reference).
 * x / y: the optimum (as vk_pdhg_solve / vk_batch_solve return it; y > 0 is an
 * active upper row bound), solved well below active_tolerance. Active rows R:
 * a finite bound within active_tolerance of A x; free columns F: strictly
 * inside both bounds. With w = the minimum-norm least-squares solution of
 * A_RF' w = dL_dx[F] (LSQR on the GPU, all instances at once):
 *   dL_dc[j]  = dL_dobj * x[j]
 *   dL_db[i]  = w[i] - dL_dobj * y[i]       (b_i: the active bound of row i;
 *                                            0 for an inactive row)
 *   dL_dA[k]  = (-w[i] + dL_dobj * y[i]) * x[j]   (stored entry k = (i, j))
 * All arrays are the instances' arrays concatenated in order: x, dL_dx and
 * dL_dc hold sum(n) doubles, y and dL_db sum(m), dL_dA sum(nnz); outputs may
 * be NULL; info is NULL or `count` records. Problems must be LPs. */
int vk_lp_adjoint(const vk_problem *problems, int32_t count, const double *x, const double *y,
                  const double *dL_dx, double dL_dobj, const vk_adjoint_options *opts, double *dL_dc,
                  double *dL_db, double *dL_dA, vk_adjoint_info *info);

#ifdef __cplusplus
}
#endif
#endif /* VIKALP_B200_H */
