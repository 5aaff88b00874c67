// Host-side declarations of the PDHG solver objects behind the C ABI.
#pragma once

#include "vikalp_b200.h"
#include "vk_csr.cuh"

#include <memory>
#include <string>
#include <vector>

namespace vk {

// The model as uploaded once by vk_pdhg_create (original coordinates, FP64).
struct DeviceModel {
    int m = 0, n = 0;
    int64_t nnz = 0, q_nnz = 0;
    bool qp = false;
    CsrPattern32 a, at, q;
    DevBuf<int> perm;               // transposed position -> CSR position
    DevBuf<double> a_val, at_val;   // original values, CSR and transposed order
    DevBuf<double> q_val;           // original Q values (full symmetric CSR)
    DevBuf<double> c, vl, vu, rl, ru;
    double offset = 0.0;
    std::vector<double> h_c;                 // for the host-side objective sum
    std::vector<int64_t> h_qro, h_qci;       // Q on the host (objective's quadratic term)
    std::vector<double> h_qv;
    std::vector<double> h_vl, h_vu;          // model bounds (override validation)
    bool tuned = false;                      // pattern variants timed (ensure_tuned)
    // Column order (order_columns_by_count): when cperm is set, the device
    // side (a, at, a_val, at_val, c, vl, vu) is in the renamed order and
    // column j' holds original column cperm[j']; the host copies above stay
    // in the caller's order.
    DevBuf<int> cperm;
    bool reordered() const { return cperm.get() != nullptr; }
};

// Device control block of the reference scheme (pdhg.cpp:75-150).
struct RefCtl {
    double tau, sigma, inv_sigma, max_step;
    double previous, last_metric, tol;
    double rp, rd; // atomic-max slots for the two infinity norms
    long long iter, limit, restarts;
    int restart, done, status, pad;
};

// Final-answer reductions of the post-processing passes.
struct PostOut {
    double primal_res, stat_res, comp_res;            // infinity norms (atomic max)
    double sums[12];                                  // relative-KKT sums (see vk_pdhg.cu)
};

class Engine;

class Solver {
public:
    Solver(const vk_problem &p, const vk_options &o);
    ~Solver();
    void solve(const double *warm, const double *lo, const double *hi, vk_result *r);
    // Returns "" on success, else the reason the options were not accepted.
    std::string set_options(const vk_options &o);
    // vk_pdhg_profile; false when the scheme has no profiling path.
    bool profile(long long iterations, vk_pass_profile *out);
    const DeviceModel &model() const { return *dm_; }
    cudaStream_t stream() const { return stream_; }

private:
    vk_options opts_;
    cudaStream_t stream_ = nullptr;
    std::unique_ptr<DeviceModel> dm_;
    std::unique_ptr<Engine> engine_;
};

// Device vectors of the ExecutionBackend primitives (vk_backend.cu).
double *dvec_ptr(vk_dvec *v);
const double *dvec_ptr(const vk_dvec *v);
int64_t dvec_size(const vk_dvec *v);

// Host work already spread over threads (a batch's members) sets this on its
// workers, so the scans inside (validate_problem) stay on their thread
// instead of starting threads of their own.
bool serial_host_work();
void set_serial_host_work(bool on);

// Validation of a vk_problem with the reference's rules and messages.
// Returns "" when valid. `unsupported` is set when the failure maps to
// SolveStatus::UnsupportedModel instead of InvalidModel.
std::string validate_problem(const vk_problem &p, const vk_options &o, bool &unsupported);

// Uploads a validated problem. The sparse-pass variants of its patterns are
// timed on first need (ensure_tuned): engines whose passes use the patterns'
// variants call it; the reference scheme tunes its own two fused passes.
// `reorder`: the column order may change (FAST passes); parity modes pass
// false and keep the caller's order.
std::unique_ptr<DeviceModel> upload_model(const vk_problem &p, cudaStream_t s, int verbose = 0, bool reorder = false);
void ensure_tuned(DeviceModel &dm, cudaStream_t s);

// Independent LPs solved together (vk_batch.cu); throws on invalid input.
void batch_solve(const vk_problem *problems, int count, const vk_options &o, vk_result *results);
// Relaxations of one LP differing in variable bounds / warm start (vk_batch.cu).
void batch_solve_shared(const vk_problem &p, int count, const double *lower, const double *upper,
                        const double *warm, const vk_options &o, vk_result *results);
// A node batch and an independent batch with both device loops in flight at
// once (vk_batch.cu).
void batch_solve_together(const vk_problem &shared, int node_count, const double *lower, const double *upper,
                          const double *warm, const vk_problem *probs, int count, const vk_options &o,
                          vk_result *node_results, vk_result *results);
// Active-set adjoint of solved LPs (vk_adjoint.cu).
void lp_adjoint(const vk_problem *probs, int count, const double *x, const double *y, const double *g, double w_obj,
                const vk_adjoint_options &o, double *dc, double *db, double *da, vk_adjoint_info *info);

} // namespace vk
