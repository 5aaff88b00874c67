// Iteration engines (one per VK_ALGO_*) and the kernels they share.
#pragma once

#include "vk_solver.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>

namespace vk {

// Primal weight and restart rule of the restarted Halpern scheme, the same for
// the single-instance engine and every member of a batch. The primal weight
// omega starts at `start` x omega_0 (omega_0 = |c^| / |b^|, scaled) and at
// every restart moves to exp(theta log(|dy|/|dx|) + (1 - theta) log omega),
// |dx|, |dy| the moves since the last restart point (theta = 0: fixed), as
// long as the relative KKT error is at least `freeze` (below it, omega keeps
// its value).
// Restart when the fixed-point residual r fell below beta_suff x its value at
// the last restart, or below beta_nec x and grew since the previous check, or
// when the iterations since the restart reach beta_art x all iterations.
// VIKALP_B200_PRIMAL_WEIGHT="start,theta,freeze" and
// VIKALP_B200_RESTART="sufficient,necessary,artificial" override the
// defaults (experiments; every engine reads them at the start of a solve).
//
// Defaults (start 1, theta 0.2, thresholds 0.2 / 0.8 / 0.2) were chosen on
// all five measured workloads at full size on a B200: PDLP's theta = 0.5
// with the 0.36 artificial restart leaves the large power-law LP (m=1e6,
// n=2e6) at 2e-5 relative KKT after 200k iterations, its primal weight
// sliding from omega_0 to 0.008 omega_0 as restarts grow rare; the smaller
// step and the earlier artificial restart solve it to 1e-6 in 132k
// iterations, and change the small LP, the QP, the node and independent LPs
// and the 1e-9 adjoint solves by -10%..+12% in iterations.
struct PrimalWeightRule {
    double start = 1.0, theta = 0.2, freeze = 0.0;
    double beta_suff = 0.2, beta_nec = 0.8, beta_art = 0.2;
};

inline PrimalWeightRule primal_weight_rule() {
    PrimalWeightRule r;
    if (const char *e = std::getenv("VIKALP_B200_PRIMAL_WEIGHT"); e && *e) {
        double a = r.start, b = r.theta, f = r.freeze;
        const int got = std::sscanf(e, "%lf,%lf,%lf", &a, &b, &f);
        if (got >= 1 && a > 0.0) r.start = a;
        if (got >= 2 && b >= 0.0 && b <= 1.0) r.theta = b;
        if (got >= 3 && f >= 0.0) r.freeze = f;
    }
    if (const char *e = std::getenv("VIKALP_B200_RESTART"); e && *e) {
        double a = r.beta_suff, b = r.beta_nec, c = r.beta_art;
        if (std::sscanf(e, "%lf,%lf,%lf", &a, &b, &c) == 3 && a > 0.0 && a < 1.0 && b > 0.0 && b < 1.0 && c > 0.0)
            r.beta_suff = a, r.beta_nec = b, r.beta_art = c;
    }
    return r;
}

struct RunInfo {
    int status = VK_STATUS_NOT_SOLVED;
    long long iterations = 0, restarts = 0, fp32_iterations = 0, kernel_launches = 0;
    double last_metric = 0.0;
    double iterate_seconds = 0.0;
};

// Device time per kernel kind of the iteration loop (vk_pdhg_profile).
struct PassProfile {
    static constexpr int kMax = 8;
    int count = 0;
    const char *name[kMax] = {};
    double ms[kMax] = {};         // summed device time (CUDA events)
    long long launches[kMax] = {};
    double bytes[kMax] = {};      // algorithmic bytes per launch (0: not modelled)
};

class Engine {
public:
    virtual ~Engine() = default;
    // Runs the iteration for one solve. d_lo / d_hi: effective original
    // variable bounds; d_warm: warm start in original coordinates or null.
    // On return d_xo [n] / d_yo [m] hold the answer in original coordinates.
    virtual void run(const double *d_warm, const double *d_lo, const double *d_hi, double *d_xo, double *d_yo,
                     RunInfo &info, std::chrono::steady_clock::time_point started) = 0;
    // Per-solve limits and tolerances (the structural options never change).
    virtual void set_limits(const vk_options &o) = 0;
    // Runs `iterations` iterations from a cold start with the model's bounds,
    // launched one by one (no graph) with CUDA events around each kernel kind
    // on the engine's stream. False when the engine has no profiling path.
    virtual bool profile(long long, PassProfile &) { return false; }
};

std::unique_ptr<Engine> make_reference_engine(const DeviceModel &dm, const vk_options &o, cudaStream_t s);
std::unique_ptr<Engine> make_halpern_engine(const DeviceModel &dm, const vk_options &o, cudaStream_t s);

// Grid for a one-thread-per-element kernel (no grid-stride loop): covers n.
inline int grid1d(int64_t n, int threads = 256) {
    const int64_t b = (n + threads - 1) / threads;
    return static_cast<int>(b > 0 ? b : 1);
}

// Deterministic reduction of per-tile partial sums: out[r] = sum_t partials[t*R + r].
void reduce_partials(const double *partials, int ntiles, int R, double *out, cudaStream_t s);

inline double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Host-side phase timings on stderr when vk_options::verbose > 0
// (`stream` is synchronized first so device work is attributed to its phase).
class PhaseLog {
public:
    PhaseLog(int verbose, const char *who, cudaStream_t s) : on_(verbose > 0), who_(who), s_(s) {}
    void mark(const char *what) {
        if (!on_) return;
        cudaStreamSynchronize(s_);
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "[vikalp_b200] %s: %-28s %8.3f s\n", who_, what,
                     std::chrono::duration<double>(now - t_).count());
        t_ = now;
    }
    void stream(cudaStream_t s) { s_ = s; }

private:
    bool on_;
    const char *who_;
    cudaStream_t s_;
    std::chrono::steady_clock::time_point t_ = std::chrono::steady_clock::now();
};

} // namespace vk
