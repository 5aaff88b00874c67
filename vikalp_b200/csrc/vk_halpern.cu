// Restarted reflected-Halpern PDHG (VK_ALGO_HALPERN), FP64 or FP32-mixed.
//
// Problem (scaled by diagonal R, D: K = R A D, c^ = D c, bounds / D, row
// bounds * R):   min c'x  s.t.  rl <= K x <= ru,  l <= x <= u,
// with the reference's sign convention for y (y > 0 <=> upper row active,
// SolveResult.hpp:31-33). One PDHG step T(x, y) with tau = eta/omega,
// sigma = eta*omega:
//   x^ = clamp(x - tau (c + K'y), l, u)
//   y^ = v - clamp(v, sigma rl, sigma ru),  v = y + sigma K (2 x^ - x)
// and the reflected Halpern update towards the anchor z0 (the last restart
// point), with lambda = (k+1)/(k+2), k = iterations since the restart:
//   z <- lambda (2 T(z) - z) + (1 - lambda) z0.
// Each iteration is two fused passes (no other kernel):
//   column pass over K' (gathers y):  x^, xbar = 2x^ - x, x <- Halpern
//   row pass over K (gathers xbar):   y^, y <- Halpern
// Every `check_every` iterations the last iteration also stores (x^, y^) and
// the squared step lengths; two more passes give K x^ and K'y^, and one
// control kernel -- all on the device, no host round trip -- evaluates the
// relative KKT error of (x^, y^) in ORIGINAL units (primal residual, dual
// residual, duality gap), stops when it is below the tolerance, and otherwise
// applies the restart rule on the fixed-point residual
//   r = sqrt(omega |x^ - x|^2 + |y^ - y|^2 / omega)
// (restart when r <= 0.2 r_restart, or r <= 0.8 r_restart and r grew since the
// previous check, or k >= 0.2 * total iterations; PrimalWeightRule,
// vk_engine.cuh), restarting at (x^, y^) and updating the primal weight omega
// by the smoothed (theta = 0.2) log-ratio of the moves of the restart points.
// The chunk of check_every iterations is one CUDA graph.
//
// Setup: 10 Ruiz infinity-norm passes then one Pock-Chambolle (alpha = 1)
// pass give R and D; eta = 0.99 / sigma_max(K) with sigma_max from power
// iteration; omega_0 = |c^| / |b^|.
//
// MIXED precision keeps K, iterates and products in float32 while every
// reduction (KKT norms, gap, step lengths) and every decision (restart,
// primal weight, stop) is float64; when float32 progress stalls or reaches the
// tolerance, the iterates move to float64 and the float64 engine finishes
// (the polish). The answer is always checked in float64.
#include "vk_engine.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <limits>

namespace vk {
namespace {

constexpr int kRuizPasses = 10;
constexpr int kPowerMax = 200;
constexpr int kColCheckSums = 2;       // |x^-x|^2, |x^-x0|^2
constexpr int kRowCheckSums = 2;       // |y^-y|^2, |y^-y0|^2
constexpr int kKktRowSums = 3;         // primal res^2, dual-obj rows, row-dual violations^2
constexpr int kKktColSums = 5;         // dual res^2, dual-obj cols, primal obj, box violation^2, x'Qx
constexpr int64_t kTunePassesMinNnz = 2000000; // per-pass variant tuning from this many nonzeros

struct HalCtl {
    double eta, omega, tau, sigma;
    double r_restart, r_prev;
    double rel_p, rel_d, rel_gap, kkt;
    double bnorm, cnorm, offset, tol;
    double knorm, lq, rho, pad_d; // sigma_max(K), lambda_max(Q^) (0: LP), reflection
    double theta, freeze;                   // primal-weight smoothing; no update below this KKT
    double beta_suff, beta_nec, beta_art;   // restart thresholds
    long long k_base, total, limit, restarts, checks;
    int done, status, restart_now, pad;
};

// Step sizes for primal weight omega: tau = eta/omega, sigma = eta*omega.
// LP (lq == 0): eta = 0.99/|K| and full reflection rho = 1. QP: the explicit
// gradient step on 0.5 x'Q^x needs 1/tau - sigma |K|^2 >= L; eta solves
// tau L + eta^2 |K|^2 = 0.99^2 and the reflection is cut to
// rho = 0.99 (1 - 1/(2 kappa)), kappa = (1/tau - sigma |K|^2) / L, which keeps
// (1+rho) T - rho I nonexpansive (Condat's bound on the relaxation of the
// primal-dual iteration with a smooth term).
__host__ __device__ inline void step_params(double knorm, double lq, double omega, double &eta, double &rho) {
    if (!(lq > 0.0)) {
        eta = knorm > 0.0 ? 0.99 / knorm : 1.0;
        rho = 1.0;
        return;
    }
    const double k2 = knorm * knorm, b = lq / omega, c = 0.9801;
    eta = 2.0 * c / (b + sqrt(b * b + 4.0 * k2 * c));
    const double tau = eta / omega;
    const double kappa = (1.0 - eta * eta * k2) / (tau * lq);
    rho = fmin(1.0, 0.99 * (1.0 - 1.0 / (2.0 * kappa)));
}

// ---- scaling (FP64, original values) -----------------------------------------

// out_i = max_k |a_k| * s_i * g_{c_k} (mode 0) or sum_k (mode 1); warp per row.
__global__ void scaled_norm_kernel(const int *__restrict__ ro, const int *__restrict__ ci,
                                   const double *__restrict__ v, const double *__restrict__ self,
                                   const double *__restrict__ other, int rows, int mode, double *__restrict__ out) {
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    double acc = 0.0;
    for (int k = ro[r] + lane; k < ro[r + 1]; k += 32) {
        const double a = fabs(v[k]) * other[ci[k]];
        acc = mode == 0 ? fmax(acc, a) : acc + a;
    }
    acc = mode == 0 ? warp_max_nonneg(acc) : warp_sum(acc);
    if (lane == 0) out[r] = acc * self[r];
}

__global__ void rescale_kernel(double *__restrict__ s, const double *__restrict__ norm, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && norm[i] > 0.0) s[i] /= sqrt(norm[i]);
}

template <class T>
__global__ void scale_matrix_kernel(const int *__restrict__ ro, const int *__restrict__ ci,
                                    const double *__restrict__ v, const double *__restrict__ rs,
                                    const double *__restrict__ cs, int rows, bool transposed, T *__restrict__ out) {
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    for (int k = ro[r] + lane; k < ro[r + 1]; k += 32) {
        const int c = ci[k];
        out[k] = static_cast<T>(transposed ? v[k] * rs[c] * cs[r] : v[k] * rs[r] * cs[c]);
    }
}

template <class T>
__global__ void scale_vec_kernel(const double *__restrict__ a, const double *__restrict__ s, int n, int mode,
                                 T *__restrict__ out) {
    // mode 0: a*s, 1: a/s (infinite entries kept), 2: a*s (infinite kept)
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = a[i];
    double r;
    if (mode == 0)
        r = v * s[i];
    else if (!isfinite(v))
        r = v;
    else
        r = mode == 1 ? v / s[i] : v * s[i];
    out[i] = static_cast<T>(r);
}

template <class TD, class TS>
__global__ void convert_kernel(const TS *__restrict__ a, int n, TD *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<TD>(a[i]);
}

// Deterministic sum of squares / dot: per-block partials then reduce_partials.
template <class T>
__global__ void dot_kernel(const T *__restrict__ a, const T *__restrict__ b, int n, double *__restrict__ partial) {
    __shared__ double scratch[32];
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        s += static_cast<double>(a[i]) * static_cast<double>(b[i]);
    double v[1] = {s};
    block_sum<1>(v, scratch);
    if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

template <class T>
__global__ void scal_kernel(T *__restrict__ a, int n, const double *__restrict__ nrm2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double s = *nrm2 > 0.0 ? 1.0 / sqrt(*nrm2) : 1.0;
    if (i < n) a[i] = static_cast<T>(a[i] * s);
}

// the power iteration's start vector, a hash of each column's index in the
// caller's order (perm: device column -> caller's column, or nullptr), so a
// renamed model starts from the same vector
__global__ void seed_kernel(double *a, int n, const int *__restrict__ perm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        unsigned h = static_cast<unsigned>(perm ? perm[i] : i) * 2654435761u + 12345u;
        h ^= h >> 13;
        h *= 2246822519u;
        h ^= h >> 16;
        a[i] = 0.5 + static_cast<double>(h & 0xffff) / 65536.0;
    }
}

// ---- iteration epilogues -------------------------------------------------------

__device__ __forceinline__ double halpern_lambda(const HalCtl *c, int it) {
    const double k = static_cast<double>(c->k_base + it);
    return (k + 1.0) / (k + 2.0);
}

// Columns (gathers y): qx = Q^ x from the preceding Q pass (QP) or null (LP).
template <class T, bool CHECK>
struct HalColEpi : EpiBase<T> {
    static constexpr int NR = CHECK ? kColCheckSums : 1;
    const HalCtl *ctl;
    int it;
    T *x, *xbar, *xhat;
    const T *x0, *c, *l, *u, *qx;
    double *partials;
    struct Pre {
        T x, x0, c, l, u, q;
    };
    __device__ bool skip() const { return ctl->done != 0; }
    __device__ Pre load(int j) const { return Pre{x[j], x0[j], c[j], l[j], u[j], qx ? qx[j] : T(0)}; }
    __device__ void row_pre(int j, const T (&s)[1], const Pre &p, double (&red)[NR]) const {
        const T tau = static_cast<T>(ctl->tau);
        const T rho = static_cast<T>(ctl->rho);
        const T lam = static_cast<T>(halpern_lambda(ctl, it));
        const T xh = clampbox(p.x - tau * (p.c + p.q + s[0]), p.l, p.u);
        const T xb = T(2) * xh - p.x;
        xbar[j] = xb;
        x[j] = lam * ((T(1) + rho) * xh - rho * p.x) + (T(1) - lam) * p.x0;
        if (CHECK) {
            xhat[j] = xh;
            const double d0 = static_cast<double>(xh) - static_cast<double>(p.x);
            const double d1 = static_cast<double>(xh) - static_cast<double>(p.x0);
            red[0] += d0 * d0;
            red[CHECK ? 1 : 0] += d1 * d1;
        }
    }
    __device__ void finish(double (&red)[NR], double *scratch, int block) const {
        if (!CHECK) return;
        block_sum<NR>(red, scratch);
        if (threadIdx.x == 0)
            for (int r = 0; r < NR; ++r) partials[(size_t)block * NR + r] = red[r];
    }
};

template <class T, bool CHECK>
struct HalRowEpi : EpiBase<T> {
    static constexpr int NR = CHECK ? kRowCheckSums : 1;
    const HalCtl *ctl;
    int it;
    T *y, *yhat;
    const T *y0, *rl, *ru;
    double *partials;
    struct Pre {
        T y, y0, rl, ru;
    };
    __device__ bool skip() const { return ctl->done != 0; }
    __device__ Pre load(int i) const { return Pre{y[i], y0[i], rl[i], ru[i]}; }
    __device__ void row_pre(int i, const T (&s)[1], const Pre &p, double (&red)[NR]) const {
        const T sigma = static_cast<T>(ctl->sigma);
        const T rho = static_cast<T>(ctl->rho);
        const T lam = static_cast<T>(halpern_lambda(ctl, it));
        const T v = p.y + sigma * s[0];
        const T yh = v - clampbox(v, sigma * p.rl, sigma * p.ru);
        y[i] = lam * ((T(1) + rho) * yh - rho * p.y) + (T(1) - lam) * p.y0;
        if (CHECK) {
            yhat[i] = yh;
            const double d0 = static_cast<double>(yh) - static_cast<double>(p.y);
            const double d1 = static_cast<double>(yh) - static_cast<double>(p.y0);
            red[0] += d0 * d0;
            red[CHECK ? 1 : 0] += d1 * d1;
        }
    }
    __device__ void finish(double (&red)[NR], double *scratch, int block) const {
        if (!CHECK) return;
        block_sum<NR>(red, scratch);
        if (threadIdx.x == 0)
            for (int r = 0; r < NR; ++r) partials[(size_t)block * NR + r] = red[r];
    }
};

// Relative-KKT pieces of (x^, y^) in original units (rows: gathers x^).
template <class T>
struct KktRowEpi : EpiBase<T> {
    static constexpr int NR = kKktRowSums;
    const HalCtl *ctl;
    const T *yhat, *rl, *ru, *rs;
    double *partials;
    struct Pre {
        T y, rl, ru, r;
    };
    __device__ bool skip() const { return ctl->done != 0; }
    __device__ Pre load(int i) const { return Pre{yhat[i], rl[i], ru[i], rs[i]}; }
    __device__ void row_pre(int, const T (&s)[1], const Pre &p, double (&red)[NR]) const {
        const double a = static_cast<double>(s[0]);
        const double lo = static_cast<double>(p.rl), hi = static_cast<double>(p.ru), r = static_cast<double>(p.r);
        const double pr = (a - clampbox(a, lo, hi)) / r;
        red[0] += pr * pr;
        const double y = static_cast<double>(p.y);
        const double yl = smax(0.0, -y), yu = smax(0.0, y);
        if (yl > 0.0) {
            if (isfinite(lo)) red[1] += lo * yl; else red[2] += (r * yl) * (r * yl);
        }
        if (yu > 0.0) {
            if (isfinite(hi)) red[1] -= hi * yu; else red[2] += (r * yu) * (r * yu);
        }
    }
    __device__ void finish(double (&red)[NR], double *scratch, int block) const {
        block_sum<NR>(red, scratch);
        if (threadIdx.x == 0)
            for (int r = 0; r < NR; ++r) partials[(size_t)block * NR + r] = red[r];
    }
};

// Columns: gathers y^; lambda^ = c^ + Q^x^ + K'y^, lambda = lambda^ / D
// (qx = Q^ x^ from a Q pass, null for an LP).
template <class T>
struct KktColEpi : EpiBase<T> {
    static constexpr int NR = kKktColSums;
    const HalCtl *ctl;
    const T *xhat, *c, *l, *u, *cs, *qx;
    double *partials;
    struct Pre {
        T x, c, l, u, d, q;
    };
    __device__ bool skip() const { return ctl->done != 0; }
    __device__ Pre load(int j) const { return Pre{xhat[j], c[j], l[j], u[j], cs[j], qx ? qx[j] : T(0)}; }
    __device__ void row_pre(int, const T (&s)[1], const Pre &p, double (&red)[NR]) const {
        const double q = static_cast<double>(p.q);
        const double lam = static_cast<double>(p.c) + q + static_cast<double>(s[0]);
        const double d = static_cast<double>(p.d);
        const double lo = static_cast<double>(p.l), hi = static_cast<double>(p.u), x = static_cast<double>(p.x);
        const double vl = smax(0.0, lam), vu = smax(0.0, -lam);
        if (vl > 0.0) {
            if (isfinite(lo)) red[1] += lo * vl; else red[0] += (vl / d) * (vl / d);
        }
        if (vu > 0.0) {
            if (isfinite(hi)) red[1] -= hi * vu; else red[0] += (vu / d) * (vu / d);
        }
        red[2] += static_cast<double>(p.c) * x;
        const double bx = (x - clampbox(x, lo, hi)) * d;
        red[3] += bx * bx;
        red[4] += x * q;
    }
    __device__ void finish(double (&red)[NR], double *scratch, int block) const {
        block_sum<NR>(red, scratch);
        if (threadIdx.x == 0)
            for (int r = 0; r < NR; ++r) partials[(size_t)block * NR + r] = red[r];
    }
};

// qx = Q^ v, skipped once the solve is done.
template <class T>
struct QStore : EpiRow<T, QStore<T>> {
    const HalCtl *ctl;
    T *y;
    __device__ bool skip() const { return ctl->done != 0; }
    __device__ void row(int i, const T (&s)[1], double (&)[1]) const { y[i] = s[0]; }
};

template <class T>
struct PlainStore : EpiRow<T, PlainStore<T>> {
    T *y;
    __device__ void row(int i, const T (&s)[1], double (&)[1]) const { y[i] = s[0]; }
};

// Partial-sum reduction of one check, then the stop / restart / primal-weight
// decisions. One block of 1024 threads; fixed order, so deterministic.
struct CheckGrids {
    int col, row, kkt_row, kkt_col;
};

__device__ double block_reduce_range(const double *p, int count, int R, int r, double *scratch) {
    double v = 0.0;
    for (int t = threadIdx.x; t < count; t += blockDim.x) v += p[(size_t)t * R + r];
    double a[1] = {v};
    block_sum<1>(a, scratch);
    __syncthreads();
    return a[0]; // valid in thread 0
}

constexpr int kControlThreads = 256;

__global__ void __launch_bounds__(kControlThreads)
    check_control_kernel(HalCtl *ctl, const double *pc, const double *pr, const double *pkr, const double *pkc,
                         CheckGrids g, int chunk) {
    __shared__ double scratch[32];
    __shared__ int skip;
    if (threadIdx.x == 0) skip = ctl->done;
    __syncthreads();
    if (skip) return;
    double s[kColCheckSums + kRowCheckSums + kKktRowSums + kKktColSums];
    int o = 0;
    for (int r = 0; r < kColCheckSums; ++r) s[o++] = block_reduce_range(pc, g.col, kColCheckSums, r, scratch);
    for (int r = 0; r < kRowCheckSums; ++r) s[o++] = block_reduce_range(pr, g.row, kRowCheckSums, r, scratch);
    for (int r = 0; r < kKktRowSums; ++r) s[o++] = block_reduce_range(pkr, g.kkt_row, kKktRowSums, r, scratch);
    for (int r = 0; r < kKktColSums; ++r) s[o++] = block_reduce_range(pkc, g.kkt_col, kKktColSums, r, scratch);
    if (threadIdx.x != 0) return;
    HalCtl c = *ctl;
    const double dx2 = s[0], dx0 = s[1], dy2 = s[2], dy0 = s[3];
    const double rp2 = s[4], dobj_r = s[5], viol2 = s[6];
    const double rd2 = s[7], dobj_c = s[8], box2 = s[10], quad = s[11];
    const double pobj = s[9] + 0.5 * quad + c.offset;
    const double dobj = dobj_r + dobj_c - 0.5 * quad + c.offset;
    c.total += chunk;
    c.checks += 1;
    c.rel_p = (sqrt(rp2) + sqrt(box2)) / (1.0 + c.bnorm);
    c.rel_d = sqrt(rd2 + viol2) / (1.0 + c.cnorm);
    c.rel_gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    c.kkt = smax(smax(c.rel_p, c.rel_d), c.rel_gap);
    c.restart_now = 0;
    if (!(c.kkt == c.kkt)) { // NaN: stop, the host reports a numerical failure
        c.done = 1;
        c.status = VK_STATUS_NUMERICAL_FAILURE;
    } else if (c.kkt <= c.tol) {
        c.done = 1;
        c.status = VK_STATUS_OPTIMAL;
    } else if (c.total >= c.limit) {
        c.done = 1;
        c.status = VK_STATUS_ITERATION_LIMIT;
    } else {
        const double r = sqrt(c.omega * dx2 + dy2 / c.omega);
        const long long k = c.k_base + chunk;
        bool restart = false;
        if (c.r_restart < 0.0) {
            c.r_restart = r;
        } else {
            restart = (r <= c.beta_suff * c.r_restart) || (r <= c.beta_nec * c.r_restart && r > c.r_prev) ||
                      (static_cast<double>(k) >= c.beta_art * static_cast<double>(c.total));
        }
        c.r_prev = r;
        if (restart) {
            const double mx = sqrt(dx0), my = sqrt(dy0);
            if (mx > 1e-10 && my > 1e-10 && c.theta > 0.0 && c.kkt >= c.freeze)
                c.omega = exp(c.theta * log(my / mx) + (1.0 - c.theta) * log(c.omega));
            step_params(c.knorm, c.lq, c.omega, c.eta, c.rho);
            c.tau = c.eta / c.omega;
            c.sigma = c.eta * c.omega;
            c.k_base = 0;
            c.restarts += 1;
            c.restart_now = 1;
            c.r_restart = r;
        } else {
            c.k_base = k;
        }
    }
    *ctl = c;
}

struct KktEval {
    double rel_p, rel_d, rel_gap, kkt;
};

// The relative KKT error of the KKT passes' partial sums (the evaluation part
// of check_control_kernel, without any decision). One block.
__global__ void __launch_bounds__(kControlThreads)
    kkt_eval_kernel(const HalCtl *ctl, const double *pkr, const double *pkc, int grid_row, int grid_col,
                    KktEval *out) {
    __shared__ double scratch[32];
    double s[kKktRowSums + kKktColSums];
    int o = 0;
    for (int r = 0; r < kKktRowSums; ++r) s[o++] = block_reduce_range(pkr, grid_row, kKktRowSums, r, scratch);
    for (int r = 0; r < kKktColSums; ++r) s[o++] = block_reduce_range(pkc, grid_col, kKktColSums, r, scratch);
    if (threadIdx.x != 0) return;
    const HalCtl &c = *ctl;
    const double rp2 = s[0], dobj_r = s[1], viol2 = s[2];
    const double rd2 = s[3], dobj_c = s[4], box2 = s[6], quad = s[7];
    const double pobj = s[5] + 0.5 * quad + c.offset;
    const double dobj = dobj_r + dobj_c - 0.5 * quad + c.offset;
    KktEval e;
    e.rel_p = (sqrt(rp2) + sqrt(box2)) / (1.0 + c.bnorm);
    e.rel_d = sqrt(rd2 + viol2) / (1.0 + c.cnorm);
    e.rel_gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    e.kkt = smax(smax(e.rel_p, e.rel_d), e.rel_gap);
    if (!(e.kkt == e.kkt)) e.kkt = std::numeric_limits<double>::infinity();
    *out = e;
}

template <class T>
__global__ void restart_apply_kernel(const HalCtl *ctl, T *x, T *x0, const T *xhat, int n, T *y, T *y0,
                                     const T *yhat, int m) {
    if (!ctl->restart_now || ctl->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        x[i] = xhat[i];
        x0[i] = xhat[i];
    }
    if (i < m) {
        y[i] = yhat[i];
        y0[i] = yhat[i];
    }
}

template <class T>
__global__ void prepare_kernel(const double *__restrict__ warm, const double *__restrict__ lo,
                               const double *__restrict__ hi, const double *__restrict__ cs, int n, T *__restrict__ l,
                               T *__restrict__ u, T *__restrict__ x, T *__restrict__ x0) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double d = cs[j];
    const double lj = isfinite(lo[j]) ? lo[j] / d : lo[j];
    const double uj = isfinite(hi[j]) ? hi[j] / d : hi[j];
    l[j] = static_cast<T>(lj);
    u[j] = static_cast<T>(uj);
    const double xv = clampbox(warm ? warm[j] / d : 0.0, lj, uj);
    x[j] = static_cast<T>(xv);
    x0[j] = static_cast<T>(xv);
}

template <class T>
__global__ void unscale_out_kernel(const T *__restrict__ a, const double *__restrict__ s, int n,
                                   double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<double>(a[i]) * s[i];
}

// ---- engine ---------------------------------------------------------------------

template <class T>
struct HalState {
    int m = 0, n = 0;
    DevBuf<T> ka, kat;                      // K values, CSR and transposed order
    DevBuf<T> c, l, u, rl, ru, rs, cs;      // scaled data and the scales
    DevBuf<T> x, x0, xbar, xhat, y, y0, yhat;
    DevBuf<T> q, qx;                        // QP: Q^ = D Q D values, Q^ x
};

class HalpernEngine final : public Engine {
public:
    HalpernEngine(const DeviceModel &dm, const vk_options &o, cudaStream_t s) : dm_(dm), o_(o), s_(s) {
        mixed_ = o.precision == VK_PREC_MIXED;
        chunk_ = std::max(2, o.check_every > 0 ? o.check_every : 64);
        const int m = dm.m, n = dm.n;
        PhaseLog log(o.verbose, "halpern setup", s);
        rs_.reset(m > 0 ? m : 1);
        cs_.reset(n);
        compute_scaling();
        log.mark("scaling");
        setup_state(s64_);
        if (mixed_) setup_state(s32_);
        log.mark("scaled state");
        step_size();
        log.mark("step size (power iteration)");
        ctl_.reset(1);
        evalctl_.reset(1);
        evalout_.reset(1);
        hctl_.reset(1);
        pc_.reset(static_cast<size_t>(kMaxGrid) * kColCheckSums);
        pr_.reset(static_cast<size_t>(kMaxGrid) * kRowCheckSums);
        pkr_.reset(static_cast<size_t>(kMaxGrid) * kKktRowSums);
        pkc_.reset(static_cast<size_t>(kMaxGrid) * kKktColSums);
    }

    ~HalpernEngine() override {
        if (g64_) cudaGraphExecDestroy(g64_);
        if (g32_) cudaGraphExecDestroy(g32_);
    }

    void run(const double *d_warm, const double *d_lo, const double *d_hi, double *d_xo, double *d_yo, RunInfo &info,
             std::chrono::steady_clock::time_point started) override {
        start(d_warm, d_lo, d_hi);
        if (!tuned_) {
            // once per model, before the graphs are captured; the passes
            // overwrite the start, so it is set up again afterwards
            tuned_ = true;
            tune_passes(s64_, 0);
            if (mixed_) {
                copy_state<float, double>(s64_, s32_);
                tune_passes(s32_, 1);
            }
            start(d_warm, d_lo, d_hi);
        }
        run_chunks(d_xo, d_yo, info, started);
    }

    // The solve's start: scaled bounds and start in float64 (copied into the
    // float32 state when mixed), zero duals, a fresh control block.
    void start(const double *d_warm, const double *d_lo, const double *d_hi) {
        const int m = dm_.m, n = dm_.n;
        prepare_kernel<double><<<grid1d(n), 256, 0, s_>>>(d_warm, d_lo, d_hi, cs_.get(), n, s64_.l.get(),
                                                          s64_.u.get(), s64_.x.get(), s64_.x0.get());
        VK_LAUNCH_CHECK();
        if (m > 0) {
            VK_CUDA(cudaMemsetAsync(s64_.y.get(), 0, m * sizeof(double), s_));
            VK_CUDA(cudaMemsetAsync(s64_.y0.get(), 0, m * sizeof(double), s_));
        }
        HalCtl c{};
        c.knorm = knorm_;
        c.lq = lq_;
        const PrimalWeightRule pw = primal_weight_rule();
        c.omega = omega0_ * pw.start;
        c.theta = pw.theta;
        c.freeze = pw.freeze;
        c.beta_suff = pw.beta_suff;
        c.beta_nec = pw.beta_nec;
        c.beta_art = pw.beta_art;
        step_params(c.knorm, c.lq, c.omega, c.eta, c.rho);
        c.tau = c.eta / c.omega;
        c.sigma = c.eta * c.omega;
        c.r_restart = -1.0;
        c.r_prev = std::numeric_limits<double>::infinity();
        c.bnorm = bnorm_;
        c.cnorm = cnorm_;
        c.offset = dm_.offset;
        c.tol = o_.relative_tolerance;
        c.limit = o_.iteration_limit;
        c.status = VK_STATUS_NOT_SOLVED;
        c.kkt = std::numeric_limits<double>::infinity();
        put_control(c);
    }

    // Times every FAST kernel variant on the two fused iteration passes of
    // one precision (q: 0 float64, 1 float32) and keeps the fastest for each:
    // their epilogues set the register pressure, so the plain product's
    // choice need not carry over (tune_variants: interleaved rounds, the
    // clearly slower variants dropped after the first). Models below
    // kTunePassesMinNnz keep the plain product's variant: there the tuning
    // (~150 timed launches, the first of each kernel loading its module)
    // costs as much as a whole solve.
    template <class T>
    void tune_passes(HalState<T> &st, int q) {
        if (forced_variant() >= 0 || dm_.nnz < kTunePassesMinNnz) return;
        for (int pass = 0; pass < (st.m > 0 ? 2 : 1); ++pass) {
            int &var = pass == 0 ? col_var_[q] : row_var_[q];
            // cached per matrix and precision for the process (tuned_pick)
            const uint64_t key = tune_key(dm_.a.fp,
                                          pass == 1 ? "halpern row pass"
                                          : dm_.qp  ? "halpern column pass, qp"
                                                    : "halpern column pass",
                                          sizeof(T));
            if (cached_pick(key, var)) continue;
            auto launch = [&](int v) {
                var = v;
                if (pass == 0)
                    col_pass<T, false>(st, 0);
                else
                    row_pass<T, false>(st, 0);
            };
            float best[kFastVariants];
            const int pick = store_pick(key, tune_variants(launch, s_, best));
            var = pick;
            if (o_.verbose > 0) {
                std::fprintf(stderr, "[vikalp_b200] halpern %s %s pass variants (ms, best timed round):",
                             q == 0 ? "float64" : "float32", pass == 0 ? "column" : "row");
                for (int v = 0; v < kFastVariants; ++v) std::fprintf(stderr, " %d:%.4f", v, best[v]);
                std::fprintf(stderr, " -> %d\n", var);
            }
        }
        check_device_error(s_);
    }

    void run_chunks(double *d_xo, double *d_yo, RunInfo &info, std::chrono::steady_clock::time_point started) {
        const int m = dm_.m, n = dm_.n;
        cudaEvent_t e0, e1;
        VK_CUDA(cudaEventCreate(&e0));
        VK_CUDA(cudaEventCreate(&e1));
        VK_CUDA(cudaEventRecord(e0, s_));
        launches_ = 0;
        bool timed_out = false;
        long long fp32_iters = 0;
        bool confirmed = false; // mixed: the float32 answer passed the float64 evaluation
        if (mixed_) {
            copy_state<float, double>(s64_, s32_);
            if (!g32_) g32_ = capture(s32_);
            // float32 phase. When its own (float32) KKT evaluation reaches the
            // tolerance, the point is evaluated again in float64 with no
            // float64 iteration: accepted there, the solve ends; otherwise the
            // float32 target is halved (down to kFp32Floor, about the noise of
            // a float32 evaluation) and the float32 iterations go on. The
            // phase also ends on the limit, or on a plateau: over a window of
            // max(32 checks, an eighth of the checks so far) the best float32
            // KKT error, once below kPlateauFrom, improved by less than
            // kPlateauGain.
            constexpr double kFp32Floor = 1e-7;
            constexpr double kPlateauGain = 1.25;
            constexpr double kPlateauFrom = 1e-3; // early stalls (restart transients) do not count
            double best = std::numeric_limits<double>::infinity();
            double win_best = best;   // best at the window's start
            long long win_start = 0;  // check count at the window's start
            double target = o_.relative_tolerance;
            for (;;) {
                if (over_time(started)) {
                    timed_out = true;
                    break;
                }
                poll_chunk(g32_);
                HalCtl h = hctl_[0];
                if (h.done) {
                    if (h.status != VK_STATUS_OPTIMAL) break;
                    const double k64 = evaluate64();
                    if (o_.verbose > 0)
                        std::fprintf(stderr,
                                     "[vikalp_b200] mixed: float32 KKT %.3e <= target %.3e at %lld iterations; "
                                     "float64 evaluation %.3e\n",
                                     h.kkt, target, h.total, k64);
                    if (k64 <= o_.relative_tolerance) {
                        confirmed = true;
                        break;
                    }
                    if (target * 0.5 < kFp32Floor) break;
                    target *= 0.5;
                    h.done = 0;
                    h.status = VK_STATUS_NOT_SOLVED;
                    h.tol = target;
                    put_control(h);
                    continue;
                }
                best = std::min(best, h.kkt);
                if (h.checks - win_start >= std::max<long long>(32, h.checks / 8)) {
                    if (best < kPlateauFrom && best * kPlateauGain > win_best) {
                        if (o_.verbose > 0)
                            std::fprintf(stderr,
                                         "[vikalp_b200] mixed: float32 plateau at KKT %.3e (best %.3e, %.3e a "
                                         "window earlier) after %lld iterations; float64 from here\n",
                                         h.kkt, best, win_best, h.total);
                        break;
                    }
                    win_start = h.checks;
                    win_best = best;
                }
            }
            fp32_iters = hctl_[0].total;
            // hand the float32 state to float64 and re-open the control block
            copy_state<double, float>(s32_, s64_);
            HalCtl h = hctl_[0];
            if (confirmed) {
                h.done = 1;
                h.status = VK_STATUS_OPTIMAL;
                h.kkt = k64_.kkt;
                h.rel_p = k64_.rel_p;
                h.rel_d = k64_.rel_d;
                h.rel_gap = k64_.rel_gap;
                put_control(h);
            } else if (h.status == VK_STATUS_OPTIMAL || h.status == VK_STATUS_NOT_SOLVED ||
                       h.status == VK_STATUS_ITERATION_LIMIT) {
                h.done = 0;
                h.status = VK_STATUS_NOT_SOLVED;
                h.tol = o_.relative_tolerance;
                h.limit = o_.iteration_limit + std::max<long long>(chunk_, 0); // the polish gets at least one check
                put_control(h);
            }
        }
        if (!timed_out && !confirmed) {
            if (!g64_) g64_ = capture(s64_);
            for (;;) {
                if (over_time(started)) {
                    timed_out = true;
                    break;
                }
                poll_chunk(g64_);
                if (hctl_[0].done) break;
            }
        }
        VK_CUDA(cudaEventRecord(e1, s_));
        VK_CUDA(cudaMemcpyAsync(hctl_.get(), ctl_.get(), sizeof(HalCtl), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaStreamSynchronize(s_));
        float ms = 0.f;
        VK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        const HalCtl &h = hctl_[0];
        info.iterations = h.total;
        info.restarts = h.restarts;
        info.last_metric = h.kkt;
        info.fp32_iterations = fp32_iters;
        info.kernel_launches = launches_;
        info.status = (timed_out && !h.done) ? VK_STATUS_TIME_LIMIT : h.status;
        info.iterate_seconds = ms * 1e-3;
        // the answer is the last PDHG output (x^, y^) in float64
        const bool have_hat = h.checks > 0;
        unscale_out_kernel<double><<<grid1d(n), 256, 0, s_>>>(have_hat ? s64_.xhat.get() : s64_.x.get(), cs_.get(),
                                                              n, d_xo);
        if (m > 0)
            unscale_out_kernel<double><<<grid1d(m), 256, 0, s_>>>(have_hat ? s64_.yhat.get() : s64_.y.get(),
                                                                  rs_.get(), m, d_yo);
        VK_LAUNCH_CHECK();
    }

    void set_limits(const vk_options &o) override { o_ = o; }

private:
    // Writes a control block to the device from the pinned host copy (later
    // reads of it on the stream, poll_chunk's included, are ordered after).
    void put_control(const HalCtl &h) {
        hctl_[0] = h;
        VK_CUDA(cudaMemcpyAsync(ctl_.get(), hctl_.get(), sizeof(HalCtl), cudaMemcpyHostToDevice, s_));
    }

    // Relative KKT error, in float64, of the float32 state's last (x^, y^):
    // converted to float64, then the two float64 KKT passes and one
    // evaluation kernel -- no iteration. Leaves the float64 x^, y^ in place.
    double evaluate64() {
        const int m = dm_.m, n = dm_.n;
        convert_kernel<double, float><<<grid1d(n), 256, 0, s_>>>(s32_.xhat.get(), n, s64_.xhat.get());
        if (m > 0) convert_kernel<double, float><<<grid1d(m), 256, 0, s_>>>(s32_.yhat.get(), m, s64_.yhat.get());
        VK_LAUNCH_CHECK();
        HalCtl e = hctl_[0]; // its norms and offset; done = 0 so the passes run
        e.done = 0;
        VK_CUDA(cudaMemcpyAsync(evalctl_.get(), &e, sizeof(e), cudaMemcpyHostToDevice, s_));
        int grid_col = 0;
        const int grid_row = kkt_passes(s64_, grid_col, evalctl_.get());
        kkt_eval_kernel<<<1, kControlThreads, 0, s_>>>(evalctl_.get(), pkr_.get(), pkc_.get(), grid_row, grid_col,
                                                      evalout_.get());
        VK_LAUNCH_CHECK();
        VK_CUDA(cudaMemcpyAsync(&k64_, evalout_.get(), sizeof(KktEval), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaStreamSynchronize(s_));
        check_device_error(s_);
        return k64_.kkt;
    }

    bool over_time(std::chrono::steady_clock::time_point t0) const {
        return std::isfinite(o_.time_limit_seconds) && seconds_since(t0) >= o_.time_limit_seconds;
    }

    void poll_chunk(cudaGraphExec_t g) {
        VK_CUDA(cudaGraphLaunch(g, s_));
        launches_ += graph_nodes_;
        VK_CUDA(cudaMemcpyAsync(hctl_.get(), ctl_.get(), sizeof(HalCtl), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaStreamSynchronize(s_));
        check_device_error(s_);
        if (o_.verbose >= 2) { // per-check trace
            const HalCtl &h = hctl_[0];
            std::fprintf(stderr, "[vikalp_b200] halpern %lld kkt %.3e p %.2e d %.2e gap %.2e omega %.4g restarts %lld\n",
                         h.total, h.kkt, h.rel_p, h.rel_d, h.rel_gap, h.omega / omega0_, h.restarts);
        }
    }

    // Ruiz (infinity norm) passes, then one Pock-Chambolle (alpha = 1) pass.
    void compute_scaling() {
        const int m = dm_.m, n = dm_.n;
        auto fill1 = [&](DevBuf<double> &b, int k) {
            std::vector<double> one(k > 0 ? k : 1, 1.0);
            VK_CUDA(cudaMemcpyAsync(b.get(), one.data(), one.size() * sizeof(double), cudaMemcpyHostToDevice, s_));
            VK_CUDA(cudaStreamSynchronize(s_));
        };
        fill1(rs_, m);
        fill1(cs_, n);
        if (dm_.nnz == 0) return;
        DevBuf<double> rn(m), cn(n);
        for (int pass = 0; pass <= kRuizPasses; ++pass) {
            const int mode = pass < kRuizPasses ? 0 : 1;
            scaled_norm_kernel<<<ceil_div(int64_t(m) * 32, 256), 256, 0, s_>>>(
                dm_.a.ro.get(), dm_.a.ci.get(), dm_.a_val.get(), rs_.get(), cs_.get(), m, mode, rn.get());
            scaled_norm_kernel<<<ceil_div(int64_t(n) * 32, 256), 256, 0, s_>>>(
                dm_.at.ro.get(), dm_.at.ci.get(), dm_.at_val.get(), cs_.get(), rs_.get(), n, mode, cn.get());
            VK_LAUNCH_CHECK();
            rescale_kernel<<<grid1d(m), 256, 0, s_>>>(rs_.get(), rn.get(), m);
            rescale_kernel<<<grid1d(n), 256, 0, s_>>>(cs_.get(), cn.get(), n);
            VK_LAUNCH_CHECK();
        }
        VK_CUDA(cudaStreamSynchronize(s_));
    }

    template <class T>
    void setup_state(HalState<T> &st) {
        const int m = dm_.m, n = dm_.n;
        const int mm = m > 0 ? m : 1;
        st.m = m;
        st.n = n;
        st.ka.reset(padded(dm_.nnz));
        st.kat.reset(padded(dm_.nnz));
        if (m > 0)
            scale_matrix_kernel<T><<<ceil_div(int64_t(m) * 32, 256), 256, 0, s_>>>(
                dm_.a.ro.get(), dm_.a.ci.get(), dm_.a_val.get(), rs_.get(), cs_.get(), m, false, st.ka.get());
        scale_matrix_kernel<T><<<ceil_div(int64_t(n) * 32, 256), 256, 0, s_>>>(
            dm_.at.ro.get(), dm_.at.ci.get(), dm_.at_val.get(), rs_.get(), cs_.get(), n, true, st.kat.get());
        for (DevBuf<T> *b : {&st.c, &st.l, &st.u, &st.cs, &st.x, &st.x0, &st.xbar, &st.xhat}) b->reset(n);
        for (DevBuf<T> *b : {&st.rl, &st.ru, &st.rs, &st.y, &st.y0, &st.yhat}) b->reset(mm);
        scale_vec_kernel<T><<<grid1d(n), 256, 0, s_>>>(dm_.c.get(), cs_.get(), n, 0, st.c.get());
        convert_kernel<T, double><<<grid1d(n), 256, 0, s_>>>(cs_.get(), n, st.cs.get());
        if (dm_.qp) {
            // Q^ = D Q D (Q symmetric, so the same column scale on both sides)
            st.q.reset(padded(dm_.q_nnz));
            st.qx.reset(n);
            scale_matrix_kernel<T><<<ceil_div(int64_t(n) * 32, 256), 256, 0, s_>>>(
                dm_.q.ro.get(), dm_.q.ci.get(), dm_.q_val.get(), cs_.get(), cs_.get(), n, false, st.q.get());
            VK_CUDA(cudaMemsetAsync(st.qx.get(), 0, n * sizeof(T), s_));
        }
        if (m > 0) {
            scale_vec_kernel<T><<<grid1d(m), 256, 0, s_>>>(dm_.rl.get(), rs_.get(), m, 2, st.rl.get());
            scale_vec_kernel<T><<<grid1d(m), 256, 0, s_>>>(dm_.ru.get(), rs_.get(), m, 2, st.ru.get());
            convert_kernel<T, double><<<grid1d(m), 256, 0, s_>>>(rs_.get(), m, st.rs.get());
            VK_CUDA(cudaMemsetAsync(st.yhat.get(), 0, m * sizeof(T), s_));
        }
        VK_LAUNCH_CHECK();
        VK_CUDA(cudaStreamSynchronize(s_));
    }

    // eta = 0.99 / sigma_max(K) (power iteration on K'K); omega_0 = |c^| / |b^|;
    // norms of c and b in original units for the relative KKT.
    void step_size() {
        const int m = dm_.m, n = dm_.n;
        DevBuf<double> v(n), w(m > 0 ? m : 1), z(n), part(1024), nrm(1);
        seed_kernel<<<grid1d(n), 256, 0, s_>>>(v.get(), n, dm_.reordered() ? dm_.cperm.get() : nullptr);
        VK_LAUNCH_CHECK();
        auto norm2 = [&](const double *a, int k) {
            dot_kernel<double><<<std::min(1024, grid1d(k)), 256, 0, s_>>>(a, a, k, part.get());
            reduce_partials(part.get(), std::min(1024, grid1d(k)), 1, nrm.get(), s_);
        };
        double sigma_max = 0.0;
        if (dm_.nnz > 0 && m > 0) {
            norm2(v.get(), n);
            scal_kernel<double><<<grid1d(n), 256, 0, s_>>>(v.get(), n, nrm.get());
            double prev = 0.0;
            for (int it = 0; it < kPowerMax; ++it) {
                PlainStore<double> ew;
                ew.y = w.get();
                launch_tiles<double, double, 1, false>(view(dm_.a, s64_.ka.get()), Gathers<double, 1>{{v.get()}}, ew, s_);
                PlainStore<double> ez;
                ez.y = z.get();
                launch_tiles<double, double, 1, false>(view(dm_.at, s64_.kat.get()), Gathers<double, 1>{{w.get()}}, ez,
                                                       s_);
                norm2(z.get(), n);
                double h = 0.0;
                VK_CUDA(cudaMemcpyAsync(&h, nrm.get(), sizeof(double), cudaMemcpyDeviceToHost, s_));
                VK_CUDA(cudaStreamSynchronize(s_));
                const double est = std::sqrt(std::sqrt(h)); // |K'K v| with |v| = 1 -> sigma_max^2
                scal_kernel<double><<<grid1d(n), 256, 0, s_>>>(z.get(), n, nrm.get());
                std::swap(v, z);
                if (it > 10 && std::abs(est - prev) <= 1e-6 * est) {
                    prev = est;
                    break;
                }
                prev = est;
            }
            sigma_max = prev;
        }
        knorm_ = sigma_max;
        // lambda_max(Q^) by power iteration on Q^ (PSD), same start and stopping rule
        lq_ = 0.0;
        if (dm_.qp && dm_.q_nnz > 0) {
            seed_kernel<<<grid1d(n), 256, 0, s_>>>(v.get(), n, dm_.reordered() ? dm_.cperm.get() : nullptr);
            norm2(v.get(), n);
            scal_kernel<double><<<grid1d(n), 256, 0, s_>>>(v.get(), n, nrm.get());
            double prev = 0.0;
            for (int it = 0; it < kPowerMax; ++it) {
                PlainStore<double> ez;
                ez.y = z.get();
                launch_tiles<double, double, 1, false>(view(dm_.q, s64_.q.get()), Gathers<double, 1>{{v.get()}}, ez, s_);
                norm2(z.get(), n);
                double h = 0.0;
                VK_CUDA(cudaMemcpyAsync(&h, nrm.get(), sizeof(double), cudaMemcpyDeviceToHost, s_));
                VK_CUDA(cudaStreamSynchronize(s_));
                const double est = std::sqrt(h); // |Q^ v| with |v| = 1
                scal_kernel<double><<<grid1d(n), 256, 0, s_>>>(z.get(), n, nrm.get());
                std::swap(v, z);
                if (it > 10 && std::abs(est - prev) <= 1e-6 * est) {
                    prev = est;
                    break;
                }
                prev = est;
            }
            lq_ = prev;
        }
        // |c^| and |b^| (scaled) for omega_0; |c| and |b| original for the KKT scales
        std::vector<double> hc(n), hrl(m), hru(m), hcs(n), hrs(m);
        VK_CUDA(cudaMemcpyAsync(hcs.data(), cs_.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(hc.data(), dm_.c.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s_)); // device order
        if (m > 0) {
            VK_CUDA(cudaMemcpyAsync(hrs.data(), rs_.get(), m * sizeof(double), cudaMemcpyDeviceToHost, s_));
            VK_CUDA(cudaMemcpyAsync(hrl.data(), dm_.rl.get(), m * sizeof(double), cudaMemcpyDeviceToHost, s_));
            VK_CUDA(cudaMemcpyAsync(hru.data(), dm_.ru.get(), m * sizeof(double), cudaMemcpyDeviceToHost, s_));
        }
        VK_CUDA(cudaStreamSynchronize(s_));
        double c2 = 0.0, cs2 = 0.0, b2 = 0.0, bs2 = 0.0;
        for (int j = 0; j < n; ++j) {
            c2 += hc[j] * hc[j];
            const double t = hc[j] * hcs[j];
            cs2 += t * t;
        }
        for (int i = 0; i < m; ++i) {
            double b = 0.0;
            if (std::isfinite(hrl[i])) b = std::max(b, std::abs(hrl[i]));
            if (std::isfinite(hru[i])) b = std::max(b, std::abs(hru[i]));
            b2 += b * b;
            bs2 += (b * hrs[i]) * (b * hrs[i]);
        }
        cnorm_ = std::sqrt(c2);
        bnorm_ = std::sqrt(b2);
        omega0_ = (cs2 > 1e-20 && bs2 > 1e-20) ? std::sqrt(cs2) / std::sqrt(bs2) : 1.0;
    }

    // Iterates (and, going to float32, the per-solve bounds) from one state to
    // the other. The float64 bounds are never overwritten by rounded ones.
    template <class TD, class TS>
    void copy_state(const HalState<TS> &a, HalState<TD> &b) {
        const int m = dm_.m, n = dm_.n;
        convert_kernel<TD, TS><<<grid1d(n), 256, 0, s_>>>(a.x.get(), n, b.x.get());
        convert_kernel<TD, TS><<<grid1d(n), 256, 0, s_>>>(a.x0.get(), n, b.x0.get());
        convert_kernel<TD, TS><<<grid1d(n), 256, 0, s_>>>(a.xhat.get(), n, b.xhat.get());
        if (sizeof(TD) < sizeof(TS)) {
            convert_kernel<TD, TS><<<grid1d(n), 256, 0, s_>>>(a.l.get(), n, b.l.get());
            convert_kernel<TD, TS><<<grid1d(n), 256, 0, s_>>>(a.u.get(), n, b.u.get());
        }
        if (m > 0) {
            convert_kernel<TD, TS><<<grid1d(m), 256, 0, s_>>>(a.y.get(), m, b.y.get());
            convert_kernel<TD, TS><<<grid1d(m), 256, 0, s_>>>(a.y0.get(), m, b.y0.get());
            convert_kernel<TD, TS><<<grid1d(m), 256, 0, s_>>>(a.yhat.get(), m, b.yhat.get());
        }
        VK_LAUNCH_CHECK();
    }

    // One chunk of check_every iterations as a CUDA graph.
    template <class T>
    cudaGraphExec_t capture(HalState<T> &st) {
        VK_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
        CheckGrids grids{0, 0, 0, 0};
        for (int it = 0; it < chunk_; ++it) {
            const bool check = it == chunk_ - 1;
            if (check) {
                q_pass(st, st.x.get());
                grids.col = col_pass<T, true>(st, it);
                grids.row = row_pass<T, true>(st, it);
                grids.kkt_row = kkt_passes(st, grids.kkt_col);
                check_control_kernel<<<1, kControlThreads, 0, s_>>>(ctl_.get(), pc_.get(), pr_.get(), pkr_.get(),
                                                                    pkc_.get(), grids, chunk_);
                VK_LAUNCH_CHECK();
                const int mx = std::max(st.m, st.n);
                restart_apply_kernel<T><<<grid1d(mx), 256, 0, s_>>>(ctl_.get(), st.x.get(), st.x0.get(),
                                                                    st.xhat.get(), st.n, st.y.get(), st.y0.get(),
                                                                    st.yhat.get(), st.m);
                VK_LAUNCH_CHECK();
            } else {
                q_pass(st, st.x.get());
                col_pass<T, false>(st, it);
                row_pass<T, false>(st, it);
            }
        }
        cudaGraph_t g;
        VK_CUDA(cudaStreamEndCapture(s_, &g));
        size_t nodes = 0;
        VK_CUDA(cudaGraphGetNodes(g, nullptr, &nodes));
        graph_nodes_ = static_cast<long long>(nodes);
        cudaGraphExec_t ex;
        VK_CUDA(cudaGraphInstantiate(&ex, g, 0));
        cudaGraphDestroy(g);
        return ex;
    }

    // QP: qx = Q^ v (no-op for an LP, and skipped once the solve is done).
    template <class T>
    void q_pass(HalState<T> &st, const T *v, const HalCtl *ctl = nullptr) {
        if (!dm_.qp) return;
        QStore<T> e;
        e.ctl = ctl ? ctl : ctl_.get();
        e.y = st.qx.get();
        launch_tiles<T, T, 1, false>(view(dm_.q, st.q.get()), Gathers<T, 1>{{v}}, e, s_);
    }

    // A pass's matrix view with the variant tuned for it (q: 0 float64, 1 float32).
    template <class T>
    CsrView<T> pass_view(const CsrPattern32 &p, const T *val, int tuned) const {
        CsrView<T> v = view(p, val);
        if (tuned >= 0) v.variant = tuned;
        return v;
    }

    template <class T, bool CHECK>
    int col_pass(HalState<T> &st, int it) {
        HalColEpi<T, CHECK> e;
        e.ctl = ctl_.get();
        e.it = it;
        e.qx = dm_.qp ? st.qx.get() : nullptr;
        e.x = st.x.get();
        e.xbar = st.xbar.get();
        e.xhat = st.xhat.get();
        e.x0 = st.x0.get();
        e.c = st.c.get();
        e.l = st.l.get();
        e.u = st.u.get();
        e.partials = pc_.get();
        const T *yg = st.m > 0 ? st.y.get() : st.x.get();
        return launch_tiles<T, T, 1, false>(pass_view(dm_.at, st.kat.get(), col_var_[sizeof(T) == 4]),
                                            Gathers<T, 1>{{yg}}, e, s_);
    }

    template <class T, bool CHECK>
    int row_pass(HalState<T> &st, int it) {
        if (st.m == 0) return 0;
        HalRowEpi<T, CHECK> e;
        e.ctl = ctl_.get();
        e.it = it;
        e.y = st.y.get();
        e.yhat = st.yhat.get();
        e.y0 = st.y0.get();
        e.rl = st.rl.get();
        e.ru = st.ru.get();
        e.partials = pr_.get();
        return launch_tiles<T, T, 1, false>(pass_view(dm_.a, st.ka.get(), row_var_[sizeof(T) == 4]),
                                            Gathers<T, 1>{{st.xbar.get()}}, e, s_);
    }

    template <class T>
    int kkt_passes(HalState<T> &st, int &grid_col, const HalCtl *ctl = nullptr) {
        if (!ctl) ctl = ctl_.get();
        int gr = 0;
        if (st.m > 0) {
            KktRowEpi<T> r;
            r.ctl = ctl;
            r.yhat = st.yhat.get();
            r.rl = st.rl.get();
            r.ru = st.ru.get();
            r.rs = st.rs.get();
            r.partials = pkr_.get();
            gr = launch_tiles<T, T, 1, false>(view(dm_.a, st.ka.get()), Gathers<T, 1>{{st.xhat.get()}}, r, s_);
        }
        q_pass(st, st.xhat.get(), ctl);
        KktColEpi<T> c;
        c.ctl = ctl;
        c.qx = dm_.qp ? st.qx.get() : nullptr;
        c.xhat = st.xhat.get();
        c.c = st.c.get();
        c.l = st.l.get();
        c.u = st.u.get();
        c.cs = st.cs.get();
        c.partials = pkc_.get();
        const T *yg = st.m > 0 ? st.yhat.get() : st.xhat.get();
        grid_col = launch_tiles<T, T, 1, false>(view(dm_.at, st.kat.get()), Gathers<T, 1>{{yg}}, c, s_);
        return gr;
    }

    const DeviceModel &dm_;
    vk_options o_;
    cudaStream_t s_;
    bool mixed_ = false;
    int chunk_ = 64;
    DevBuf<double> rs_, cs_;
    HalState<double> s64_;
    HalState<float> s32_;
    DevBuf<HalCtl> ctl_, evalctl_;
    HostBuf<HalCtl> hctl_;
    DevBuf<KktEval> evalout_;
    KktEval k64_{};
    DevBuf<double> pc_, pr_, pkr_, pkc_;
    double knorm_ = 0.0, lq_ = 0.0, omega0_ = 1.0, bnorm_ = 0.0, cnorm_ = 0.0;
    cudaGraphExec_t g64_ = nullptr, g32_ = nullptr;
    long long graph_nodes_ = 0, launches_ = 0;
    bool tuned_ = false;
    int col_var_[2] = {-1, -1}, row_var_[2] = {-1, -1}; // tuned pass variants [float64, float32]
};

} // namespace

std::unique_ptr<Engine> make_halpern_engine(const DeviceModel &dm, const vk_options &o, cudaStream_t s) {
    return std::make_unique<HalpernEngine>(dm, o, s);
}

} // namespace vk
