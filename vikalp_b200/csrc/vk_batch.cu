// Batched restarted-Halpern PDHG over many independent LPs of uneven size.
//
// The instances are laid out as one block-diagonal problem (rows, columns and
// nonzeros concatenated; warp-tiles never cross an instance), so one launch of
// each fused pass advances every instance. Each instance keeps its own step
// size eta_b (power iteration run on all instances at once, normalised per
// instance), primal weight omega_b, Halpern counter, restart state and
// convergence mask: per-row / per-column epilogues look their instance up, and
// the tiles of an instance that has converged are skipped, so a draining
// batch stops streaming the finished instances. Check reductions are written
// per tile and summed per instance in a fixed order (deterministic); a
// control kernel with one thread per instance applies the same stop / restart
// / primal-weight rules as the single-instance engine (vk_halpern.cu). The
// chunk of check_every iterations is one CUDA graph.
#include "vk_blockdiag.cuh"
#include "vk_engine.cuh"
#include "vk_stage.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <exception>
#include <limits>
#include <numeric>
#include <string>
#include <system_error>
#include <thread>
#include <type_traits>

namespace vk {
namespace {

constexpr double kRhoB = 1.0;
constexpr int kRuizB = 10;

// Per-instance control, structure of arrays (device).
struct BCtl {
    double *eta, *omega, *tau, *sigma, *r_restart, *r_prev, *bnorm, *cnorm, *offset, *kkt, *rel_p, *rel_d, *rel_gap;
    long long *k_base, *iters, *restarts;
    int *done, *status, *restart_now;
    double tol;
    double theta, freeze, beta_suff, beta_nec, beta_art; // primal_weight_rule()
    long long limit;
    int count;
};

__device__ __forceinline__ double lam_of(const BCtl &c, int b, int it) {
    const double k = static_cast<double>(c.k_base[b] + it);
    return (k + 1.0) / (k + 2.0);
}

template <class T, bool CHECK>
struct BColEpi : EpiBase<T> {
    static constexpr int NR = CHECK ? 2 : 1;
    static constexpr bool kPerTile = CHECK;
    BCtl ctl;
    int it;
    const int *inst, *tile_inst;
    T *x, *xbar, *xhat;
    const T *x0, *c, *l, *u;
    double *partials;
    struct Pre {
        T x, x0, c, l, u;
        int b;
    };
    static constexpr bool kSkipTiles = true;
    __device__ bool skip_tile(int t) const { return ctl.done[tile_inst[t]] != 0; }
    __device__ Pre load(int j) const { return Pre{x[j], x0[j], c[j], l[j], u[j], inst[j]}; }
    __device__ void row_pre(int j, const T (&s)[1], const Pre &p, double (&red)[NR]) const {
        const T tau = static_cast<T>(ctl.tau[p.b]);
        const T lam = static_cast<T>(lam_of(ctl, p.b, it));
        const T xh = clampbox(p.x - tau * (p.c + s[0]), p.l, p.u);
        xbar[j] = T(2) * xh - p.x;
        x[j] = lam * ((T(1) + T(kRhoB)) * xh - T(kRhoB) * p.x) + (T(1) - lam) * p.x0;
        if (CHECK) {
            xhat[j] = xh;
            const double d0 = static_cast<double>(xh) - static_cast<double>(p.x);
            const double d1 = static_cast<double>(xh) - static_cast<double>(p.x0);
            red[0] += d0 * d0;
            red[CHECK ? 1 : 0] += d1 * d1;
        }
    }
    template <int R>
    __device__ void tile_done(int t, double (&red)[R]) const {
        for (int r = 0; r < R; ++r) partials[(size_t)t * R + r] = red[r];
    }
};

template <class T, bool CHECK>
struct BRowEpi : EpiBase<T> {
    static constexpr int NR = CHECK ? 2 : 1;
    static constexpr bool kPerTile = CHECK;
    BCtl ctl;
    int it;
    const int *inst, *tile_inst;
    T *y, *yhat;
    const T *y0, *rl, *ru;
    double *partials;
    struct Pre {
        T y, y0, rl, ru;
        int b;
    };
    static constexpr bool kSkipTiles = true;
    __device__ bool skip_tile(int t) const { return ctl.done[tile_inst[t]] != 0; }
    __device__ Pre load(int i) const { return Pre{y[i], y0[i], rl[i], ru[i], inst[i]}; }
    __device__ void row_pre(int i, const T (&s)[1], const Pre &p, double (&red)[NR]) const {
        const T sigma = static_cast<T>(ctl.sigma[p.b]);
        const T lam = static_cast<T>(lam_of(ctl, p.b, it));
        const T v = p.y + sigma * s[0];
        const T yh = v - clampbox(v, sigma * p.rl, sigma * p.ru);
        y[i] = lam * ((T(1) + T(kRhoB)) * yh - T(kRhoB) * p.y) + (T(1) - lam) * p.y0;
        if (CHECK) {
            yhat[i] = yh;
            const double d0 = static_cast<double>(yh) - static_cast<double>(p.y);
            const double d1 = static_cast<double>(yh) - static_cast<double>(p.y0);
            red[0] += d0 * d0;
            red[CHECK ? 1 : 0] += d1 * d1;
        }
    }
    template <int R>
    __device__ void tile_done(int t, double (&red)[R]) const {
        for (int r = 0; r < R; ++r) partials[(size_t)t * R + r] = red[r];
    }
};

template <class T>
struct BKktRowEpi : EpiBase<T> {
    static constexpr int NR = 3;
    static constexpr bool kPerTile = true;
    BCtl ctl;
    const int *tile_inst;
    const T *yhat, *rl, *ru, *rs;
    double *partials;
    struct Pre {
        T y, rl, ru, r;
    };
    static constexpr bool kSkipTiles = true;
    __device__ bool skip_tile(int t) const { return ctl.done[tile_inst[t]] != 0; }
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
    template <int R>
    __device__ void tile_done(int t, double (&red)[R]) const {
        for (int r = 0; r < R; ++r) partials[(size_t)t * R + r] = red[r];
    }
};

template <class T>
struct BKktColEpi : EpiBase<T> {
    static constexpr int NR = 4;
    static constexpr bool kPerTile = true;
    BCtl ctl;
    const int *tile_inst;
    const T *xhat, *c, *l, *u, *cs;
    double *partials;
    struct Pre {
        T x, c, l, u, d;
    };
    static constexpr bool kSkipTiles = true;
    __device__ bool skip_tile(int t) const { return ctl.done[tile_inst[t]] != 0; }
    __device__ Pre load(int j) const { return Pre{xhat[j], c[j], l[j], u[j], cs[j]}; }
    __device__ void row_pre(int, const T (&s)[1], const Pre &p, double (&red)[NR]) const {
        const double lam = static_cast<double>(p.c) + static_cast<double>(s[0]);
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
    }
    template <int R>
    __device__ void tile_done(int t, double (&red)[R]) const {
        for (int r = 0; r < R; ++r) partials[(size_t)t * R + r] = red[r];
    }
};

template <class T>
struct BStore : EpiRow<T, BStore<T>> {
    T *y;
    __device__ void row(int i, const T (&s)[1], double (&)[1]) const { y[i] = s[0]; }
};

// out[b*R + r] = sum of partials over tiles [begin[b], begin[b+1]) (fixed order).
__global__ void segment_reduce_kernel(const double *__restrict__ partials, const int *__restrict__ begin, int count,
                                      int R, double *__restrict__ out) {
    const int b = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= count) return;
    for (int r = 0; r < R; ++r) {
        double s = 0.0;
        for (int t = begin[b] + lane; t < begin[b + 1]; t += 32) s += partials[(size_t)t * R + r];
        s = warp_sum(s);
        if (lane == 0) out[(size_t)b * R + r] = s;
    }
}

// out[b] = sum_{i in segment b} a_i * a_i (contiguous segments; one block
// each, fixed reduction tree, so deterministic).
template <class T>
__global__ void segment_norm2_kernel(const T *__restrict__ a, const int *__restrict__ off, int count,
                                     double *__restrict__ out) {
    __shared__ double scratch[32];
    const int b = blockIdx.x;
    if (b >= count) return;
    double s[1] = {0.0};
    for (int i = off[b] + threadIdx.x; i < off[b + 1]; i += blockDim.x)
        s[0] += static_cast<double>(a[i]) * static_cast<double>(a[i]);
    block_sum<1>(s, scratch);
    if (threadIdx.x == 0) out[b] = s[0];
}

template <class T>
__global__ void segment_scale_kernel(T *__restrict__ a, const int *__restrict__ inst, int n,
                                     const double *__restrict__ nrm2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = nrm2[inst[i]];
    if (v > 0.0) a[i] = static_cast<T>(a[i] / sqrt(v));
}

__global__ void bscaled_norm_kernel(const int *__restrict__ ro, const int *__restrict__ ci,
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

__global__ void brescale_kernel(double *__restrict__ s, const double *__restrict__ norm, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && norm[i] > 0.0) s[i] /= sqrt(norm[i]);
}

template <class T>
__global__ void bscale_matrix_kernel(const int *__restrict__ ro, const int *__restrict__ ci,
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
__global__ void bscale_vec_kernel(const double *__restrict__ a, const double *__restrict__ s, int n, int mode,
                                  T *__restrict__ out) {
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
__global__ void bconvert_kernel(const TS *__restrict__ a, int n, TD *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<TD>(a[i]);
}

// Power-iteration start vector: the single-instance engine's hash of the
// column index, taken per instance (local index), so both start alike.
__global__ void bseed_kernel(double *a, const int *__restrict__ inst, const int *__restrict__ off, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        unsigned h = static_cast<unsigned>(i - off[inst[i]]) * 2654435761u + 12345u;
        h ^= h >> 13;
        h *= 2246822519u;
        h ^= h >> 16;
        a[i] = 0.5 + static_cast<double>(h & 0xffff) / 65536.0;
    }
}

// One thread per instance: the single-instance check rules (vk_halpern.cu).
__global__ void batch_control_kernel(BCtl c, const double *cs, const double *rs, const double *kr, const double *kc,
                                     int chunk) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= c.count || c.done[b]) return;
    const double dx2 = cs[b * 2], dx0 = cs[b * 2 + 1], dy2 = rs[b * 2], dy0 = rs[b * 2 + 1];
    const double rp2 = kr[b * 3], dobj_r = kr[b * 3 + 1], viol2 = kr[b * 3 + 2];
    const double rd2 = kc[b * 4], dobj_c = kc[b * 4 + 1], pobj = kc[b * 4 + 2] + c.offset[b], box2 = kc[b * 4 + 3];
    const double dobj = dobj_r + dobj_c + c.offset[b];
    c.iters[b] += chunk;
    c.rel_p[b] = (sqrt(rp2) + sqrt(box2)) / (1.0 + c.bnorm[b]);
    c.rel_d[b] = sqrt(rd2 + viol2) / (1.0 + c.cnorm[b]);
    c.rel_gap[b] = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    const double kkt = smax(smax(c.rel_p[b], c.rel_d[b]), c.rel_gap[b]);
    c.kkt[b] = kkt;
    c.restart_now[b] = 0;
    if (!(kkt == kkt)) {
        c.done[b] = 1;
        c.status[b] = VK_STATUS_NUMERICAL_FAILURE;
        return;
    }
    if (kkt <= c.tol) {
        c.done[b] = 1;
        c.status[b] = VK_STATUS_OPTIMAL;
        return;
    }
    if (c.iters[b] >= c.limit) {
        c.done[b] = 1;
        c.status[b] = VK_STATUS_ITERATION_LIMIT;
        return;
    }
    const double omega = c.omega[b];
    const double r = sqrt(omega * dx2 + dy2 / omega);
    const long long k = c.k_base[b] + chunk;
    bool restart = false;
    if (c.r_restart[b] < 0.0) {
        c.r_restart[b] = r;
    } else {
        restart = (r <= c.beta_suff * c.r_restart[b]) || (r <= c.beta_nec * c.r_restart[b] && r > c.r_prev[b]) ||
                  (static_cast<double>(k) >= c.beta_art * static_cast<double>(c.iters[b]));
    }
    c.r_prev[b] = r;
    if (restart) {
        const double mx = sqrt(dx0), my = sqrt(dy0);
        double w = omega;
        if (mx > 1e-10 && my > 1e-10 && c.theta > 0.0 && kkt >= c.freeze)
            w = exp(c.theta * log(my / mx) + (1.0 - c.theta) * log(omega));
        c.omega[b] = w;
        c.tau[b] = c.eta[b] / w;
        c.sigma[b] = c.eta[b] * w;
        c.k_base[b] = 0;
        c.restarts[b] += 1;
        c.restart_now[b] = 1;
        c.r_restart[b] = r;
    } else {
        c.k_base[b] = k;
    }
}

template <class T>
__global__ void brestart_kernel(BCtl c, const int *ci, const int *ri, T *x, T *x0, const T *xhat, int n, T *y, T *y0,
                                const T *yhat, int m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int b = ci[i];
        if (c.restart_now[b] && !c.done[b]) {
            x[i] = xhat[i];
            x0[i] = xhat[i];
        }
    }
    if (i < m) {
        const int b = ri[i];
        if (c.restart_now[b] && !c.done[b]) {
            y[i] = yhat[i];
            y0[i] = yhat[i];
        }
    }
}

template <class T>
__global__ void bunscale_kernel(const T *__restrict__ a, const double *__restrict__ s, int n, double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<double>(a[i]) * s[i];
}

template <class T>
struct BState {
    DevBuf<T> ka, kat, c, l, u, rl, ru, rs, cs, x, x0, xbar, xhat, y, y0, yhat;
};

class SharedEngine;

class BatchEngine {
    friend class SharedEngine; // reuses the scaled model of a one-instance batch

public:
    // the objective vector in original units, concatenated over the instances
    const double *c_orig() const { return c_orig_.get(); }
    BatchEngine(const vk_problem *probs, int count, const vk_options &o) : o_(o), B_(count) {
        VK_CUDA(cudaSetDevice(o.device));
        device_error_flag();
        VK_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
        mixed_ = o.precision == VK_PREC_MIXED;
        chunk_ = std::max(2, o.check_every > 0 ? o.check_every : 64);
        log_.stream(s_);
        log_.mark("stream");
        concatenate(probs);
        log_.mark("concatenate (host)");
        setup_device();
        log_.mark("step sizes");
    }
    ~BatchEngine() {
        if (g64_) cudaGraphExecDestroy(g64_);
        if (g32_) cudaGraphExecDestroy(g32_);
        if (s_) cudaStreamDestroy(s_);
    }

    void solve(vk_result *results) {
        const auto started = std::chrono::steady_clock::now();
        reset_control();
        cudaEvent_t e0, e1;
        VK_CUDA(cudaEventCreate(&e0));
        VK_CUDA(cudaEventCreate(&e1));
        VK_CUDA(cudaEventRecord(e0, s_));
        long long launches = 0, fp32_iters = 0;
        bool timed_out = false;
        if (mixed_) {
            copy_state<float, double>(s64_, s32_, true);
            if (!g32_) g32_ = capture(s32_);
            std::vector<double> best(B_, std::numeric_limits<double>::infinity());
            int stall = 0;
            for (;;) {
                if (over_time(started)) {
                    timed_out = true;
                    break;
                }
                VK_CUDA(cudaGraphLaunch(g32_, s_));
                launches += nodes_;
                read_control();
                check_device_error(s_);
                bool improved = false, all_done = true;
                double worst = 0.0;
                for (int b = 0; b < B_; ++b) {
                    if (h_done_[b]) continue;
                    all_done = false;
                    worst = std::max(worst, h_kkt_[b]);
                    if (h_kkt_[b] < 0.7 * best[b]) {
                        best[b] = h_kkt_[b];
                        improved = true;
                    }
                }
                if (all_done) break;
                if (improved)
                    stall = 0;
                else if (++stall >= 6 && worst < 1e-3)
                    break;
            }
            fp32_iters = *std::max_element(h_iters_.begin(), h_iters_.end());
            copy_state<double, float>(s32_, s64_, false);
            // re-open every instance that stopped on the float32 measurement
            reopen_after_fp32();
        }
        if (!timed_out) {
            if (!g64_) g64_ = capture(s64_);
            for (;;) {
                if (over_time(started)) {
                    timed_out = true;
                    break;
                }
                VK_CUDA(cudaGraphLaunch(g64_, s_));
                launches += nodes_;
                read_control();
                check_device_error(s_);
                if (std::all_of(h_done_.begin(), h_done_.end(), [](int d) { return d != 0; })) break;
            }
        }
        VK_CUDA(cudaEventRecord(e1, s_));
        read_control();
        float ms = 0.f;
        VK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        // answers: (x^, y^) of the last check, unscaled
        DevBuf<double> xo(n_), yo(m_ > 0 ? m_ : 1);
        bunscale_kernel<double><<<grid1d(n_), 256, 0, s_>>>(s64_.xhat.get(), cs_.get(), n_, xo.get());
        if (m_ > 0) bunscale_kernel<double><<<grid1d(m_), 256, 0, s_>>>(s64_.yhat.get(), rs_.get(), m_, yo.get());
        VK_LAUNCH_CHECK();
        std::vector<double> hx(n_), hy(m_);
        stage_d2h(hx.data(), xo.get(), n_ * sizeof(double), s_);
        if (m_ > 0) stage_d2h(hy.data(), yo.get(), m_ * sizeof(double), s_);
        const double secs = seconds_since(started);
        for (int b = 0; b < B_; ++b) {
            vk_result &r = results[b];
            const int c0 = col_off_[b], c1 = col_off_[b + 1], r0 = row_off_[b], r1 = row_off_[b + 1];
            if (r.x) std::copy(hx.begin() + c0, hx.begin() + c1, r.x);
            if (r.y) std::copy(hy.begin() + r0, hy.begin() + r1, r.y);
            double obj = offset_[b];
            for (int j = c0; j < c1; ++j) obj += h_c_[j] * hx[j];
            r.objective = obj;
            r.status = h_done_[b] ? h_status_[b] : (timed_out ? VK_STATUS_TIME_LIMIT : VK_STATUS_ITERATION_LIMIT);
            r.iterations = h_iters_[b];
            r.restarts = h_restarts_[b];
            r.rel_primal = h_rel_p_[b];
            r.rel_dual = h_rel_d_[b];
            r.rel_gap = h_rel_gap_[b];
            r.last_metric = h_kkt_[b];
            r.solve_seconds = secs;
            r.iterate_seconds = ms * 1e-3;
            r.fp32_iterations = std::min<long long>(fp32_iters, h_iters_[b]);
            r.kernel_launches = launches;
            r.primal_residual = r.stationarity_residual = r.complementarity_residual =
                std::numeric_limits<double>::quiet_NaN();
            r.message[0] = '\0';
        }
    }

private:
    bool over_time(std::chrono::steady_clock::time_point t0) const {
        return std::isfinite(o_.time_limit_seconds) && seconds_since(t0) >= o_.time_limit_seconds;
    }

    void concatenate(const vk_problem *probs) {
        BlockDiag bd;
        concat_instances(probs, B_, bd);
        m_ = bd.m;
        n_ = bd.n;
        nnz_ = bd.nnz;
        row_off_ = std::move(bd.row_off);
        col_off_ = std::move(bd.col_off);
        h_rinst_ = std::move(bd.rinst);
        h_cinst_ = std::move(bd.cinst);
        h_ro_ = std::move(bd.ro);
        h_ci_ = std::move(bd.ci);
        h_v_ = std::move(bd.v);
        h_c_ = std::move(bd.c);
        h_vl_ = std::move(bd.vl);
        h_vu_ = std::move(bd.vu);
        h_rl_ = std::move(bd.rl);
        h_ru_ = std::move(bd.ru);
        offset_ = std::move(bd.offset);
        // norms in original units per instance
        bnorm_.assign(B_, 0.0);
        cnorm_.assign(B_, 0.0);
        for (int b = 0; b < B_; ++b) {
            double c2 = 0.0, b2 = 0.0;
            for (int j = col_off_[b]; j < col_off_[b + 1]; ++j) c2 += h_c_[j] * h_c_[j];
            for (int i = row_off_[b]; i < row_off_[b + 1]; ++i) {
                double v = 0.0;
                if (std::isfinite(h_rl_[i])) v = std::max(v, std::abs(h_rl_[i]));
                if (std::isfinite(h_ru_[i])) v = std::max(v, std::abs(h_ru_[i]));
                b2 += v * v;
            }
            cnorm_[b] = std::sqrt(c2);
            bnorm_[b] = std::sqrt(b2);
        }
    }

    template <class V>
    void up(DevBuf<V> &d, const std::vector<V> &h) {
        d.reset(h.empty() ? 1 : h.size());
        if (!h.empty()) VK_CUDA(cudaMemcpyAsync(d.get(), h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice, s_));
    }

    void setup_device() {
        // block-diagonal A and A' with instance-aligned tiles
        {
            BlockDiag bd;
            bd.count = B_;
            bd.m = m_;
            bd.n = n_;
            bd.nnz = nnz_;
            bd.row_off = row_off_;
            bd.col_off = col_off_;
            bd.rinst = h_rinst_;
            bd.cinst = h_cinst_;
            bd.ro = std::move(h_ro_);
            bd.ci = std::move(h_ci_);
            bd.v = std::move(h_v_);
            DeviceBlockDiag dd;
            upload_block_diag(bd, dd, s_, true);
            a_ = std::move(dd.a);
            at_ = std::move(dd.at);
            perm_ = std::move(dd.perm);
            a_val_ = std::move(dd.a_val);
            at_val_ = std::move(dd.at_val);
            rinst_ = std::move(dd.rinst);
            cinst_ = std::move(dd.cinst);
            tinst_a_ = std::move(dd.tinst_a);
            tinst_at_ = std::move(dd.tinst_at);
            tbeg_a_ = std::move(dd.tbeg_a);
            tbeg_at_ = std::move(dd.tbeg_at);
        }
        log_.mark("upload + transpose + autotune");
        const DevBuf<double> &a_val = a_val_;
        const DevBuf<double> &at_val = at_val_;
        DevBuf<double> c, vl, vu, rl, ru;
        up(c, h_c_);
        c_orig_.reset(n_ > 0 ? n_ : 1);
        if (n_ > 0)
            VK_CUDA(cudaMemcpyAsync(c_orig_.get(), c.get(), n_ * sizeof(double), cudaMemcpyDeviceToDevice, s_));
        up(vl, h_vl_);
        up(vu, h_vu_);
        up(rl, h_rl_);
        up(ru, h_ru_);
        // Ruiz + Pock-Chambolle, per instance by construction (block-diagonal)
        rs_.reset(m_ > 0 ? m_ : 1);
        cs_.reset(n_);
        {
            std::vector<double> one_m(m_ > 0 ? m_ : 1, 1.0), one_n(n_, 1.0);
            VK_CUDA(cudaMemcpyAsync(rs_.get(), one_m.data(), one_m.size() * 8, cudaMemcpyHostToDevice, s_));
            VK_CUDA(cudaMemcpyAsync(cs_.get(), one_n.data(), one_n.size() * 8, cudaMemcpyHostToDevice, s_));
            VK_CUDA(cudaStreamSynchronize(s_));
        }
        if (nnz_ > 0) {
            DevBuf<double> rn(m_), cn(n_);
            for (int pass = 0; pass <= kRuizB; ++pass) {
                const int mode = pass < kRuizB ? 0 : 1;
                bscaled_norm_kernel<<<ceil_div(int64_t(m_) * 32, 256), 256, 0, s_>>>(
                    a_.ro.get(), a_.ci.get(), a_val.get(), rs_.get(), cs_.get(), m_, mode, rn.get());
                bscaled_norm_kernel<<<ceil_div(int64_t(n_) * 32, 256), 256, 0, s_>>>(
                    at_.ro.get(), at_.ci.get(), at_val.get(), cs_.get(), rs_.get(), n_, mode, cn.get());
                VK_LAUNCH_CHECK();
                brescale_kernel<<<grid1d(m_), 256, 0, s_>>>(rs_.get(), rn.get(), m_);
                brescale_kernel<<<grid1d(n_), 256, 0, s_>>>(cs_.get(), cn.get(), n_);
                VK_LAUNCH_CHECK();
            }
        }
        log_.mark("scaling");
        setup_state(s64_, a_val, at_val, c, rl, ru);
        if (mixed_) setup_state(s32_, a_val, at_val, c, rl, ru);
        log_.mark("scaled copies");
        // model bounds, scaled, into the float64 state (the float32 copy is made per solve)
        bscale_vec_kernel<double><<<grid1d(n_), 256, 0, s_>>>(vl.get(), cs_.get(), n_, 1, s64_.l.get());
        bscale_vec_kernel<double><<<grid1d(n_), 256, 0, s_>>>(vu.get(), cs_.get(), n_, 1, s64_.u.get());
        VK_LAUNCH_CHECK();
        step_sizes();
        a_val_.release(); // the scaled copies carry on
        at_val_.release();
        // control arrays
        const size_t Bs = static_cast<size_t>(B_);
        for (DevBuf<double> *d : {&eta_, &omega_, &tau_, &sigma_, &rr_, &rp_, &bn_, &cn_, &off_, &kkt_, &relp_, &reld_,
                                  &relg_})
            d->reset(Bs);
        for (DevBuf<long long> *d : {&kb_, &it_, &rst_}) d->reset(Bs);
        for (DevBuf<int> *d : {&done_, &status_, &rnow_}) d->reset(Bs);
        VK_CUDA(cudaMemcpyAsync(bn_.get(), bnorm_.data(), Bs * 8, cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaMemcpyAsync(cn_.get(), cnorm_.data(), Bs * 8, cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaMemcpyAsync(off_.get(), offset_.data(), Bs * 8, cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaMemcpyAsync(eta_.get(), h_eta_.data(), Bs * 8, cudaMemcpyHostToDevice, s_));
        pc_.reset(static_cast<size_t>(std::max(at_.ntiles, 1)) * 2);
        pr_.reset(static_cast<size_t>(std::max(a_.ntiles, 1)) * 2);
        pkr_.reset(static_cast<size_t>(std::max(a_.ntiles, 1)) * 3);
        pkc_.reset(static_cast<size_t>(std::max(at_.ntiles, 1)) * 4);
        sc_.reset(Bs * 2);
        sr_.reset(Bs * 2);
        skr_.reset(Bs * 3);
        skc_.reset(Bs * 4);
        for (DevBuf<double> *d : {&pc_, &pr_, &pkr_, &pkc_, &sc_, &sr_, &skr_, &skc_})
            VK_CUDA(cudaMemsetAsync(d->get(), 0, d->bytes(), s_));
        h_done_.resize(B_);
        h_status_.resize(B_);
        h_iters_.resize(B_);
        h_restarts_.resize(B_);
        h_kkt_.resize(B_);
        h_rel_p_.resize(B_);
        h_rel_d_.resize(B_);
        h_rel_gap_.resize(B_);
        VK_CUDA(cudaStreamSynchronize(s_));
    }

    template <class T>
    void setup_state(BState<T> &st, const DevBuf<double> &a_val, const DevBuf<double> &at_val, const DevBuf<double> &c,
                     const DevBuf<double> &rl, const DevBuf<double> &ru) {
        const int m = m_, n = n_, mm = m > 0 ? m : 1;
        st.ka.reset(padded(nnz_));
        st.kat.reset(padded(nnz_));
        if (m > 0)
            bscale_matrix_kernel<T><<<ceil_div(int64_t(m) * 32, 256), 256, 0, s_>>>(
                a_.ro.get(), a_.ci.get(), a_val.get(), rs_.get(), cs_.get(), m, false, st.ka.get());
        bscale_matrix_kernel<T><<<ceil_div(int64_t(n) * 32, 256), 256, 0, s_>>>(
            at_.ro.get(), at_.ci.get(), at_val.get(), rs_.get(), cs_.get(), n, true, st.kat.get());
        for (DevBuf<T> *b : {&st.c, &st.l, &st.u, &st.cs, &st.x, &st.x0, &st.xbar, &st.xhat}) b->reset(n);
        for (DevBuf<T> *b : {&st.rl, &st.ru, &st.rs, &st.y, &st.y0, &st.yhat}) b->reset(mm);
        bscale_vec_kernel<T><<<grid1d(n), 256, 0, s_>>>(c.get(), cs_.get(), n, 0, st.c.get());
        bconvert_kernel<T, double><<<grid1d(n), 256, 0, s_>>>(cs_.get(), n, st.cs.get());
        VK_CUDA(cudaMemsetAsync(st.xhat.get(), 0, n * sizeof(T), s_));
        if (m > 0) {
            bscale_vec_kernel<T><<<grid1d(m), 256, 0, s_>>>(rl.get(), rs_.get(), m, 2, st.rl.get());
            bscale_vec_kernel<T><<<grid1d(m), 256, 0, s_>>>(ru.get(), rs_.get(), m, 2, st.ru.get());
            bconvert_kernel<T, double><<<grid1d(m), 256, 0, s_>>>(rs_.get(), m, st.rs.get());
            VK_CUDA(cudaMemsetAsync(st.yhat.get(), 0, m * sizeof(T), s_));
        }
        VK_LAUNCH_CHECK();
    }

    // Per-instance power iteration (segment norms), omega_0 per instance.
    void step_sizes() {
        const int n = n_, m = m_;
        DevBuf<double> v(n), w(m > 0 ? m : 1), z(n), nrm(B_);
        DevBuf<int> coff;
        up(coff, col_off_);
        bseed_kernel<<<grid1d(n), 256, 0, s_>>>(v.get(), cinst_.get(), coff.get(), n);
        VK_LAUNCH_CHECK();
        segment_norm2_kernel<double><<<B_, 256, 0, s_>>>(v.get(), coff.get(), B_, nrm.get());
        segment_scale_kernel<double><<<grid1d(n), 256, 0, s_>>>(v.get(), cinst_.get(), n, nrm.get());
        // Each instance keeps the estimate of the iteration at which its own
        // sequence settled (the single-instance stopping rule); the shared
        // loop runs until every instance has settled.
        std::vector<double> est(B_, 0.0), prev(B_, 0.0), h(B_);
        std::vector<char> settled(B_, 0);
        if (nnz_ > 0 && m > 0) {
            for (int it = 0; it < 200; ++it) {
                BStore<double> ew;
                ew.y = w.get();
                launch_tiles<double, double, 1, false>(view(a_, s64_.ka.get()), Gathers<double, 1>{{v.get()}}, ew, s_);
                BStore<double> ez;
                ez.y = z.get();
                launch_tiles<double, double, 1, false>(view(at_, s64_.kat.get()), Gathers<double, 1>{{w.get()}}, ez, s_);
                segment_norm2_kernel<double><<<B_, 256, 0, s_>>>(z.get(), coff.get(), B_, nrm.get());
                VK_CUDA(cudaMemcpyAsync(h.data(), nrm.get(), B_ * 8, cudaMemcpyDeviceToHost, s_));
                VK_CUDA(cudaStreamSynchronize(s_));
                segment_scale_kernel<double><<<grid1d(n), 256, 0, s_>>>(z.get(), cinst_.get(), n, nrm.get());
                std::swap(v, z);
                bool all = true;
                for (int b = 0; b < B_; ++b) {
                    if (settled[b]) continue;
                    const double e = std::sqrt(std::sqrt(h[b]));
                    if (it > 10 && std::abs(e - prev[b]) <= 1e-6 * e) settled[b] = 1;
                    else all = false;
                    prev[b] = e;
                    est[b] = e;
                }
                if (all) break;
            }
        }
        h_eta_.resize(B_);
        for (int b = 0; b < B_; ++b) h_eta_[b] = est[b] > 0.0 ? 0.99 / est[b] : 1.0;
        // omega_0 = |c^_b| / |b^_b| (scaled)
        std::vector<double> hcs(n), hrs(m);
        VK_CUDA(cudaMemcpyAsync(hcs.data(), cs_.get(), n * 8, cudaMemcpyDeviceToHost, s_));
        if (m > 0) VK_CUDA(cudaMemcpyAsync(hrs.data(), rs_.get(), m * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaStreamSynchronize(s_));
        h_omega0_.assign(B_, 1.0);
        for (int b = 0; b < B_; ++b) {
            double cs2 = 0.0, bs2 = 0.0;
            for (int j = col_off_[b]; j < col_off_[b + 1]; ++j) cs2 += (h_c_[j] * hcs[j]) * (h_c_[j] * hcs[j]);
            for (int i = row_off_[b]; i < row_off_[b + 1]; ++i) {
                double v2 = 0.0;
                if (std::isfinite(h_rl_[i])) v2 = std::max(v2, std::abs(h_rl_[i]));
                if (std::isfinite(h_ru_[i])) v2 = std::max(v2, std::abs(h_ru_[i]));
                bs2 += (v2 * hrs[i]) * (v2 * hrs[i]);
            }
            if (cs2 > 1e-20 && bs2 > 1e-20) h_omega0_[b] = std::sqrt(cs2) / std::sqrt(bs2);
        }
    }

    BCtl ctl() {
        BCtl c{};
        c.eta = eta_.get();
        c.omega = omega_.get();
        c.tau = tau_.get();
        c.sigma = sigma_.get();
        c.r_restart = rr_.get();
        c.r_prev = rp_.get();
        c.bnorm = bn_.get();
        c.cnorm = cn_.get();
        c.offset = off_.get();
        c.kkt = kkt_.get();
        c.rel_p = relp_.get();
        c.rel_d = reld_.get();
        c.rel_gap = relg_.get();
        c.k_base = kb_.get();
        c.iters = it_.get();
        c.restarts = rst_.get();
        c.done = done_.get();
        c.status = status_.get();
        c.restart_now = rnow_.get();
        c.tol = o_.relative_tolerance;
        c.limit = o_.iteration_limit;
        c.count = B_;
        const PrimalWeightRule pw = primal_weight_rule();
        c.theta = pw.theta;
        c.freeze = pw.freeze;
        c.beta_suff = pw.beta_suff;
        c.beta_nec = pw.beta_nec;
        c.beta_art = pw.beta_art;
        return c;
    }

    void reset_control() {
        const size_t Bs = B_;
        std::vector<double> tau(Bs), sigma(Bs), neg(Bs, -1.0), inf(Bs, std::numeric_limits<double>::infinity());
        std::vector<double> w(Bs);
        const double start = primal_weight_rule().start;
        for (int b = 0; b < B_; ++b) {
            w[b] = h_omega0_[b] * start;
            tau[b] = h_eta_[b] / w[b];
            sigma[b] = h_eta_[b] * w[b];
        }
        VK_CUDA(cudaMemcpyAsync(omega_.get(), w.data(), Bs * 8, cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaMemcpyAsync(tau_.get(), tau.data(), Bs * 8, cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaMemcpyAsync(sigma_.get(), sigma.data(), Bs * 8, cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaMemcpyAsync(rr_.get(), neg.data(), Bs * 8, cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaMemcpyAsync(rp_.get(), inf.data(), Bs * 8, cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaMemcpyAsync(kkt_.get(), inf.data(), Bs * 8, cudaMemcpyHostToDevice, s_));
        for (DevBuf<long long> *d : {&kb_, &it_, &rst_}) VK_CUDA(cudaMemsetAsync(d->get(), 0, d->bytes(), s_));
        for (DevBuf<int> *d : {&done_, &status_, &rnow_}) VK_CUDA(cudaMemsetAsync(d->get(), 0, d->bytes(), s_));
        // cold start: x = clamp(0, l, u), y = 0
        start_kernel_launch();
        VK_CUDA(cudaStreamSynchronize(s_));
    }

    void start_kernel_launch();

    void reopen_after_fp32() {
        read_control();
        std::vector<int> done(B_), status(B_);
        for (int b = 0; b < B_; ++b) {
            const bool keep = h_status_[b] == VK_STATUS_NUMERICAL_FAILURE;
            done[b] = keep ? 1 : 0;
            status[b] = keep ? h_status_[b] : VK_STATUS_NOT_SOLVED;
        }
        VK_CUDA(cudaMemcpyAsync(done_.get(), done.data(), B_ * sizeof(int), cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaMemcpyAsync(status_.get(), status.data(), B_ * sizeof(int), cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaStreamSynchronize(s_));
    }

    void read_control() {
        VK_CUDA(cudaMemcpyAsync(h_done_.data(), done_.get(), B_ * sizeof(int), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_status_.data(), status_.get(), B_ * sizeof(int), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_iters_.data(), it_.get(), B_ * sizeof(long long), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_restarts_.data(), rst_.get(), B_ * sizeof(long long), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_kkt_.data(), kkt_.get(), B_ * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_rel_p_.data(), relp_.get(), B_ * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_rel_d_.data(), reld_.get(), B_ * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_rel_gap_.data(), relg_.get(), B_ * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaStreamSynchronize(s_));
    }

    template <class TD, class TS>
    void copy_state(const BState<TS> &a, BState<TD> &b, bool bounds) {
        const int m = m_, n = n_;
        for (auto pr : {std::make_pair(&a.x, &b.x), std::make_pair(&a.x0, &b.x0), std::make_pair(&a.xhat, &b.xhat)})
            bconvert_kernel<TD, TS><<<grid1d(n), 256, 0, s_>>>(pr.first->get(), n, pr.second->get());
        if (bounds) {
            bconvert_kernel<TD, TS><<<grid1d(n), 256, 0, s_>>>(a.l.get(), n, b.l.get());
            bconvert_kernel<TD, TS><<<grid1d(n), 256, 0, s_>>>(a.u.get(), n, b.u.get());
        }
        if (m > 0)
            for (auto pr : {std::make_pair(&a.y, &b.y), std::make_pair(&a.y0, &b.y0), std::make_pair(&a.yhat, &b.yhat)})
                bconvert_kernel<TD, TS><<<grid1d(m), 256, 0, s_>>>(pr.first->get(), m, pr.second->get());
        VK_LAUNCH_CHECK();
    }

    template <class T>
    cudaGraphExec_t capture(BState<T> &st) {
        VK_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
        const BCtl c = ctl();
        for (int it = 0; it < chunk_; ++it) {
            const bool check = it == chunk_ - 1;
            if (check) {
                pass_col<T, true>(st, c, it);
                pass_row<T, true>(st, c, it);
                kkt(st, c);
                const int wb = ceil_div(int64_t(B_) * 32, 256);
                segment_reduce_kernel<<<wb, 256, 0, s_>>>(pc_.get(), tbeg_at_.get(), B_, 2, sc_.get());
                segment_reduce_kernel<<<wb, 256, 0, s_>>>(pr_.get(), tbeg_a_.get(), B_, 2, sr_.get());
                segment_reduce_kernel<<<wb, 256, 0, s_>>>(pkr_.get(), tbeg_a_.get(), B_, 3, skr_.get());
                segment_reduce_kernel<<<wb, 256, 0, s_>>>(pkc_.get(), tbeg_at_.get(), B_, 4, skc_.get());
                batch_control_kernel<<<ceil_div(B_, 128), 128, 0, s_>>>(c, sc_.get(), sr_.get(), skr_.get(),
                                                                        skc_.get(), chunk_);
                brestart_kernel<T><<<grid1d(std::max(m_, n_)), 256, 0, s_>>>(
                    c, cinst_.get(), rinst_.get(), st.x.get(), st.x0.get(), st.xhat.get(), n_, st.y.get(), st.y0.get(),
                    st.yhat.get(), m_);
                VK_LAUNCH_CHECK();
            } else {
                pass_col<T, false>(st, c, it);
                pass_row<T, false>(st, c, it);
            }
        }
        cudaGraph_t g;
        VK_CUDA(cudaStreamEndCapture(s_, &g));
        size_t nodes = 0;
        VK_CUDA(cudaGraphGetNodes(g, nullptr, &nodes));
        nodes_ = static_cast<long long>(nodes);
        cudaGraphExec_t ex;
        VK_CUDA(cudaGraphInstantiate(&ex, g, 0));
        cudaGraphDestroy(g);
        return ex;
    }

    template <class T, bool CHECK>
    void pass_col(BState<T> &st, const BCtl &c, int it) {
        BColEpi<T, CHECK> e;
        e.ctl = c;
        e.it = it;
        e.inst = cinst_.get();
        e.tile_inst = tinst_at_.get();
        e.x = st.x.get();
        e.xbar = st.xbar.get();
        e.xhat = st.xhat.get();
        e.x0 = st.x0.get();
        e.c = st.c.get();
        e.l = st.l.get();
        e.u = st.u.get();
        e.partials = pc_.get();
        const T *yg = m_ > 0 ? st.y.get() : st.x.get();
        launch_tiles<T, T, 1, false>(view(at_, st.kat.get()), Gathers<T, 1>{{yg}}, e, s_);
    }

    template <class T, bool CHECK>
    void pass_row(BState<T> &st, const BCtl &c, int it) {
        if (m_ == 0) return;
        BRowEpi<T, CHECK> e;
        e.ctl = c;
        e.it = it;
        e.inst = rinst_.get();
        e.tile_inst = tinst_a_.get();
        e.y = st.y.get();
        e.yhat = st.yhat.get();
        e.y0 = st.y0.get();
        e.rl = st.rl.get();
        e.ru = st.ru.get();
        e.partials = pr_.get();
        launch_tiles<T, T, 1, false>(view(a_, st.ka.get()), Gathers<T, 1>{{st.xbar.get()}}, e, s_);
    }

    template <class T>
    void kkt(BState<T> &st, const BCtl &c) {
        if (m_ > 0) {
            BKktRowEpi<T> r;
            r.ctl = c;
            r.tile_inst = tinst_a_.get();
            r.yhat = st.yhat.get();
            r.rl = st.rl.get();
            r.ru = st.ru.get();
            r.rs = st.rs.get();
            r.partials = pkr_.get();
            launch_tiles<T, T, 1, false>(view(a_, st.ka.get()), Gathers<T, 1>{{st.xhat.get()}}, r, s_);
        }
        BKktColEpi<T> k;
        k.ctl = c;
        k.tile_inst = tinst_at_.get();
        k.xhat = st.xhat.get();
        k.c = st.c.get();
        k.l = st.l.get();
        k.u = st.u.get();
        k.cs = st.cs.get();
        k.partials = pkc_.get();
        const T *yg = m_ > 0 ? st.yhat.get() : st.xhat.get();
        launch_tiles<T, T, 1, false>(view(at_, st.kat.get()), Gathers<T, 1>{{yg}}, k, s_);
    }

    vk_options o_;
    int B_;
    PhaseLog log_{o_.verbose, "batch", nullptr};
    cudaStream_t s_ = nullptr;
    bool mixed_ = false;
    int chunk_ = 64;
    int m_ = 0, n_ = 0;
    int64_t nnz_ = 0;
    std::vector<int> row_off_, col_off_, h_rinst_, h_cinst_;
    std::vector<int64_t> h_ro_, h_ci_;
    std::vector<double> h_v_, h_c_, h_vl_, h_vu_, h_rl_, h_ru_, offset_, bnorm_, cnorm_, h_eta_, h_omega0_;
    CsrPattern32 a_, at_;
    DevBuf<int> perm_, rinst_, cinst_, tinst_a_, tinst_at_, tbeg_a_, tbeg_at_;
    DevBuf<double> a_val_, at_val_; // original values (setup only)
    DevBuf<double> rs_, cs_;
    DevBuf<double> c_orig_;
    BState<double> s64_;
    BState<float> s32_;
    DevBuf<double> eta_, omega_, tau_, sigma_, rr_, rp_, bn_, cn_, off_, kkt_, relp_, reld_, relg_;
    DevBuf<long long> kb_, it_, rst_;
    DevBuf<int> done_, status_, rnow_;
    DevBuf<double> pc_, pr_, pkr_, pkc_, sc_, sr_, skr_, skc_;
    std::vector<int> h_done_, h_status_;
    std::vector<long long> h_iters_, h_restarts_;
    std::vector<double> h_kkt_, h_rel_p_, h_rel_d_, h_rel_gap_;
    cudaGraphExec_t g64_ = nullptr, g32_ = nullptr;
    long long nodes_ = 0;
};

__global__ void bstart_kernel(const double *__restrict__ l, const double *__restrict__ u, int n, double *__restrict__ x,
                              double *__restrict__ x0) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) {
        const double v = clampbox(0.0, l[j], u[j]);
        x[j] = v;
        x0[j] = v;
    }
}

void BatchEngine::start_kernel_launch() {
    bstart_kernel<<<grid1d(n_), 256, 0, s_>>>(s64_.l.get(), s64_.u.get(), n_, s64_.x.get(), s64_.x0.get());
    VK_LAUNCH_CHECK();
    if (m_ > 0) {
        VK_CUDA(cudaMemsetAsync(s64_.y.get(), 0, m_ * sizeof(double), s_));
        VK_CUDA(cudaMemsetAsync(s64_.y0.get(), 0, m_ * sizeof(double), s_));
    }
}

// ---- shared-A batches: relaxations of one LP that differ in variable bounds ----
//
// The vectors of all instances are interleaved, instance-minor: X[j * ld + b]
// (ld = instance count rounded up to the lane width). One warp handles one
// matrix row for a group of 32 * VEC instances, each lane VEC adjacent
// instances, so every nonzero (column index, value: one broadcast load) pulls a
// contiguous 16-byte slice per lane of the gathered vector: the products of all
// instances share one read of the matrix, and the gathers are coalesced. The
// blocks of a group all serve the same instances, so per-instance check sums
// are reduced in registers, then across the block's warps in shared memory and
// finally over the blocks in a fixed order (deterministic).

template <class T, int VEC>
__device__ __forceinline__ void ldg_vec(const T *p, T (&o)[VEC]) {
    if constexpr (VEC == 1) {
        o[0] = __ldg(p);
    } else if constexpr (std::is_same<T, double>::value && VEC == 2) {
        const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
        o[0] = v.x;
        o[1] = v.y;
    } else {
        static_assert(std::is_same<T, float>::value && VEC == 4, "16-byte packs only");
        const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
        o[0] = v.x;
        o[1] = v.y;
        o[2] = v.z;
        o[3] = v.w;
    }
}

template <class T, int VEC>
__device__ __forceinline__ void ld_vec(const T *p, T (&o)[VEC]) {
    if constexpr (VEC == 1) {
        o[0] = *p;
    } else if constexpr (std::is_same<T, double>::value && VEC == 2) {
        const double2 v = *reinterpret_cast<const double2 *>(p);
        o[0] = v.x;
        o[1] = v.y;
    } else {
        const float4 v = *reinterpret_cast<const float4 *>(p);
        o[0] = v.x;
        o[1] = v.y;
        o[2] = v.z;
        o[3] = v.w;
    }
}

// Stores the lanes' active elements: one vector store when all are active.
template <class T, int VEC>
__device__ __forceinline__ void st_vec(T *p, const T (&v)[VEC], const bool (&act)[VEC], bool all) {
    if (all) {
        if constexpr (VEC == 1) {
            *p = v[0];
        } else if constexpr (std::is_same<T, double>::value && VEC == 2) {
            *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
        } else {
            *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
        }
    } else {
#pragma unroll
        for (int q = 0; q < VEC; ++q)
            if (act[q]) p[q] = v[q];
    }
}

constexpr int kSpmmWarps = 8;
constexpr int kSpmmMaxR = 4;
#ifndef VK_SPMM_UNROLL
#define VK_SPMM_UNROLL 4
#endif
#ifndef VK_SPMM_MINB
#define VK_SPMM_MINB 6
#endif
// Nonzeros of a row in flight per warp step, and resident blocks per SM the
// registers are held to. Timed on the 512-node batch (B200, 1,280
// iterations): unroll 4 with 6 blocks 0.628 s float32 / 1.173 s float64; 5
// blocks 0.649 / 1.337; unroll 8 with 4 blocks 0.641 / 1.198; unroll 6 or 8
// with 5 blocks and unroll 2 with 8 blocks slower still (register spills).
constexpr int kSpmmUnroll = VK_SPMM_UNROLL;
constexpr int kSpmmMinBlocks = VK_SPMM_MINB;

// Per-lane instance state common to the epilogues.
template <class T, int VEC>
struct LaneBase {
    bool act[VEC];
    bool all;
};

template <class T, int VEC>
__device__ __forceinline__ void lane_activity(const BCtl &c, int b0, LaneBase<T, VEC> &L) {
    L.all = true;
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
        const int b = b0 + q;
        L.act[q] = b < c.count && c.done[b] == 0;
        L.all = L.all && L.act[q];
    }
}

// Variable bounds of instance slice [b0, b0+VEC) at column j: the shared
// scaled model bounds unless the column has an override row.
template <class T, int VEC>
__device__ __forceinline__ void col_bounds(int j, int b0, int ld, const T *l, const T *u, const int *ovr,
                                           const T *ovl, const T *ovu, T (&lo)[VEC], T (&hi)[VEC]) {
    const int o = __ldg(ovr + j);
    if (o >= 0) {
        ldg_vec<T, VEC>(ovl + static_cast<size_t>(o) * ld + b0, lo);
        ldg_vec<T, VEC>(ovu + static_cast<size_t>(o) * ld + b0, hi);
    } else {
        const T a = __ldg(l + j), b = __ldg(u + j);
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            lo[q] = a;
            hi[q] = b;
        }
    }
}

template <class T, int VEC, bool CHECK>
struct SColEpi {
    static constexpr int NR = CHECK ? 2 : 0;
    BCtl ctl;
    int it, ld;
    T *x, *xbar, *xhat;
    const T *x0, *c, *l, *u, *ovl, *ovu;
    const int *ovr;
    struct Lane : LaneBase<T, VEC> {
        T tau[VEC], lam[VEC];
    };
    __device__ Lane lane(int b0) const {
        Lane L;
        lane_activity<T, VEC>(ctl, b0, L);
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            const int b = L.act[q] ? b0 + q : 0;
            L.tau[q] = static_cast<T>(ctl.tau[b]);
            L.lam[q] = static_cast<T>(lam_of(ctl, b, it));
        }
        return L;
    }
    // the iterate and the anchor, loaded before the row's gathers
    struct Pre {
        T x[VEC], x0[VEC];
    };
    __device__ Pre pre(int j, int b0) const {
        const size_t at = static_cast<size_t>(j) * ld + b0;
        Pre p;
        ld_vec<T, VEC>(x + at, p.x);
        ld_vec<T, VEC>(x0 + at, p.x0);
        return p;
    }
    __device__ void row(int j, int b0, const Lane &L, const T (&s)[VEC], double (&red)[kSpmmMaxR][VEC],
                        const Pre &p) const {
        const size_t at = static_cast<size_t>(j) * ld + b0;
        T lo[VEC], hi[VEC], xh[VEC], xb[VEC], xn[VEC];
        const T(&xv)[VEC] = p.x;
        const T(&x0v)[VEC] = p.x0;
        col_bounds<T, VEC>(j, b0, ld, l, u, ovr, ovl, ovu, lo, hi);
        const T cj = __ldg(c + j);
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            xh[q] = clampbox(xv[q] - L.tau[q] * (cj + s[q]), lo[q], hi[q]);
            xb[q] = T(2) * xh[q] - xv[q];
            xn[q] = L.lam[q] * ((T(1) + T(kRhoB)) * xh[q] - T(kRhoB) * xv[q]) + (T(1) - L.lam[q]) * x0v[q];
            if (CHECK && L.act[q]) {
                const double d0 = static_cast<double>(xh[q]) - static_cast<double>(xv[q]);
                const double d1 = static_cast<double>(xh[q]) - static_cast<double>(x0v[q]);
                red[0][q] += d0 * d0;
                red[1][q] += d1 * d1;
            }
        }
        st_vec<T, VEC>(xbar + at, xb, L.act, L.all);
        st_vec<T, VEC>(x + at, xn, L.act, L.all);
        if (CHECK) st_vec<T, VEC>(xhat + at, xh, L.act, L.all);
    }
};

template <class T, int VEC, bool CHECK>
struct SRowEpi {
    static constexpr int NR = CHECK ? 2 : 0;
    BCtl ctl;
    int it, ld;
    T *y, *yhat;
    const T *y0, *rl, *ru;
    struct Lane : LaneBase<T, VEC> {
        T sigma[VEC], lam[VEC];
    };
    __device__ Lane lane(int b0) const {
        Lane L;
        lane_activity<T, VEC>(ctl, b0, L);
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            const int b = L.act[q] ? b0 + q : 0;
            L.sigma[q] = static_cast<T>(ctl.sigma[b]);
            L.lam[q] = static_cast<T>(lam_of(ctl, b, it));
        }
        return L;
    }
    // the iterate, the anchor and the row bounds, loaded before the row's gathers
    struct Pre {
        T y[VEC], y0[VEC];
        T lo, hi;
    };
    __device__ Pre pre(int i, int b0) const {
        const size_t at = static_cast<size_t>(i) * ld + b0;
        Pre p;
        ld_vec<T, VEC>(y + at, p.y);
        ld_vec<T, VEC>(y0 + at, p.y0);
        p.lo = __ldg(rl + i);
        p.hi = __ldg(ru + i);
        return p;
    }
    __device__ void row(int i, int b0, const Lane &L, const T (&s)[VEC], double (&red)[kSpmmMaxR][VEC],
                        const Pre &p) const {
        const size_t at = static_cast<size_t>(i) * ld + b0;
        T yh[VEC], yn[VEC];
        const T(&yv)[VEC] = p.y;
        const T(&y0v)[VEC] = p.y0;
        const T lo = p.lo, hi = p.hi;
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            const T v = yv[q] + L.sigma[q] * s[q];
            yh[q] = v - clampbox(v, L.sigma[q] * lo, L.sigma[q] * hi);
            yn[q] = L.lam[q] * ((T(1) + T(kRhoB)) * yh[q] - T(kRhoB) * yv[q]) + (T(1) - L.lam[q]) * y0v[q];
            if (CHECK && L.act[q]) {
                const double d0 = static_cast<double>(yh[q]) - static_cast<double>(yv[q]);
                const double d1 = static_cast<double>(yh[q]) - static_cast<double>(y0v[q]);
                red[0][q] += d0 * d0;
                red[1][q] += d1 * d1;
            }
        }
        st_vec<T, VEC>(y + at, yn, L.act, L.all);
        if (CHECK) st_vec<T, VEC>(yhat + at, yh, L.act, L.all);
    }
};

// Relative-KKT pieces (the single-instance definitions, per instance).
template <class T, int VEC>
struct SKktRowEpi {
    static constexpr int NR = 3;
    BCtl ctl;
    int ld;
    const T *yhat, *rl, *ru, *rs;
    using Lane = LaneBase<T, VEC>;
    __device__ Lane lane(int b0) const {
        Lane L;
        lane_activity<T, VEC>(ctl, b0, L);
        return L;
    }
    struct Pre {};
    __device__ Pre pre(int, int) const { return Pre{}; }
    __device__ void row(int i, int b0, const Lane &L, const T (&s)[VEC], double (&red)[kSpmmMaxR][VEC],
                        const Pre &) const {
        T yv[VEC];
        ld_vec<T, VEC>(yhat + static_cast<size_t>(i) * ld + b0, yv);
        const double lo = static_cast<double>(__ldg(rl + i)), hi = static_cast<double>(__ldg(ru + i));
        const double r = static_cast<double>(__ldg(rs + i));
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            if (!L.act[q]) continue;
            const double a = static_cast<double>(s[q]);
            const double pr = (a - clampbox(a, lo, hi)) / r;
            red[0][q] += pr * pr;
            const double y = static_cast<double>(yv[q]);
            const double yl = smax(0.0, -y), yu = smax(0.0, y);
            if (yl > 0.0) {
                if (isfinite(lo)) red[1][q] += lo * yl; else red[2][q] += (r * yl) * (r * yl);
            }
            if (yu > 0.0) {
                if (isfinite(hi)) red[1][q] -= hi * yu; else red[2][q] += (r * yu) * (r * yu);
            }
        }
    }
};

template <class T, int VEC>
struct SKktColEpi {
    static constexpr int NR = 4;
    BCtl ctl;
    int ld;
    const T *xhat, *c, *l, *u, *ovl, *ovu, *cs;
    const int *ovr;
    using Lane = LaneBase<T, VEC>;
    __device__ Lane lane(int b0) const {
        Lane L;
        lane_activity<T, VEC>(ctl, b0, L);
        return L;
    }
    struct Pre {};
    __device__ Pre pre(int, int) const { return Pre{}; }
    __device__ void row(int j, int b0, const Lane &L, const T (&s)[VEC], double (&red)[kSpmmMaxR][VEC],
                        const Pre &) const {
        T xv[VEC], lo[VEC], hi[VEC];
        ld_vec<T, VEC>(xhat + static_cast<size_t>(j) * ld + b0, xv);
        col_bounds<T, VEC>(j, b0, ld, l, u, ovr, ovl, ovu, lo, hi);
        const double cj = static_cast<double>(__ldg(c + j)), d = static_cast<double>(__ldg(cs + j));
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            if (!L.act[q]) continue;
            const double lam = cj + static_cast<double>(s[q]);
            const double a = static_cast<double>(lo[q]), b = static_cast<double>(hi[q]);
            const double x = static_cast<double>(xv[q]);
            const double vl = smax(0.0, lam), vu = smax(0.0, -lam);
            if (vl > 0.0) {
                if (isfinite(a)) red[1][q] += a * vl; else red[0][q] += (vl / d) * (vl / d);
            }
            if (vu > 0.0) {
                if (isfinite(b)) red[1][q] -= b * vu; else red[0][q] += (vu / d) * (vu / d);
            }
            red[2][q] += cj * x;
            const double bx = (x - clampbox(x, a, b)) * d;
            red[3][q] += bx * bx;
        }
    }
};

template <class T>
struct SpmmMat {
    const int *ro, *ci;
    const T *val;
    int rows;
};

// One pass: for every row i and instance b, s = sum_k val_k * X[ci_k * ld + b],
// handed to the epilogue. blockIdx.x = p * G + g: group g of 32*VEC instances,
// block p of the P blocks serving that group (rows p*8 + warp, stride P*8).
// One pass of the shared matrix for every instance group: block p takes rows
// p*kSpmmWarps + warp, stepping by gridDim.x*kSpmmWarps, and walks the
// instance groups g = 0..G-1 in order, so all blocks gather from one group's
// slice of X (n * 32 * VEC values) at a time and that slice stays in L2. A
// group whose instances have all stopped is skipped.
template <class T, int VEC, class Epi>
__global__ void __launch_bounds__(kSpmmWarps * 32, kSpmmMinBlocks)
    spmm_kernel(SpmmMat<T> M, const T *__restrict__ X, int ld, int G, Epi epi, double *__restrict__ partials) {
    constexpr int NR = Epi::NR;
    const int p = blockIdx.x, P = gridDim.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int g = 0; g < G; ++g) {
        const int b0 = g * 32 * VEC + lane * VEC;
        const typename Epi::Lane L = epi.lane(b0);
        double red[kSpmmMaxR][VEC];
#pragma unroll
        for (int r = 0; r < kSpmmMaxR; ++r)
#pragma unroll
            for (int q = 0; q < VEC; ++q) red[r][q] = 0.0;
        const T *Xb = X + b0;
        // the warp's lanes cover the whole group: skip its rows when every
        // instance of the group has stopped (the partials below stay zero)
        bool mine = false;
#pragma unroll
        for (int q = 0; q < VEC; ++q) mine = mine || L.act[q];
        const int rows = __any_sync(0xffffffffu, mine) ? M.rows : 0;
        for (int i = p * kSpmmWarps + warp; i < rows; i += P * kSpmmWarps) {
            const int k0 = __ldg(M.ro + i), k1 = __ldg(M.ro + i + 1);
            const typename Epi::Pre pre = epi.pre(i, b0);
            T acc[VEC];
#pragma unroll
            for (int q = 0; q < VEC; ++q) acc[q] = T(0);
            constexpr int U = kSpmmUnroll;
            int k = k0;
            for (; k + U <= k1; k += U) {
                int cc[U];
                T vv[U], xv[U][VEC];
#pragma unroll
                for (int t = 0; t < U; ++t) {
                    cc[t] = __ldg(M.ci + k + t);
                    vv[t] = __ldg(M.val + k + t);
                }
#pragma unroll
                for (int t = 0; t < U; ++t) ldg_vec<T, VEC>(Xb + static_cast<size_t>(cc[t]) * ld, xv[t]);
#pragma unroll
                for (int t = 0; t < U; ++t)
#pragma unroll
                    for (int q = 0; q < VEC; ++q) acc[q] += vv[t] * xv[t][q];
            }
            for (; k < k1; ++k) {
                const int cc = __ldg(M.ci + k);
                const T vv = __ldg(M.val + k);
                T xv[VEC];
                ldg_vec<T, VEC>(Xb + static_cast<size_t>(cc) * ld, xv);
#pragma unroll
                for (int q = 0; q < VEC; ++q) acc[q] += vv * xv[q];
            }
            epi.row(i, b0, L, acc, red, pre);
        }
        if constexpr (NR > 0) {
            __shared__ double sred[kSpmmWarps][NR][32 * VEC];
#pragma unroll
            for (int r = 0; r < NR; ++r)
#pragma unroll
                for (int q = 0; q < VEC; ++q) sred[warp][r][lane * VEC + q] = red[r][q];
            __syncthreads();
            for (int e = threadIdx.x; e < NR * 32 * VEC; e += blockDim.x) {
                const int r = e / (32 * VEC), t = e % (32 * VEC);
                double acc = 0.0;
                for (int w = 0; w < kSpmmWarps; ++w) acc += sred[w][r][t];
                partials[(static_cast<size_t>(p) * NR + r) * ld + g * 32 * VEC + t] = acc;
            }
            __syncthreads(); // sred is refilled by the next group
        }
    }
}

// out[b * R + r] = sum_p partials[(p * R + r) * ld + b], p in order.
__global__ void spmm_reduce_kernel(const double *__restrict__ partials, int P, int R, int ld, int count,
                                   double *__restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count * R) return;
    const int b = e / R, r = e % R;
    double acc = 0.0;
    for (int p = 0; p < P; ++p) acc += partials[(static_cast<size_t>(p) * R + r) * ld + b];
    out[e] = acc;
}

template <class T>
__global__ void srestart_kernel(BCtl c, int ld, T *x, T *x0, const T *xhat, int64_t nx, T *y, T *y0, const T *yhat,
                                int64_t ny) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int b = static_cast<int>(e % ld);
    if (b >= c.count || !c.restart_now[b] || c.done[b]) return;
    if (e < nx) {
        x[e] = xhat[e];
        x0[e] = xhat[e];
    }
    if (e < ny) {
        y[e] = yhat[e];
        y0[e] = yhat[e];
    }
}

template <class TD, class TS>
__global__ void sconvert_kernel(const TS *__restrict__ a, int64_t n, TD *__restrict__ out) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<TD>(a[i]);
}

// Start point per instance: clamp(warm / D or 0, bounds), interleaved.
__global__ void sstart_kernel(const double *__restrict__ warm, const double *__restrict__ lo,
                              const double *__restrict__ hi, const double *__restrict__ cs, int n, int count, int ld,
                              double *__restrict__ x, double *__restrict__ x0) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<int64_t>(n) * ld) return;
    const int j = static_cast<int>(e / ld), b = static_cast<int>(e % ld);
    double v = 0.0;
    if (b < count) {
        const size_t src = static_cast<size_t>(b) * n + j;
        const double d = cs[j];
        const double l = isfinite(lo[src]) ? lo[src] / d : lo[src];
        const double u = isfinite(hi[src]) ? hi[src] / d : hi[src];
        v = clampbox(warm ? warm[src] / d : 0.0, l, u);
    }
    x[e] = v;
    x0[e] = v;
}

// Override table rows: for each overridden column, the scaled bounds of every instance.
__global__ void soverride_kernel(const double *__restrict__ lo, const double *__restrict__ hi,
                                 const double *__restrict__ cs, const int *__restrict__ cols, int nov, int n,
                                 int count, int ld, double *__restrict__ ovl, double *__restrict__ ovu) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<int64_t>(nov) * ld) return;
    const int o = static_cast<int>(e / ld), b = static_cast<int>(e % ld);
    double l = 0.0, u = 0.0;
    if (b < count) {
        const int j = cols[o];
        const size_t src = static_cast<size_t>(b) * n + j;
        const double d = cs[j];
        l = isfinite(lo[src]) ? lo[src] / d : lo[src];
        u = isfinite(hi[src]) ? hi[src] / d : hi[src];
    }
    ovl[e] = l;
    ovu[e] = u;
}

// out[b] = sum_j c[j] * x[b * n + j] (one block per instance, fixed tree).
__global__ void sobjective_kernel(const double *__restrict__ x, const double *__restrict__ c, int n,
                                  double *__restrict__ out) {
    __shared__ double scratch[32];
    const int b = blockIdx.x;
    const double *xb = x + static_cast<size_t>(b) * n;
    double s[1] = {0.0};
    for (int j = threadIdx.x; j < n; j += blockDim.x) s[0] += c[j] * xb[j];
    block_sum<1>(s, scratch);
    if (threadIdx.x == 0) out[b] = s[0];
}

// out[b * n + j] = a[j * ld + b] * s[j]: unscale and de-interleave.
__global__ void sunscale_kernel(const double *__restrict__ a, const double *__restrict__ s, int n, int count, int ld,
                                double *__restrict__ out) {
    const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<int64_t>(n) * count) return;
    const int b = static_cast<int>(e / n), j = static_cast<int>(e % n);
    out[e] = a[static_cast<size_t>(j) * ld + b] * s[j];
}

template <class T>
struct SState {
    DevBuf<T> x, x0, xbar, xhat, y, y0, yhat, l, u, ovl, ovu, c, rl, ru, rs, cs;
};

inline int grid_for64(int64_t n) { return static_cast<int>(std::max<int64_t>(1, (n + 255) / 256)); }

class SharedEngine {
public:
    SharedEngine(const vk_problem &p, int count, const vk_options &o)
        : o_(o), B_(count), base_(&p, 1, base_options(o)), model_(p) {
        m_ = base_.m_;
        n_ = base_.n_;
        s_ = base_.s_;
        mixed_ = o.precision == VK_PREC_MIXED;
        chunk_ = base_.chunk_;
        const int width = B_ >= 128 ? 128 : 32;
        ld_ = (B_ + width - 1) / width * width;
        vec32_ = B_ >= 128 ? 4 : 1;
        vec64_ = (B_ >= 64 && ld_ % 64 == 0) ? 2 : 1;
        const int sms = sm_count();
        // one resident wave of blocks (kSpmmMinBlocks per SM, the launch bound); each walks every instance group
        P32_ = kSpmmMinBlocks * sms;
        P64_ = kSpmmMinBlocks * sms;
        control_arrays();
        pmax_ = std::max(P32_, P64_);
        partial_.reset(static_cast<size_t>(pmax_) * kSpmmMaxR * ld_);
        sc_.reset(static_cast<size_t>(B_) * 2);
        sr_.reset(static_cast<size_t>(B_) * 2);
        skr_.reset(static_cast<size_t>(B_) * 3);
        skc_.reset(static_cast<size_t>(B_) * 4);
    }
    ~SharedEngine() {
        const auto t0 = std::chrono::steady_clock::now();
        if (g64_) cudaGraphExecDestroy(g64_);
        if (g32_) cudaGraphExecDestroy(g32_);
        if (o_.verbose > 0)
            std::fprintf(stderr, "[vikalp_b200] shared: graphs destroyed          %8.3f s\n", seconds_since(t0));
    }

    void solve(const double *lower, const double *upper, const double *warm, vk_result *results) {
        const auto started = std::chrono::steady_clock::now();
        PhaseLog lg(o_.verbose, "shared", s_);
        const int n = n_, m = m_;
        // per-instance checks (continuous_common.hpp:80-110, pdhg.cpp:29-33)
        std::vector<int> invalid(B_, 0);
        std::vector<std::string> why(B_);
        std::vector<char> overridden(n, 0);
        // instances [b0, b1); `ovr` marks the columns whose bounds differ from the model's
        auto check = [&](int b0, int b1, std::vector<char> &ovr) {
            for (int b = b0; b < b1; ++b) {
                const size_t o = static_cast<size_t>(b) * n;
                for (int j = 0; j < n && !invalid[b]; ++j) {
                    const double l = lower ? lower[o + j] : model_.var_lower[j];
                    const double u = upper ? upper[o + j] : model_.var_upper[j];
                    if ((lower && std::isnan(lower[o + j])) || (upper && std::isnan(upper[o + j]))) {
                        invalid[b] = 1;
                        why[b] = "variable bound overrides must be empty or sized and non-NaN";
                    } else if (std::isnan(l) || std::isnan(u) || l > u) {
                        invalid[b] = 1;
                        why[b] = "variable bound overrides contain an invalid interval";
                    } else if (warm && !std::isfinite(warm[o + j])) {
                        invalid[b] = 1;
                        why[b] = "warm start must be empty or finite and sized to the model";
                    }
                    if (l != model_.var_lower[j] || u != model_.var_upper[j]) ovr[j] = 1;
                }
            }
        };
        {
            // instances split over host threads (each its own column marks)
            const unsigned hw = std::thread::hardware_concurrency();
            const int64_t work = static_cast<int64_t>(B_) * n;
            const int T = work < (int64_t(1) << 20) ? 1 : std::min<int>({B_, 16, static_cast<int>(hw == 0 ? 1 : hw)});
            std::vector<std::vector<char>> marks(T, std::vector<char>(T > 1 ? n : 0, 0));
            if (T <= 1) {
                check(0, B_, overridden);
            } else {
                std::vector<std::thread> pool;
                for (int t = 1; t < T; ++t)
                    pool.emplace_back([&, t] { check(B_ * t / T, B_ * (t + 1) / T, marks[t]); });
                check(0, B_ / T, marks[0]);
                for (std::thread &th : pool) th.join();
                for (int t = 0; t < T; ++t)
                    for (int j = 0; j < n; ++j) overridden[j] |= marks[t][j];
            }
        }
        std::vector<int> ov_cols, ov_index(n, -1);
        for (int j = 0; j < n; ++j)
            if (overridden[j]) {
                ov_index[j] = static_cast<int>(ov_cols.size());
                ov_cols.push_back(j);
            }
        const int nov = static_cast<int>(ov_cols.size());
        lg.mark("instance checks (host)");
        // bounds and warm start of every instance, on the device
        const size_t bn = static_cast<size_t>(B_) * n;
        DevBuf<double> dlo(bn), dhi(bn), dwarm(warm ? bn : 1);
        {
            std::vector<double> tmp;
            for (int side = 0; side < 2; ++side) {
                const double *src = side == 0 ? lower : upper;
                const double *model = side == 0 ? model_.var_lower : model_.var_upper;
                DevBuf<double> &dst = side == 0 ? dlo : dhi;
                if (src) {
                    stage_h2d(dst.get(), src, bn * sizeof(double), s_);
                } else {
                    tmp.resize(bn);
                    for (int b = 0; b < B_; ++b) std::copy(model, model + n, tmp.begin() + static_cast<size_t>(b) * n);
                    stage_h2d(dst.get(), tmp.data(), bn * sizeof(double), s_);
                }
            }
            if (warm) stage_h2d(dwarm.get(), warm, bn * sizeof(double), s_);
        }
        DevBuf<int> dov_index, dov_cols;
        dov_index.reset(n);
        VK_CUDA(cudaMemcpyAsync(dov_index.get(), ov_index.data(), n * sizeof(int), cudaMemcpyHostToDevice, s_));
        dov_cols.reset(std::max(nov, 1));
        if (nov > 0)
            VK_CUDA(cudaMemcpyAsync(dov_cols.get(), ov_cols.data(), nov * sizeof(int), cudaMemcpyHostToDevice, s_));
        // float64 state
        alloc_state(s64_, nov);
        state_model(s64_);
        const int64_t nx = static_cast<int64_t>(n) * ld_, ny = static_cast<int64_t>(m) * ld_;
        sstart_kernel<<<grid_for64(nx), 256, 0, s_>>>(warm ? dwarm.get() : nullptr, dlo.get(), dhi.get(),
                                                      base_.cs_.get(), n, B_, ld_, s64_.x.get(), s64_.x0.get());
        if (nov > 0)
            soverride_kernel<<<grid_for64(static_cast<int64_t>(nov) * ld_), 256, 0, s_>>>(
                dlo.get(), dhi.get(), base_.cs_.get(), dov_cols.get(), nov, n, B_, ld_, s64_.ovl.get(), s64_.ovu.get());
        VK_LAUNCH_CHECK();
        if (m > 0) {
            VK_CUDA(cudaMemsetAsync(s64_.y.get(), 0, ny * sizeof(double), s_));
            VK_CUDA(cudaMemsetAsync(s64_.y0.get(), 0, ny * sizeof(double), s_));
            VK_CUDA(cudaMemsetAsync(s64_.yhat.get(), 0, ny * sizeof(double), s_));
        }
        VK_CUDA(cudaMemsetAsync(s64_.xhat.get(), 0, nx * sizeof(double), s_));
        VK_CUDA(cudaMemsetAsync(s64_.xbar.get(), 0, nx * sizeof(double), s_));
        ov_ = dov_index.get();
        reset_control(invalid);
        lg.mark("upload + start points");

        cudaEvent_t e0, e1;
        VK_CUDA(cudaEventCreate(&e0));
        VK_CUDA(cudaEventCreate(&e1));
        VK_CUDA(cudaEventRecord(e0, s_));
        long long launches = 0, fp32_iters = 0;
        bool timed_out = false;
        if (g64_) {
            cudaGraphExecDestroy(g64_);
            g64_ = nullptr;
        }
        if (g32_) {
            cudaGraphExecDestroy(g32_);
            g32_ = nullptr;
        }
        if (mixed_) {
            alloc_state(s32_, nov);
            state_model(s32_);
            copy_state<float, double>(s64_, s32_, nov, true);
            g32_ = vec32_ == 4 ? capture<float, 4>(s32_) : capture<float, 1>(s32_);
            lg.mark("float32 state + graph");
            std::vector<double> best(B_, std::numeric_limits<double>::infinity());
            int stall = 0;
            for (;;) {
                if (over_time(started)) {
                    timed_out = true;
                    break;
                }
                VK_CUDA(cudaGraphLaunch(g32_, s_));
                launches += nodes_;
                read_control();
                check_device_error(s_);
                bool improved = false, all_done = true;
                double worst = 0.0;
                for (int b = 0; b < B_; ++b) {
                    if (h_done_[b]) continue;
                    all_done = false;
                    worst = std::max(worst, h_kkt_[b]);
                    if (h_kkt_[b] < 0.7 * best[b]) {
                        best[b] = h_kkt_[b];
                        improved = true;
                    }
                }
                if (all_done) break;
                if (improved)
                    stall = 0;
                else if (++stall >= 6 && worst < 1e-3)
                    break;
            }
            fp32_iters = h_iters_.empty() ? 0 : *std::max_element(h_iters_.begin(), h_iters_.end());
            lg.mark("float32 iterations");
            copy_state<double, float>(s32_, s64_, nov, false);
            reopen(invalid);
        }
        if (!timed_out) {
            g64_ = vec64_ == 2 ? capture<double, 2>(s64_) : capture<double, 1>(s64_);
            for (;;) {
                if (over_time(started)) {
                    timed_out = true;
                    break;
                }
                VK_CUDA(cudaGraphLaunch(g64_, s_));
                launches += nodes_;
                read_control();
                check_device_error(s_);
                if (std::all_of(h_done_.begin(), h_done_.end(), [](int d) { return d != 0; })) break;
            }
        }
        lg.mark("float64 iterations");
        VK_CUDA(cudaEventRecord(e1, s_));
        read_control();
        float ms = 0.f;
        VK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        // answers (x^, y^) in original units, instance-major
        DevBuf<double> xo(bn), yo(std::max<size_t>(1, static_cast<size_t>(B_) * m));
        sunscale_kernel<<<grid_for64(static_cast<int64_t>(bn)), 256, 0, s_>>>(s64_.xhat.get(), base_.cs_.get(), n, B_,
                                                                             ld_, xo.get());
        if (m > 0)
            sunscale_kernel<<<grid_for64(static_cast<int64_t>(B_) * m), 256, 0, s_>>>(
                s64_.yhat.get(), base_.rs_.get(), m, B_, ld_, yo.get());
        // objectives on the device (one block per instance), then x and y
        // straight into the caller's arrays
        DevBuf<double> dobj(B_);
        sobjective_kernel<<<B_, 256, 0, s_>>>(xo.get(), base_.c_orig(), n, dobj.get());
        VK_LAUNCH_CHECK();
        std::vector<double> hobj(B_);
        VK_CUDA(cudaMemcpyAsync(hobj.data(), dobj.get(), B_ * sizeof(double), cudaMemcpyDeviceToHost, s_));
        std::vector<StageCopy> copies;
        copies.reserve(2 * static_cast<size_t>(B_));
        for (int b = 0; b < B_; ++b) {
            if (invalid[b]) continue;
            if (results[b].x) copies.push_back({results[b].x, xo.get() + static_cast<size_t>(b) * n, n * sizeof(double)});
            if (results[b].y && m > 0)
                copies.push_back({results[b].y, yo.get() + static_cast<size_t>(b) * m, m * sizeof(double)});
        }
        stage_d2h_many(copies.data(), static_cast<int64_t>(copies.size()), s_);
        VK_CUDA(cudaStreamSynchronize(s_));
        lg.mark("results to host");
        const double secs = seconds_since(started);
        for (int b = 0; b < B_; ++b) {
            vk_result &r = results[b];
            r.message[0] = '\0';
            r.primal_residual = r.stationarity_residual = r.complementarity_residual =
                std::numeric_limits<double>::quiet_NaN();
            r.solve_seconds = secs;
            r.iterate_seconds = ms * 1e-3;
            r.kernel_launches = launches;
            if (invalid[b]) {
                r.status = VK_STATUS_INVALID_MODEL;
                std::snprintf(r.message, sizeof(r.message), "%s", why[b].c_str());
                r.iterations = r.restarts = r.fp32_iterations = 0;
                r.objective = r.rel_primal = r.rel_dual = r.rel_gap = r.last_metric =
                    std::numeric_limits<double>::quiet_NaN();
                continue;
            }
            r.objective = model_.objective_offset + hobj[b];
            r.status = h_done_[b] ? h_status_[b] : (timed_out ? VK_STATUS_TIME_LIMIT : VK_STATUS_ITERATION_LIMIT);
            r.iterations = h_iters_[b];
            r.restarts = h_restarts_[b];
            r.rel_primal = h_rel_p_[b];
            r.rel_dual = h_rel_d_[b];
            r.rel_gap = h_rel_gap_[b];
            r.last_metric = h_kkt_[b];
            r.fp32_iterations = std::min<long long>(fp32_iters, h_iters_[b]);
        }
    }

private:
    static vk_options base_options(const vk_options &o) {
        vk_options b = o;
        b.precision = VK_PREC_MIXED; // builds float32 and float64 copies of the scaled model
        return b;
    }
    static int sm_count() {
        int dev = 0, sms = 148;
        VK_CUDA(cudaGetDevice(&dev));
        VK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        return sms;
    }
    bool over_time(std::chrono::steady_clock::time_point t0) const {
        return std::isfinite(o_.time_limit_seconds) && seconds_since(t0) >= o_.time_limit_seconds;
    }

    template <class T>
    void alloc_state(SState<T> &st, int nov) {
        const size_t nx = static_cast<size_t>(n_) * ld_, ny = std::max<size_t>(1, static_cast<size_t>(m_) * ld_);
        const size_t no = std::max<size_t>(1, static_cast<size_t>(nov) * ld_);
        for (DevBuf<T> *b : {&st.x, &st.x0, &st.xbar, &st.xhat}) b->reset(nx);
        for (DevBuf<T> *b : {&st.y, &st.y0, &st.yhat}) b->reset(ny);
        st.ovl.reset(no);
        st.ovu.reset(no);
    }

    // Shared scaled model vectors in T (c, bounds, row bounds, scales).
    template <class T>
    void state_model(SState<T> &st) {
        const int n = n_, m = std::max(m_, 1);
        for (DevBuf<T> *b : {&st.l, &st.u, &st.c, &st.cs}) b->reset(n);
        for (DevBuf<T> *b : {&st.rl, &st.ru, &st.rs}) b->reset(m);
        auto &src = base_.s64_;
        sconvert_kernel<T, double><<<grid1d(n), 256, 0, s_>>>(src.l.get(), n, st.l.get());
        sconvert_kernel<T, double><<<grid1d(n), 256, 0, s_>>>(src.u.get(), n, st.u.get());
        sconvert_kernel<T, double><<<grid1d(n), 256, 0, s_>>>(src.c.get(), n, st.c.get());
        sconvert_kernel<T, double><<<grid1d(n), 256, 0, s_>>>(base_.cs_.get(), n, st.cs.get());
        if (m_ > 0) {
            sconvert_kernel<T, double><<<grid1d(m_), 256, 0, s_>>>(src.rl.get(), m_, st.rl.get());
            sconvert_kernel<T, double><<<grid1d(m_), 256, 0, s_>>>(src.ru.get(), m_, st.ru.get());
            sconvert_kernel<T, double><<<grid1d(m_), 256, 0, s_>>>(base_.rs_.get(), m_, st.rs.get());
        }
        VK_LAUNCH_CHECK();
    }

    template <class TD, class TS>
    void copy_state(const SState<TS> &a, SState<TD> &b, int nov, bool bounds) {
        const int64_t nx = static_cast<int64_t>(n_) * ld_, ny = static_cast<int64_t>(m_) * ld_;
        for (auto pr : {std::make_pair(&a.x, &b.x), std::make_pair(&a.x0, &b.x0), std::make_pair(&a.xhat, &b.xhat),
                        std::make_pair(&a.xbar, &b.xbar)})
            sconvert_kernel<TD, TS><<<grid_for64(nx), 256, 0, s_>>>(pr.first->get(), nx, pr.second->get());
        if (ny > 0)
            for (auto pr : {std::make_pair(&a.y, &b.y), std::make_pair(&a.y0, &b.y0), std::make_pair(&a.yhat, &b.yhat)})
                sconvert_kernel<TD, TS><<<grid_for64(ny), 256, 0, s_>>>(pr.first->get(), ny, pr.second->get());
        if (bounds && nov > 0) {
            const int64_t no = static_cast<int64_t>(nov) * ld_;
            sconvert_kernel<TD, TS><<<grid_for64(no), 256, 0, s_>>>(a.ovl.get(), no, b.ovl.get());
            sconvert_kernel<TD, TS><<<grid_for64(no), 256, 0, s_>>>(a.ovu.get(), no, b.ovu.get());
        }
        VK_LAUNCH_CHECK();
    }

    void control_arrays() {
        const size_t Bs = B_;
        for (DevBuf<double> *d : {&eta_, &omega_, &tau_, &sigma_, &rr_, &rp_, &bn_, &cn_, &off_, &kkt_, &relp_, &reld_,
                                  &relg_})
            d->reset(Bs);
        for (DevBuf<long long> *d : {&kb_, &it_, &rst_}) d->reset(Bs);
        for (DevBuf<int> *d : {&done_, &status_, &rnow_}) d->reset(Bs);
        h_done_.resize(B_);
        h_status_.resize(B_);
        h_iters_.resize(B_);
        h_restarts_.resize(B_);
        h_kkt_.resize(B_);
        h_rel_p_.resize(B_);
        h_rel_d_.resize(B_);
        h_rel_gap_.resize(B_);
    }

    BCtl ctl() {
        BCtl c{};
        c.eta = eta_.get();
        c.omega = omega_.get();
        c.tau = tau_.get();
        c.sigma = sigma_.get();
        c.r_restart = rr_.get();
        c.r_prev = rp_.get();
        c.bnorm = bn_.get();
        c.cnorm = cn_.get();
        c.offset = off_.get();
        c.kkt = kkt_.get();
        c.rel_p = relp_.get();
        c.rel_d = reld_.get();
        c.rel_gap = relg_.get();
        c.k_base = kb_.get();
        c.iters = it_.get();
        c.restarts = rst_.get();
        c.done = done_.get();
        c.status = status_.get();
        c.restart_now = rnow_.get();
        c.tol = o_.relative_tolerance;
        c.limit = o_.iteration_limit;
        c.count = B_;
        const PrimalWeightRule pw = primal_weight_rule();
        c.theta = pw.theta;
        c.freeze = pw.freeze;
        c.beta_suff = pw.beta_suff;
        c.beta_nec = pw.beta_nec;
        c.beta_art = pw.beta_art;
        return c;
    }

    void fill(DevBuf<double> &d, double v) {
        std::vector<double> h(B_, v);
        VK_CUDA(cudaMemcpyAsync(d.get(), h.data(), B_ * sizeof(double), cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaStreamSynchronize(s_));
    }

    void reset_control(const std::vector<int> &invalid) {
        const double eta = base_.h_eta_[0], w0 = base_.h_omega0_[0] * primal_weight_rule().start;
        fill(eta_, eta);
        fill(omega_, w0);
        fill(tau_, eta / w0);
        fill(sigma_, eta * w0);
        fill(rr_, -1.0);
        fill(rp_, std::numeric_limits<double>::infinity());
        fill(kkt_, std::numeric_limits<double>::infinity());
        fill(bn_, base_.bnorm_[0]);
        fill(cn_, base_.cnorm_[0]);
        fill(off_, model_.objective_offset);
        for (DevBuf<long long> *d : {&kb_, &it_, &rst_}) VK_CUDA(cudaMemsetAsync(d->get(), 0, d->bytes(), s_));
        VK_CUDA(cudaMemsetAsync(rnow_.get(), 0, rnow_.bytes(), s_));
        std::vector<int> st(B_);
        for (int b = 0; b < B_; ++b) st[b] = invalid[b] ? VK_STATUS_INVALID_MODEL : VK_STATUS_NOT_SOLVED;
        VK_CUDA(cudaMemcpyAsync(done_.get(), invalid.data(), B_ * sizeof(int), cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaMemcpyAsync(status_.get(), st.data(), B_ * sizeof(int), cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaStreamSynchronize(s_));
    }

    void reopen(const std::vector<int> &invalid) {
        read_control();
        std::vector<int> done(B_), status(B_);
        for (int b = 0; b < B_; ++b) {
            const bool keep = invalid[b] || h_status_[b] == VK_STATUS_NUMERICAL_FAILURE;
            done[b] = keep ? 1 : 0;
            status[b] = keep ? h_status_[b] : VK_STATUS_NOT_SOLVED;
        }
        VK_CUDA(cudaMemcpyAsync(done_.get(), done.data(), B_ * sizeof(int), cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaMemcpyAsync(status_.get(), status.data(), B_ * sizeof(int), cudaMemcpyHostToDevice, s_));
        VK_CUDA(cudaStreamSynchronize(s_));
    }

    void read_control() {
        VK_CUDA(cudaMemcpyAsync(h_done_.data(), done_.get(), B_ * sizeof(int), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_status_.data(), status_.get(), B_ * sizeof(int), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_iters_.data(), it_.get(), B_ * sizeof(long long), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_restarts_.data(), rst_.get(), B_ * sizeof(long long), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_kkt_.data(), kkt_.get(), B_ * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_rel_p_.data(), relp_.get(), B_ * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_rel_d_.data(), reld_.get(), B_ * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(h_rel_gap_.data(), relg_.get(), B_ * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaStreamSynchronize(s_));
    }

    template <class T>
    SpmmMat<T> mat(bool transposed) {
        const CsrPattern32 &p = transposed ? base_.at_ : base_.a_;
        const T *val;
        if constexpr (std::is_same<T, double>::value)
            val = transposed ? base_.s64_.kat.get() : base_.s64_.ka.get();
        else
            val = transposed ? base_.s32_.kat.get() : base_.s32_.ka.get();
        return SpmmMat<T>{p.ro.get(), p.ci.get(), val, p.rows};
    }

    template <class T, int VEC, class Epi>
    void pass(bool transposed, const T *X, const Epi &e) {
        const int G = ld_ / (32 * VEC);
        const int P = std::is_same<T, double>::value ? P64_ : P32_;
        const SpmmMat<T> M = mat<T>(transposed);
        if (M.rows == 0) return;
        spmm_kernel<T, VEC, Epi><<<P, kSpmmWarps * 32, 0, s_>>>(M, X, ld_, G, e, partial_.get());
        VK_LAUNCH_CHECK();
    }

    void reduce(int R, DevBuf<double> &out, int P) {
        spmm_reduce_kernel<<<grid1d(int64_t(B_) * R), 256, 0, s_>>>(partial_.get(), P, R, ld_, B_, out.get());
        VK_LAUNCH_CHECK();
    }

    template <class T, int VEC>
    cudaGraphExec_t capture(SState<T> &st) {
        const int P = std::is_same<T, double>::value ? P64_ : P32_;
        VK_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
        const BCtl c = ctl();
        // without rows the transposed matrix has n empty rows: the column
        // passes still run (s = 0) and never read the gathered vector
        const T *yg = m_ > 0 ? st.y.get() : st.x.get();
        const T *yhg = m_ > 0 ? st.yhat.get() : st.x.get();
        for (int it = 0; it < chunk_; ++it) {
            const bool check = it == chunk_ - 1;
            if (check) {
                pass<T, VEC>(true, yg, SColEpi<T, VEC, true>{c, it, ld_, st.x.get(), st.xbar.get(), st.xhat.get(),
                                                             st.x0.get(), st.c.get(), st.l.get(), st.u.get(),
                                                             st.ovl.get(), st.ovu.get(), ov_});
                reduce(2, sc_, P);
                if (m_ > 0) {
                    pass<T, VEC>(false, st.xbar.get(),
                                 SRowEpi<T, VEC, true>{c, it, ld_, st.y.get(), st.yhat.get(), st.y0.get(),
                                                       st.rl.get(), st.ru.get()});
                    reduce(2, sr_, P);
                    pass<T, VEC>(false, st.xhat.get(),
                                 SKktRowEpi<T, VEC>{c, ld_, st.yhat.get(), st.rl.get(), st.ru.get(), st.rs.get()});
                    reduce(3, skr_, P);
                } else {
                    VK_CUDA(cudaMemsetAsync(sr_.get(), 0, sr_.bytes(), s_));
                    VK_CUDA(cudaMemsetAsync(skr_.get(), 0, skr_.bytes(), s_));
                }
                pass<T, VEC>(true, yhg, SKktColEpi<T, VEC>{c, ld_, st.xhat.get(), st.c.get(), st.l.get(), st.u.get(),
                                                          st.ovl.get(), st.ovu.get(), st.cs.get(), ov_});
                reduce(4, skc_, P);
                batch_control_kernel<<<ceil_div(B_, 128), 128, 0, s_>>>(c, sc_.get(), sr_.get(), skr_.get(),
                                                                        skc_.get(), chunk_);
                const int64_t nx = static_cast<int64_t>(n_) * ld_, ny = static_cast<int64_t>(m_) * ld_;
                srestart_kernel<T><<<grid_for64(std::max(nx, ny)), 256, 0, s_>>>(
                    c, ld_, st.x.get(), st.x0.get(), st.xhat.get(), nx, st.y.get(), st.y0.get(), st.yhat.get(), ny);
                VK_LAUNCH_CHECK();
            } else {
                pass<T, VEC>(true, yg, SColEpi<T, VEC, false>{c, it, ld_, st.x.get(), st.xbar.get(), st.xhat.get(),
                                                              st.x0.get(), st.c.get(), st.l.get(), st.u.get(),
                                                              st.ovl.get(), st.ovu.get(), ov_});
                if (m_ > 0)
                    pass<T, VEC>(false, st.xbar.get(),
                                 SRowEpi<T, VEC, false>{c, it, ld_, st.y.get(), st.yhat.get(), st.y0.get(),
                                                        st.rl.get(), st.ru.get()});
            }
        }
        cudaGraph_t g;
        VK_CUDA(cudaStreamEndCapture(s_, &g));
        size_t nodes = 0;
        VK_CUDA(cudaGraphGetNodes(g, nullptr, &nodes));
        nodes_ = static_cast<long long>(nodes);
        cudaGraphExec_t ex;
        VK_CUDA(cudaGraphInstantiate(&ex, g, 0));
        cudaGraphDestroy(g);
        return ex;
    }

    vk_options o_;
    int B_;
    BatchEngine base_;
    const vk_problem &model_;
    int m_ = 0, n_ = 0, ld_ = 0, vec32_ = 1, vec64_ = 1, P32_ = 1, P64_ = 1, pmax_ = 1, chunk_ = 64;
    bool mixed_ = false;
    cudaStream_t s_ = nullptr;
    const int *ov_ = nullptr;
    SState<double> s64_;
    SState<float> s32_;
    DevBuf<double> partial_, sc_, sr_, skr_, skc_;
    DevBuf<double> eta_, omega_, tau_, sigma_, rr_, rp_, bn_, cn_, off_, kkt_, relp_, reld_, relg_;
    DevBuf<long long> kb_, it_, rst_;
    DevBuf<int> done_, status_, rnow_;
    std::vector<int> h_done_, h_status_;
    std::vector<long long> h_iters_, h_restarts_;
    std::vector<double> h_kkt_, h_rel_p_, h_rel_d_, h_rel_gap_;
    cudaGraphExec_t g64_ = nullptr, g32_ = nullptr;
    long long nodes_ = 0;
};

} // namespace

// Validates every instance (LP only) and runs the batch.
namespace {

// Post-processing of one batch member's point (x, y) in original
// coordinates, as the single-instance solve does it (pdhg.cpp:153-264): split
// row duals max(0, -y) / max(0, y), stationarity s = c + A'y, variable duals
// max(0, s) / max(0, -s) at bounds within active_tol, and the reference's
// three infinity-norm residuals (row and box violation; |x - clamp(x - s)|;
// complementarity). A x is summed row by row and A'y is scattered in row
// order onto c, the reference CPU backend's orders (cpu_ops.cpp:418-427,
// 444-458). Writes only the arrays the caller supplied (non-null).
void postprocess_member(const vk_csr &A, const double *c, const double *rl, const double *ru, const double *lo,
                        const double *hi, double atol, vk_result &r, std::vector<double> &s) {
    const int64_t m = A.rows, n = A.cols;
    const double *x = r.x, *y = r.y;
    double pres = 0.0, stat = 0.0, comp = 0.0;
    s.assign(c, c + n);
    for (int64_t i = 0; i < m; ++i) {
        double v = 0.0;
        const double yi = y[i];
        for (int64_t k = A.row_offsets[i]; k < A.row_offsets[i + 1]; ++k) {
            v += A.values[k] * x[A.col_indices[k]];
            s[A.col_indices[k]] += A.values[k] * yi;
        }
        const double l = rl[i], u = ru[i];
        const bool fl = std::isfinite(l), fu = std::isfinite(u);
        if (fl) pres = std::max(pres, l - v);
        if (fu) pres = std::max(pres, v - u);
        const double dl = std::max(0.0, -yi), du = std::max(0.0, yi);
        if (r.row_lower_dual) r.row_lower_dual[i] = dl;
        if (r.row_upper_dual) r.row_upper_dual[i] = du;
        if (fl) comp = std::max(comp, std::abs((v - l) * dl));
        if (fu) comp = std::max(comp, std::abs((u - v) * du));
    }
    for (int64_t j = 0; j < n; ++j) {
        const double st = s[j], xj = x[j], l = lo[j], u = hi[j];
        const bool fl = std::isfinite(l), fu = std::isfinite(u);
        const double t = xj - st;
        const double proj = (t < l) ? l : ((u < t) ? u : t); // std::clamp (pdhg.cpp:206-208)
        stat = std::max(stat, std::abs(xj - proj));
        double dl = 0.0, du = 0.0;
        if (fl && xj - l <= atol) {
            dl = std::max(0.0, st);
            comp = std::max(comp, std::abs((xj - l) * dl));
        }
        if (fu && u - xj <= atol) {
            du = std::max(0.0, -st);
            comp = std::max(comp, std::abs((u - xj) * du));
        }
        if (r.var_lower_dual) r.var_lower_dual[j] = dl;
        if (r.var_upper_dual) r.var_upper_dual[j] = du;
        if (fl) pres = std::max(pres, l - xj);
        if (fu) pres = std::max(pres, xj - u);
    }
    r.primal_residual = pres;
    r.stationarity_residual = stat;
    r.complementarity_residual = comp;
}

bool wants_duals(const vk_result &r) {
    return r.row_lower_dual || r.row_upper_dual || r.var_lower_dual || r.var_upper_dual;
}

// Runs f(b) for b in [0, count) over up to 16 host threads; the first
// exception (in member order) is rethrown on the calling thread.
template <class F>
void for_members(int count, F &&f) {
    const unsigned hw = std::thread::hardware_concurrency();
    const int T = std::max(1, std::min<int>({count, 16, static_cast<int>(hw == 0 ? 1 : hw)}));
    std::atomic<int> next{0};
    std::vector<std::exception_ptr> err(count);
    auto work = [&] {
        const bool was = serial_host_work();
        set_serial_host_work(true); // no threads of their own inside the members' work
        for (int b = next++; b < count; b = next++) {
            try {
                f(b);
            } catch (...) {
                err[b] = std::current_exception();
            }
        }
        set_serial_host_work(was);
    };
    std::vector<std::thread> pool;
    try {
        for (int t = 1; t < T; ++t) pool.emplace_back(work);
    } catch (const std::system_error &) {
        // fewer threads than asked for: the ones running (and this one) share the members
    }
    work();
    for (std::thread &th : pool) th.join();
    for (const std::exception_ptr &e : err)
        if (e) std::rethrow_exception(e);
}

double active_tolerance(const vk_options &o) { return std::max(10.0 * o.primal_tolerance, 1e-8); }

} // namespace

namespace {

// Checks of an independent batch (every member with vk_pdhg_create's rules,
// over host threads; the first failing member in order is reported).
void validate_batch(const vk_problem *probs, int count, const vk_options &o) {
    if (count <= 0) throw InvalidInput("count must be positive");
    if (o.algorithm != VK_ALGO_HALPERN) throw Unsupported("batched solves use VK_ALGO_HALPERN");
    std::vector<std::string> msgs(count);
    std::vector<char> unsup(count, 0);
    for_members(count, [&](int b) {
        bool unsupported = false;
        msgs[b] = validate_problem(probs[b], o, unsupported);
        unsup[b] = unsupported ? 1 : 0;
    });
    int64_t m = 0, n = 0, nnz = 0;
    for (int b = 0; b < count; ++b) {
        if (!msgs[b].empty()) {
            const std::string full = "instance " + std::to_string(b) + ": " + msgs[b];
            if (unsup[b]) throw Unsupported(full);
            throw InvalidInput(full);
        }
        if (probs[b].Q.rows > 0 && probs[b].Q.row_offsets && probs[b].Q.row_offsets[probs[b].Q.rows] > 0)
            throw Unsupported("instance " + std::to_string(b) + ": batched solves take LPs");
        m += probs[b].A.rows;
        n += probs[b].A.cols;
        nnz += probs[b].A.rows > 0 ? probs[b].A.row_offsets[probs[b].A.rows] : 0;
    }
    if (m >= (int64_t(1) << 31) || n >= (int64_t(1) << 31) || nnz >= (int64_t(1) << 31))
        throw Unsupported("the batch exceeds the int32 index range of the device structures");
}

// Checks of a node batch (the model, LP only, and the batch's size).
void validate_shared(const vk_problem &p, int count, const vk_options &o) {
    if (count <= 0) throw InvalidInput("count must be positive");
    if (o.algorithm != VK_ALGO_HALPERN) throw Unsupported("batched solves use VK_ALGO_HALPERN");
    bool unsupported = false;
    const std::string msg = validate_problem(p, o, unsupported);
    if (!msg.empty()) {
        if (unsupported) throw Unsupported(msg);
        throw InvalidInput(msg);
    }
    if (p.Q.rows > 0 && p.Q.row_offsets && p.Q.row_offsets[p.Q.rows] > 0) throw Unsupported("batched solves take LPs");
    const int64_t ld = (static_cast<int64_t>(count) + 127) / 128 * 128;
    if ((p.A.cols + 1) * ld >= (int64_t(1) << 40) || count >= (1 << 24))
        throw Unsupported("the batch is too large for one device");
}

// Split duals and the reference's residuals of every independent member whose
// caller asked for dual arrays (and passed x, y).
void post_batch(const vk_problem *probs, int count, const vk_options &o, vk_result *results) {
    for_members(count, [&](int b) {
        vk_result &r = results[b];
        if (!wants_duals(r) || !r.x || (!r.y && probs[b].A.rows > 0)) return;
        const vk_problem &p = probs[b];
        std::vector<double> s;
        postprocess_member(p.A, p.c, p.row_lower, p.row_upper, p.var_lower, p.var_upper, active_tolerance(o), r, s);
    });
}

// The same for every node, under the node's own bounds.
void post_shared(const vk_problem &p, int count, const double *lower, const double *upper, const vk_options &o,
                 vk_result *results) {
    const int64_t n = p.A.cols;
    for_members(count, [&](int b) {
        vk_result &r = results[b];
        if (r.status == VK_STATUS_INVALID_MODEL || !wants_duals(r) || !r.x || (!r.y && p.A.rows > 0)) return;
        const double *lo = lower ? lower + static_cast<size_t>(b) * n : p.var_lower;
        const double *hi = upper ? upper + static_cast<size_t>(b) * n : p.var_upper;
        std::vector<double> s;
        postprocess_member(p.A, p.c, p.row_lower, p.row_upper, lo, hi, active_tolerance(o), r, s);
    });
}

} // namespace

void batch_solve(const vk_problem *probs, int count, const vk_options &o, vk_result *results) {
    validate_batch(probs, count, o);
    const auto t0 = std::chrono::steady_clock::now();
    {
        BatchEngine eng(probs, count, o);
        eng.solve(results);
    }
    post_batch(probs, count, o, results);
    if (o.verbose > 0)
        std::fprintf(stderr, "[vikalp_b200] batch: total incl. release       %8.3f s\n", seconds_since(t0));
}

// Validates the model (LP only) and solves `count` relaxations of it that
// differ in variable bounds / warm start.
void batch_solve_shared(const vk_problem &p, int count, const double *lower, const double *upper,
                        const double *warm, const vk_options &o, vk_result *results) {
    validate_shared(p, count, o);
    const auto t0 = std::chrono::steady_clock::now();
    std::chrono::steady_clock::time_point t1;
    {
        SharedEngine eng(p, count, o);
        eng.solve(lower, upper, warm, results);
        t1 = std::chrono::steady_clock::now();
    }
    post_shared(p, count, lower, upper, o, results);
    if (o.verbose > 0) {
        std::fprintf(stderr, "[vikalp_b200] shared: release (graphs, memory)  %8.3f s\n", seconds_since(t1));
        std::fprintf(stderr, "[vikalp_b200] shared: total incl. release      %8.3f s\n", seconds_since(t0));
    }
}

void batch_solve_together(const vk_problem &shared, int node_count, const double *lower, const double *upper,
                          const double *warm, const vk_problem *probs, int count, const vk_options &o,
                          vk_result *node_results, vk_result *results) {
    validate_shared(shared, node_count, o);
    validate_batch(probs, count, o);
    const auto t0 = std::chrono::steady_clock::now();
    {
        // both set-ups first (they allocate and free device memory, which
        // synchronises the device), then both iteration loops at once, each
        // engine on its own stream from its own host thread
        SharedEngine nodes(shared, node_count, o);
        BatchEngine lps(probs, count, o);
        if (o.verbose > 0)
            std::fprintf(stderr, "[vikalp_b200] together: both set-ups         %8.3f s\n", seconds_since(t0));
        std::exception_ptr err;
        std::thread other([&] {
            try {
                VK_CUDA(cudaSetDevice(o.device));
                lps.solve(results);
            } catch (...) {
                err = std::current_exception();
            }
        });
        std::exception_ptr mine;
        try {
            nodes.solve(lower, upper, warm, node_results);
        } catch (...) {
            mine = std::current_exception();
        }
        other.join();
        if (mine) std::rethrow_exception(mine);
        if (err) std::rethrow_exception(err);
    }
    post_shared(shared, node_count, lower, upper, o, node_results);
    post_batch(probs, count, o, results);
    if (o.verbose > 0)
        std::fprintf(stderr, "[vikalp_b200] together: total incl. release   %8.3f s\n", seconds_since(t0));
}

} // namespace vk
