// Adjoint of solved LPs: gradients of L = g'x* + w_obj * c'x* with respect to
// c, the row bounds and the stored values of A, for many LPs at once.
//
// At an optimum with active rows R (equality rows and rows at a bound) and free
// columns F (strictly inside their bounds), x_F solves A_RF x_F = b_R - A_RN x_N
// and c_F + A_RF' y_R = 0 (y in the reference's sign convention,
// SolveResult.hpp:31-33). The adjoint of that active-set KKT system is the
// least-squares problem
//     w = argmin |A_RF' w - g_F|   (minimum norm),
// after which
//     dL/dc   = w_obj x                    (x* is locally constant in c)
//     dL/db_i = w_i - w_obj y_i            (b_i: the active bound of row i)
//     dL/dA_ij = (-w_i + w_obj y_i) x_j    (every stored entry)
// (the w_obj terms are the envelope theorem for the optimal objective).
//
// The least-squares problem is solved by LSQR (Paige & Saunders, 1982) on the
// masked operator M = A_RF' of every instance, all instances at once on the
// block-diagonal layout: M v is a pass over A' (gathers v, masks the output by
// F), M'u a pass over A (gathers u, masks by R) -- the same fused sparse-pass
// kernels as the solver, with the LSQR vector updates in their epilogues and
// per-tile partial sums reduced per instance in a fixed order. The scalar
// recurrences run on the device, one thread per instance; a chunk of
// iterations is one CUDA graph.
#include "vk_blockdiag.cuh"
#include "vk_engine.cuh"

#include <algorithm>
#include <cmath>
#include <limits>

namespace vk {
namespace {

constexpr int kAdjChunk = 16; // LSQR iterations per graph launch

// Per-instance LSQR state (device arrays).
struct LsqrCtl {
    double *alpha, *beta, *phibar, *rhobar, *beta1, *anorm2, *t1, *t2, *rnorm, *arnorm;
    long long *iters;
    int *stop, *done, *status;
    const int *tbeg_a, *tbeg_at; // first tile of every instance (A, A')
    const double *pa, *pat;      // per-tile partial sums of |v|^2 (A pass) / |u|^2 (A' pass)
    double tol;
    long long limit;
    int count;
};

template <class T>
struct StoreEpi : EpiRow<T, StoreEpi<T>> {
    T *y;
    __device__ void row(int i, const T (&s)[1], double (&)[1]) const { y[i] = s[0]; }
};

// Active rows: a finite bound within tol * (1 + |bound|) of A x.
__global__ void active_rows_kernel(const double *__restrict__ ax, const double *__restrict__ rl,
                                   const double *__restrict__ ru, int m, double tol, double *__restrict__ rmask) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const double a = ax[i], lo = rl[i], hi = ru[i];
    const bool at_lo = isfinite(lo) && fabs(a - lo) <= tol * (1.0 + fabs(lo));
    const bool at_hi = isfinite(hi) && fabs(a - hi) <= tol * (1.0 + fabs(hi));
    rmask[i] = (at_lo || at_hi) ? 1.0 : 0.0;
}

// Free columns: strictly inside both bounds by more than tol * (1 + |bound|);
// u = F g (the right-hand side), v = w = 0.
__global__ void free_cols_kernel(const double *__restrict__ x, const double *__restrict__ l,
                                 const double *__restrict__ u, const double *__restrict__ g, int n, double tol,
                                 double *__restrict__ fmask, double *__restrict__ ubar) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double v = x[j], lo = l[j], hi = u[j];
    const bool at_lo = isfinite(lo) && v - lo <= tol * (1.0 + fabs(lo));
    const bool at_hi = isfinite(hi) && hi - v <= tol * (1.0 + fabs(hi));
    const double f = (at_lo || at_hi) ? 0.0 : 1.0;
    fmask[j] = f;
    ubar[j] = f * g[j];
}

// |u|^2 of every instance over its columns (one warp per instance, fixed order).
__global__ void segment_norm2_kernel(const double *__restrict__ a, const int *__restrict__ off, int count,
                                     double *__restrict__ out) {
    const int b = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= count) return;
    double s = 0.0;
    for (int i = off[b] + lane; i < off[b + 1]; i += 32) s += a[i] * a[i];
    s = warp_sum(s);
    if (lane == 0) out[b] = s;
}

__device__ double tile_sum(const double *p, int t0, int t1) {
    double s = 0.0;
    for (int t = t0; t < t1; ++t) s += p[t];
    return s;
}

// Start: beta_1 = |F g|; alpha = 1 and v = 0 so the first A pass gives
// v = M'u / beta_1 exactly; an instance with g_F = 0 has w = 0.
__global__ void lsqr_start_kernel(LsqrCtl c, const double *nrm2) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= c.count) return;
    const double beta = sqrt(nrm2[b]);
    c.beta[b] = beta;
    c.beta1[b] = beta;
    c.alpha[b] = 1.0;
    c.anorm2[b] = 0.0;
    c.iters[b] = 0;
    c.rnorm[b] = beta;
    c.arnorm[b] = 0.0;
    c.stop[b] = beta > 0.0 ? 0 : 1;
    c.done[b] = beta > 0.0 ? 0 : 1;
    c.status[b] = beta > 0.0 ? VK_STATUS_NOT_SOLVED : VK_STATUS_OPTIMAL;
}

// The first alpha: alpha_1 = |M'u_1|; phibar = beta_1, rhobar = alpha_1,
// and the search direction starts at v_1 (t1 = 0, t2 = 0 in the update kernel).
__global__ void lsqr_first_alpha_kernel(LsqrCtl c) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= c.count || c.done[b]) return;
    const double alpha = sqrt(tile_sum(c.pa, c.tbeg_a[b], c.tbeg_a[b + 1]));
    c.alpha[b] = alpha;
    c.phibar[b] = c.beta[b];
    c.rhobar[b] = alpha;
    c.anorm2[b] = alpha * alpha;
    c.t1[b] = 0.0;
    c.t2[b] = 0.0;
    c.arnorm[b] = alpha * c.beta[b];
    if (!(alpha > 0.0)) { // g_F orthogonal to the range of M: w = 0 is the answer
        c.stop[b] = 1;
        c.status[b] = VK_STATUS_OPTIMAL;
    }
}

// A' pass (rows = columns j, gathers vbar): u <- F (M v) - alpha u with
// v = vbar / alpha, u = ubar / beta (previous norms). Sums |u|^2 per tile.
struct AdjColEpi : EpiBase<double> {
    static constexpr int NR = 1;
    static constexpr bool kPerTile = true;
    LsqrCtl c;
    const int *inst, *tile_inst;
    const double *fmask;
    double *ubar, *partials;
    struct Pre {
        double f, u;
        int b;
    };
    static constexpr bool kSkipTiles = true;
    __device__ bool skip_tile(int t) const { return c.done[tile_inst[t]] != 0; }
    __device__ Pre load(int j) const { return Pre{fmask[j], ubar[j], inst[j]}; }
    __device__ void row_pre(int j, const double (&s)[1], const Pre &p, double (&red)[1]) const {
        const double alpha = c.alpha[p.b], beta = c.beta[p.b];
        const double u = alpha > 0.0 ? p.f * (s[0] / alpha) - alpha * (p.u / beta) : 0.0;
        ubar[j] = u;
        red[0] += u * u;
    }
    template <int R>
    __device__ void tile_done(int t, double (&red)[R]) const {
        partials[t] = red[0];
    }
};

// beta <- |u|; a finished instance (stop set by the previous alpha step) is
// marked done here, after its last search-direction update.
__global__ void lsqr_beta_kernel(LsqrCtl c) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= c.count || c.done[b]) return;
    if (c.stop[b]) {
        c.done[b] = 1;
        return;
    }
    c.beta[b] = sqrt(tile_sum(c.pat, c.tbeg_at[b], c.tbeg_at[b + 1]));
}

// A pass (rows i, gathers ubar): v <- R (M'u) - beta v with u = ubar / beta
// (new norm) and v = vbar / alpha (previous norm). Sums |v|^2 per tile.
struct AdjRowEpi : EpiBase<double> {
    static constexpr int NR = 1;
    static constexpr bool kPerTile = true;
    LsqrCtl c;
    const int *inst, *tile_inst;
    const double *rmask;
    double *vbar, *partials;
    struct Pre {
        double r, v;
        int b;
    };
    static constexpr bool kSkipTiles = true;
    __device__ bool skip_tile(int t) const { return c.done[tile_inst[t]] != 0; }
    __device__ Pre load(int i) const { return Pre{rmask[i], vbar[i], inst[i]}; }
    __device__ void row_pre(int i, const double (&s)[1], const Pre &p, double (&red)[1]) const {
        const double alpha = c.alpha[p.b], beta = c.beta[p.b];
        // beta = 0: the residual vanished; this step only finishes the update
        const double v = beta > 0.0 ? p.r * (s[0] / beta) - beta * (p.v / alpha) : 0.0;
        vbar[i] = v;
        red[0] += v * v;
    }
    template <int R>
    __device__ void tile_done(int t, double (&red)[R]) const {
        partials[t] = red[0];
    }
};

// alpha <- |v|, then the plane rotation of LSQR and its stopping tests:
// |r| <= tol |g_F| (consistent system) or |M'r| <= tol |M|_F |r| (least squares).
__global__ void lsqr_alpha_kernel(LsqrCtl c) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= c.count || c.done[b] || c.stop[b]) return;
    const double alpha = sqrt(tile_sum(c.pa, c.tbeg_a[b], c.tbeg_a[b + 1]));
    const double beta = c.beta[b];
    const double rhobar = c.rhobar[b], phibar = c.phibar[b];
    const double rho = hypot(rhobar, beta);
    const double cs = rhobar / rho, sn = beta / rho;
    const double theta = sn * alpha;
    c.rhobar[b] = -cs * alpha;
    const double phi = cs * phibar;
    c.phibar[b] = sn * phibar;
    c.t1[b] = phi / rho;
    c.t2[b] = theta / rho;
    c.alpha[b] = alpha;
    c.anorm2[b] += alpha * alpha + beta * beta;
    const long long it = ++c.iters[b];
    const double rnorm = sn * phibar;
    const double arnorm = rnorm * alpha * fabs(cs);
    c.rnorm[b] = rnorm;
    c.arnorm[b] = arnorm;
    const bool ok1 = rnorm <= c.tol * c.beta1[b];
    const bool ok2 = arnorm <= c.tol * sqrt(c.anorm2[b]) * rnorm;
    if (ok1 || ok2 || !(alpha > 0.0)) {
        c.stop[b] = 1;
        c.status[b] = VK_STATUS_OPTIMAL;
    } else if (it >= c.limit) {
        c.stop[b] = 1;
        c.status[b] = VK_STATUS_ITERATION_LIMIT;
    }
}

// w <- w + t1 d;  d <- v - t2 d  (v = vbar / alpha), rows of active instances.
__global__ void lsqr_update_kernel(LsqrCtl c, const int *__restrict__ inst, const double *__restrict__ vbar,
                                   double *__restrict__ w, double *__restrict__ d, int m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int b = inst[i];
    if (c.done[b]) return;
    const double di = d[i];
    w[i] += c.t1[b] * di;
    const double a = c.alpha[b];
    d[i] = (a > 0.0 ? vbar[i] / a : 0.0) - c.t2[b] * di;
}

// dL/dA_k = (-w_i + w_obj y_i) x_{col k} for the stored entries of row i;
// dL/db_i = w_i - w_obj y_i. One warp per row.
__global__ void adjoint_a_kernel(const int *__restrict__ ro, const int *__restrict__ ci,
                                 const double *__restrict__ w, const double *__restrict__ y,
                                 const double *__restrict__ x, double w_obj, int m, double *__restrict__ da,
                                 double *__restrict__ db) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= m) return;
    const double f = -w[i] + w_obj * y[i];
    for (int k = ro[i] + lane; k < ro[i + 1]; k += 32) da[k] = f * x[ci[k]];
    if (lane == 0) db[i] = w[i] - w_obj * y[i];
}

class AdjointEngine {
public:
    AdjointEngine(const vk_problem *probs, int count, const vk_adjoint_options &o) : o_(o), B_(count) {
        VK_CUDA(cudaSetDevice(o.device));
        device_error_flag();
        VK_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
        concat_instances(probs, count, h_);
        upload_block_diag(h_, d_, s_, false);
    }
    ~AdjointEngine() {
        if (g_) cudaGraphExecDestroy(g_);
        if (s_) cudaStreamDestroy(s_);
    }

    void run(const double *x, const double *y, const double *g, double w_obj, double *dc, double *db, double *da,
             vk_adjoint_info *info) {
        const int m = h_.m, n = h_.n, B = B_;
        const int mm = std::max(m, 1);
        DevBuf<double> dx(n), dy(mm), dg(n), l(n), u(n), rl(mm), ru(mm);
        auto up = [&](DevBuf<double> &d, const double *h, int k) {
            if (k > 0) VK_CUDA(cudaMemcpyAsync(d.get(), h, k * sizeof(double), cudaMemcpyHostToDevice, s_));
        };
        up(dx, x, n);
        up(dy, y, m);
        up(dg, g, n);
        up(l, h_.vl.data(), n);
        up(u, h_.vu.data(), n);
        up(rl, h_.rl.data(), m);
        up(ru, h_.ru.data(), m);
        // active set
        rmask_.reset(mm);
        fmask_.reset(n);
        ubar_.reset(n);
        vbar_.reset(mm);
        w_.reset(mm);
        dir_.reset(mm);
        for (DevBuf<double> *b : {&vbar_, &w_, &dir_}) VK_CUDA(cudaMemsetAsync(b->get(), 0, b->bytes(), s_));
        if (m > 0) {
            DevBuf<double> ax(m);
            StoreEpi<double> e;
            e.y = ax.get();
            launch_tiles<double, double, 1, false>(view(d_.a, d_.a_val.get()), Gathers<double, 1>{{dx.get()}}, e, s_);
            active_rows_kernel<<<grid1d(m), 256, 0, s_>>>(ax.get(), rl.get(), ru.get(), m, o_.active_tolerance,
                                                         rmask_.get());
            VK_CUDA(cudaStreamSynchronize(s_));
        }
        free_cols_kernel<<<grid1d(n), 256, 0, s_>>>(dx.get(), l.get(), u.get(), dg.get(), n, o_.active_tolerance,
                                                    fmask_.get(), ubar_.get());
        VK_LAUNCH_CHECK();
        // LSQR control
        for (DevBuf<double> *b : {&alpha_, &beta_, &phibar_, &rhobar_, &beta1_, &anorm2_, &t1_, &t2_, &rnorm_,
                                  &arnorm_, &nrm2_})
            b->reset(B);
        iters_.reset(B);
        for (DevBuf<int> *b : {&stop_, &done_, &status_}) b->reset(B);
        pa_.reset(std::max(d_.a.ntiles, 1));
        pat_.reset(std::max(d_.at.ntiles, 1));
        VK_CUDA(cudaMemsetAsync(pa_.get(), 0, pa_.bytes(), s_));
        VK_CUDA(cudaMemsetAsync(pat_.get(), 0, pat_.bytes(), s_));
        DevBuf<int> coff;
        coff.reset(B + 1);
        VK_CUDA(cudaMemcpyAsync(coff.get(), h_.col_off.data(), (B + 1) * sizeof(int), cudaMemcpyHostToDevice, s_));
        segment_norm2_kernel<<<ceil_div(int64_t(B) * 32, 256), 256, 0, s_>>>(ubar_.get(), coff.get(), B,
                                                                            nrm2_.get());
        const LsqrCtl c = ctl();
        lsqr_start_kernel<<<ceil_div(B, 128), 128, 0, s_>>>(c, nrm2_.get());
        VK_LAUNCH_CHECK();
        // v_1 = M'u_1 / beta_1, alpha_1 = |v_1|, d_1 = v_1
        if (m > 0) {
            row_pass(c);
            lsqr_first_alpha_kernel<<<ceil_div(B, 128), 128, 0, s_>>>(c);
            lsqr_update_kernel<<<grid1d(m), 256, 0, s_>>>(c, d_.rinst.get(), vbar_.get(), w_.get(), dir_.get(), m);
            VK_LAUNCH_CHECK();
        }
        // iterations, a chunk per graph launch
        if (m > 0) {
            if (g_) cudaGraphExecDestroy(g_);
            g_ = capture(c);
            std::vector<int> hstop(B);
            for (;;) {
                VK_CUDA(cudaGraphLaunch(g_, s_));
                VK_CUDA(cudaMemcpyAsync(hstop.data(), stop_.get(), B * sizeof(int), cudaMemcpyDeviceToHost, s_));
                VK_CUDA(cudaStreamSynchronize(s_));
                check_device_error(s_);
                if (std::all_of(hstop.begin(), hstop.end(), [](int v) { return v != 0; })) break;
            }
        }
        // gradients
        DevBuf<double> dA(std::max<int64_t>(h_.nnz, 1)), dB(mm);
        if (m > 0) {
            adjoint_a_kernel<<<ceil_div(int64_t(m) * 32, 256), 256, 0, s_>>>(
                d_.a.ro.get(), d_.a.ci.get(), w_.get(), dy.get(), dx.get(), w_obj, m, dA.get(), dB.get());
            VK_LAUNCH_CHECK();
        }
        if (da && h_.nnz > 0)
            VK_CUDA(cudaMemcpyAsync(da, dA.get(), h_.nnz * sizeof(double), cudaMemcpyDeviceToHost, s_));
        if (db && m > 0) VK_CUDA(cudaMemcpyAsync(db, dB.get(), m * sizeof(double), cudaMemcpyDeviceToHost, s_));
        std::vector<double> hr(m), hf(n), hrn(B), hb1(B), har(B), han(B);
        std::vector<long long> hit(B);
        std::vector<int> hst(B);
        if (m > 0) VK_CUDA(cudaMemcpyAsync(hr.data(), rmask_.get(), m * sizeof(double), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(hf.data(), fmask_.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(hrn.data(), rnorm_.get(), B * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(hb1.data(), beta1_.get(), B * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(har.data(), arnorm_.get(), B * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(han.data(), anorm2_.get(), B * 8, cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(hit.data(), iters_.get(), B * sizeof(long long), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaMemcpyAsync(hst.data(), status_.get(), B * sizeof(int), cudaMemcpyDeviceToHost, s_));
        VK_CUDA(cudaStreamSynchronize(s_));
        if (dc)
            for (int j = 0; j < n; ++j) dc[j] = w_obj * x[j];
        if (info) {
            for (int b = 0; b < B; ++b) {
                vk_adjoint_info &f = info[b];
                f.rows_active = 0;
                f.cols_free = 0;
                for (int i = h_.row_off[b]; i < h_.row_off[b + 1]; ++i) f.rows_active += hr[i] != 0.0;
                for (int j = h_.col_off[b]; j < h_.col_off[b + 1]; ++j) f.cols_free += hf[j] != 0.0;
                f.iterations = hit[b];
                f.status = m > 0 ? hst[b] : VK_STATUS_OPTIMAL;
                f.residual = hb1[b] > 0.0 ? hrn[b] / hb1[b] : 0.0;
                f.normal_residual = (han[b] > 0.0 && hrn[b] > 0.0) ? har[b] / (std::sqrt(han[b]) * hrn[b]) : 0.0;
            }
        }
    }

private:
    LsqrCtl ctl() {
        LsqrCtl c{};
        c.alpha = alpha_.get();
        c.beta = beta_.get();
        c.phibar = phibar_.get();
        c.rhobar = rhobar_.get();
        c.beta1 = beta1_.get();
        c.anorm2 = anorm2_.get();
        c.t1 = t1_.get();
        c.t2 = t2_.get();
        c.rnorm = rnorm_.get();
        c.arnorm = arnorm_.get();
        c.iters = iters_.get();
        c.stop = stop_.get();
        c.done = done_.get();
        c.status = status_.get();
        c.tbeg_a = d_.tbeg_a.get();
        c.tbeg_at = d_.tbeg_at.get();
        c.pa = pa_.get();
        c.pat = pat_.get();
        c.tol = o_.solve_tolerance;
        c.limit = o_.iteration_limit;
        c.count = B_;
        return c;
    }

    void row_pass(const LsqrCtl &c) {
        AdjRowEpi e;
        e.c = c;
        e.inst = d_.rinst.get();
        e.tile_inst = d_.tinst_a.get();
        e.rmask = rmask_.get();
        e.vbar = vbar_.get();
        e.partials = pa_.get();
        launch_tiles<double, double, 1, false>(view(d_.a, d_.a_val.get()), Gathers<double, 1>{{ubar_.get()}}, e, s_);
    }

    void col_pass(const LsqrCtl &c) {
        AdjColEpi e;
        e.c = c;
        e.inst = d_.cinst.get();
        e.tile_inst = d_.tinst_at.get();
        e.fmask = fmask_.get();
        e.ubar = ubar_.get();
        e.partials = pat_.get();
        launch_tiles<double, double, 1, false>(view(d_.at, d_.at_val.get()), Gathers<double, 1>{{vbar_.get()}}, e, s_);
    }

    cudaGraphExec_t capture(const LsqrCtl &c) {
        const int m = h_.m;
        VK_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
        for (int it = 0; it < kAdjChunk; ++it) {
            col_pass(c);
            lsqr_beta_kernel<<<ceil_div(B_, 128), 128, 0, s_>>>(c);
            row_pass(c);
            lsqr_alpha_kernel<<<ceil_div(B_, 128), 128, 0, s_>>>(c);
            lsqr_update_kernel<<<grid1d(m), 256, 0, s_>>>(c, d_.rinst.get(), vbar_.get(), w_.get(), dir_.get(), m);
            VK_LAUNCH_CHECK();
        }
        cudaGraph_t g;
        VK_CUDA(cudaStreamEndCapture(s_, &g));
        cudaGraphExec_t ex;
        VK_CUDA(cudaGraphInstantiate(&ex, g, 0));
        cudaGraphDestroy(g);
        return ex;
    }

    vk_adjoint_options o_;
    int B_;
    cudaStream_t s_ = nullptr;
    BlockDiag h_;
    DeviceBlockDiag d_;
    DevBuf<double> rmask_, fmask_, ubar_, vbar_, w_, dir_;
    DevBuf<double> alpha_, beta_, phibar_, rhobar_, beta1_, anorm2_, t1_, t2_, rnorm_, arnorm_, nrm2_, pa_, pat_;
    DevBuf<long long> iters_;
    DevBuf<int> stop_, done_, status_;
    cudaGraphExec_t g_ = nullptr;
};

} // namespace

void lp_adjoint(const vk_problem *probs, int count, const double *x, const double *y, const double *g, double w_obj,
                const vk_adjoint_options &o, double *dc, double *db, double *da, vk_adjoint_info *info) {
    if (count <= 0) throw InvalidInput("count must be positive");
    if (!(o.active_tolerance >= 0.0) || !(o.solve_tolerance > 0.0) || o.iteration_limit <= 0)
        throw InvalidInput("adjoint tolerances and iteration limit must be positive");
    vk_options vo;
    vk_default_options(&vo);
    int64_t m = 0, n = 0, nnz = 0;
    for (int b = 0; b < count; ++b) {
        bool unsupported = false;
        const std::string msg = validate_problem(probs[b], vo, unsupported);
        if (!msg.empty()) {
            const std::string full = "instance " + std::to_string(b) + ": " + msg;
            if (unsupported) throw Unsupported(full);
            throw InvalidInput(full);
        }
        if (probs[b].Q.rows > 0 && probs[b].Q.row_offsets && probs[b].Q.row_offsets[probs[b].Q.rows] > 0)
            throw Unsupported("instance " + std::to_string(b) + ": the adjoint takes LPs");
        m += probs[b].A.rows;
        n += probs[b].A.cols;
        nnz += probs[b].A.rows > 0 ? probs[b].A.row_offsets[probs[b].A.rows] : 0;
    }
    if (m >= (int64_t(1) << 31) || n >= (int64_t(1) << 31) || nnz >= (int64_t(1) << 31))
        throw Unsupported("the batch exceeds the int32 index range of the device structures");
    for (int64_t j = 0; j < n; ++j)
        if (!std::isfinite(x[j]) || !std::isfinite(g[j])) throw InvalidInput("x and dL_dx must be finite");
    for (int64_t i = 0; i < m; ++i)
        if (!std::isfinite(y[i])) throw InvalidInput("y must be finite");
    if (!std::isfinite(w_obj)) throw InvalidInput("dL_dobj must be finite");
    AdjointEngine eng(probs, count, o);
    eng.run(x, y, g, w_obj, dc, db, da, info);
}

} // namespace vk
