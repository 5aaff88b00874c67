// extern "C" entry points of include/vikalp_b200.h. Every call catches and
// maps exceptions to status codes; the message is kept per thread.
#include "vk_engine.cuh"
#include "vk_stage.cuh"
#include "vk_vec.cuh"

#include <cstring>
#include <memory>
#include <string>

namespace {

thread_local std::string g_last_error;

int set_error(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

template <class F>
int guarded(F &&f) {
    try {
        return f();
    } catch (const vk::CudaFailure &e) {
        return set_error(VK_ERR_CUDA, e.what());
    } catch (const vk::InvalidInput &e) {
        return set_error(VK_ERR_INVALID, e.what());
    } catch (const vk::Unsupported &e) {
        return set_error(VK_ERR_UNSUPPORTED, e.what());
    } catch (const std::bad_alloc &) {
        return set_error(VK_ERR_INTERNAL, "out of host memory");
    } catch (const std::exception &e) {
        return set_error(VK_ERR_INTERNAL, e.what());
    } catch (...) {
        return set_error(VK_ERR_INTERNAL, "unknown failure");
    }
}

// CsrPattern checks of the reference backends (cpu_ops.cpp:38-63,
// cuda_ops.cu:48-76): offsets start at 0 and ascend, columns in range and
// strictly increasing per row.
void check_csr(const vk_csr *a) {
    if (!a) throw vk::InvalidInput("matrix is null");
    if (a->rows < 0 || a->cols < 0) throw vk::InvalidInput("matrix dimensions must be non-negative");
    if (a->rows >= (int64_t(1) << 31) || a->cols >= (int64_t(1) << 31))
        throw vk::Unsupported("matrix exceeds the int32 index range of the device structures");
    const int64_t *ro = a->row_offsets;
    if (!ro) throw vk::InvalidInput("CsrPattern row_offsets size != rows+1");
    if (ro[0] != 0) throw vk::InvalidInput("CsrPattern row_offsets do not describe column_indices");
    const int64_t nnz = ro[a->rows];
    if (nnz >= (int64_t(1) << 31)) throw vk::Unsupported("matrix exceeds the int32 index range");
    for (int64_t r = 0; r < a->rows; ++r) {
        const int64_t b = ro[r], e = ro[r + 1];
        if (b < 0 || b > e || e > nnz) throw vk::InvalidInput("CsrPattern row_offsets must be ordered and in range");
        int64_t prev = -1;
        for (int64_t k = b; k < e; ++k) {
            const int64_t c = a->col_indices[k];
            if (c < 0 || c >= a->cols || c <= prev)
                throw vk::InvalidInput("CsrPattern columns must be ordered and in range");
            prev = c;
        }
    }
}

template <class T>
struct PlainEpi : vk::EpiRow<T, PlainEpi<T>> {
    T *y;
    __device__ void row(int i, const T (&s)[1], double (&)[1]) const { y[i] = s[0]; }
};

// y = alpha * acc + beta * y (cpu_ops.cpp:426)
struct AxpbyEpi : vk::EpiRow<double, AxpbyEpi> {
    double alpha, beta;
    double *y;
    __device__ void row(int i, const double (&s)[1], double (&)[1]) const {
        y[i] = __dadd_rn(__dmul_rn(alpha, s[0]), __dmul_rn(beta, y[i]));
    }
};

// y *= beta, then y[col] += v * (alpha * x[row]) in row order (cpu_ops.cpp:444-458)
struct ScatterEpi : vk::EpiRow<double, ScatterEpi> {
    double alpha, beta;
    double *y;
    __device__ double init(int j, int) const { return __dmul_rn(beta, y[j]); }
    __device__ double gscale(int) const { return alpha; }
    __device__ void row(int j, const double (&s)[1], double (&)[1]) const { y[j] = s[0]; }
};

struct Stream {
    cudaStream_t s = nullptr;
    Stream() { VK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~Stream() {
        if (s) cudaStreamDestroy(s);
    }
};

} // namespace

namespace vk {
// Records `msg` as the calling thread's last error and returns `code`.
int record_error(int code, const std::string &msg) { return set_error(code, msg); }
} // namespace vk

struct vk_pdhg {
    std::unique_ptr<vk::Solver> solver;
};

struct vk_spmat {
    int precision = VK_PREC_FP64;
    vk::CsrPattern32 a, at;
    vk::DevBuf<int> perm;
    vk::DevBuf<double> v64, vt64;
    vk::DevBuf<float> v32, vt32;
};

extern "C" {

void vk_default_options(vk_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->iteration_limit = 100000;
    o->time_limit_seconds = __builtin_inf();
    o->primal_tolerance = 1e-7;
    o->dual_tolerance = 1e-7;
    o->continuous_method = 0;
    o->algorithm = VK_ALGO_REFERENCE;
    o->precision = VK_PREC_FP64;
    o->spmv_order = VK_SPMV_FAST;
    o->check_every = 64;
    o->relative_tolerance = 1e-6;
    o->device = 0;
    o->verbose = 0;
}

const char *vk_last_error(void) { return g_last_error.c_str(); }

const char *vk_version(void) { return "vikalp_b200 0.1 (sm_100a)"; }

int vk_pdhg_create(const vk_problem *problem, const vk_options *opts, vk_pdhg **out) {
    return guarded([&] {
        if (!problem || !out) return set_error(VK_ERR_INVALID, "null argument");
        *out = nullptr;
        vk_options o;
        if (opts)
            o = *opts;
        else
            vk_default_options(&o);
        bool unsupported = false;
        const auto t0 = std::chrono::steady_clock::now();
        const std::string msg = vk::validate_problem(*problem, o, unsupported);
        if (!msg.empty()) return set_error(unsupported ? VK_ERR_UNSUPPORTED : VK_ERR_INVALID, msg);
        if (o.verbose > 0)
            std::fprintf(stderr, "[vikalp_b200] create: %-28s %8.3f s\n", "validation (host)",
                         std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
        auto h = std::make_unique<vk_pdhg>();
        h->solver = std::make_unique<vk::Solver>(*problem, o);
        *out = h.release();
        return VK_OK;
    });
}

int vk_pdhg_solve(vk_pdhg *h, const double *warm, const double *lo, const double *hi, vk_result *result) {
    return guarded([&] {
        if (!h || !result) return set_error(VK_ERR_INVALID, "null argument");
        h->solver->solve(warm, lo, hi, result);
        return VK_OK;
    });
}

int vk_pdhg_set_options(vk_pdhg *h, const vk_options *opts) {
    return guarded([&] {
        if (!h || !opts) return set_error(VK_ERR_INVALID, "null argument");
        const std::string msg = h->solver->set_options(*opts);
        if (!msg.empty()) return set_error(VK_ERR_INVALID, msg);
        return VK_OK;
    });
}

int vk_pdhg_profile(vk_pdhg *h, int64_t iterations, vk_pass_profile *out) {
    return guarded([&] {
        if (!h || !out) return set_error(VK_ERR_INVALID, "null argument");
        if (iterations < 1 || iterations > 100000) return set_error(VK_ERR_INVALID, "iterations must be in [1, 100000]");
        if (!h->solver->profile(iterations, out))
            return set_error(VK_ERR_UNSUPPORTED, "this scheme has no profiling path (VK_ALGO_REFERENCE has)");
        return VK_OK;
    });
}

void vk_pdhg_destroy(vk_pdhg *h) {
    try {
        delete h;
    } catch (...) {
    }
}

int vk_csr_transpose(const vk_csr *a, int64_t *t_row_offsets, int64_t *t_col_indices, double *t_values,
                     int64_t *perm) {
    return guarded([&] {
        check_csr(a);
        Stream st;
        vk::CsrPattern32 p, pt;
        vk::DevBuf<int> pm;
        static const int64_t zero = 0;
        vk::upload_pattern(a->rows, a->cols, a->rows > 0 ? a->row_offsets : &zero, a->col_indices, p, st.s);
        vk::transpose_pattern(p, pt, pm, st.s);
        const int64_t nnz = p.nnz;
        std::vector<int> tro(a->cols + 1), tci(nnz), tp(nnz);
        VK_CUDA(cudaMemcpyAsync(tro.data(), pt.ro.get(), (a->cols + 1) * sizeof(int), cudaMemcpyDeviceToHost, st.s));
        if (nnz > 0) {
            VK_CUDA(cudaMemcpyAsync(tci.data(), pt.ci.get(), nnz * sizeof(int), cudaMemcpyDeviceToHost, st.s));
            VK_CUDA(cudaMemcpyAsync(tp.data(), pm.get(), nnz * sizeof(int), cudaMemcpyDeviceToHost, st.s));
        }
        vk::DevBuf<double> v(nnz > 0 ? nnz : 1), tv(nnz > 0 ? nnz : 1);
        if (t_values && nnz > 0) {
            VK_CUDA(cudaMemcpyAsync(v.get(), a->values, nnz * sizeof(double), cudaMemcpyHostToDevice, st.s));
            vk::gather_values<double, double>(pm.get(), v.get(), tv.get(), nnz, st.s);
            VK_CUDA(cudaMemcpyAsync(t_values, tv.get(), nnz * sizeof(double), cudaMemcpyDeviceToHost, st.s));
        }
        VK_CUDA(cudaStreamSynchronize(st.s));
        for (int64_t j = 0; j <= a->cols; ++j) t_row_offsets[j] = tro[j];
        for (int64_t t = 0; t < nnz; ++t) t_col_indices[t] = tci[t];
        if (perm)
            for (int64_t t = 0; t < nnz; ++t) perm[t] = tp[t];
        return VK_OK;
    });
}

int vk_spmv(const vk_csr *a, double alpha, const double *x, double beta, double *y, int transpose,
            int spmv_order) {
    return guarded([&] {
        check_csr(a);
        Stream st;
        vk::CsrPattern32 p;
        static const int64_t zero = 0;
        vk::upload_pattern(a->rows, a->cols, a->rows > 0 ? a->row_offsets : &zero, a->col_indices, p, st.s);
        const int64_t nnz = p.nnz;
        const int64_t xl = transpose ? a->rows : a->cols, yl = transpose ? a->cols : a->rows;
        vk::DevBuf<double> v(vk::padded(nnz)), dx(xl > 0 ? xl : 1), dy(yl > 0 ? yl : 1);
        if (nnz > 0) VK_CUDA(cudaMemcpyAsync(v.get(), a->values, nnz * sizeof(double), cudaMemcpyHostToDevice, st.s));
        if (xl > 0) VK_CUDA(cudaMemcpyAsync(dx.get(), x, xl * sizeof(double), cudaMemcpyHostToDevice, st.s));
        if (yl > 0) VK_CUDA(cudaMemcpyAsync(dy.get(), y, yl * sizeof(double), cudaMemcpyHostToDevice, st.s));
        const bool exact = spmv_order == VK_SPMV_SEQUENTIAL;
        if (!transpose) {
            AxpbyEpi e;
            e.alpha = alpha;
            e.beta = beta;
            e.y = dy.get();
            auto M = vk::view(p, v.get());
            if (exact)
                vk::launch_tiles<double, double, 1, true>(M, vk::Gathers<double, 1>{{dx.get()}}, e, st.s);
            else
                vk::launch_tiles<double, double, 1, false>(M, vk::Gathers<double, 1>{{dx.get()}}, e, st.s);
        } else {
            vk::CsrPattern32 pt;
            vk::DevBuf<int> pm;
            vk::transpose_pattern(p, pt, pm, st.s);
            vk::DevBuf<double> tv(vk::padded(nnz));
            vk::gather_values<double, double>(pm.get(), v.get(), tv.get(), nnz, st.s);
            ScatterEpi e;
            e.alpha = alpha;
            e.beta = beta;
            e.y = dy.get();
            auto M = vk::view(pt, tv.get());
            if (exact)
                vk::launch_tiles<double, double, 1, true>(M, vk::Gathers<double, 1>{{dx.get()}}, e, st.s);
            else
                vk::launch_tiles<double, double, 1, false>(M, vk::Gathers<double, 1>{{dx.get()}}, e, st.s);
        }
        if (yl > 0) VK_CUDA(cudaMemcpyAsync(y, dy.get(), yl * sizeof(double), cudaMemcpyDeviceToHost, st.s));
        VK_CUDA(cudaStreamSynchronize(st.s));
        vk::check_device_error(st.s);
        return VK_OK;
    });
}

int vk_spmat_create(const vk_csr *a, int32_t precision, vk_spmat **out) {
    return guarded([&] {
        if (!out) return set_error(VK_ERR_INVALID, "null argument");
        *out = nullptr;
        check_csr(a);
        if (precision != VK_PREC_FP64 && precision != VK_PREC_MIXED) return set_error(VK_ERR_INVALID, "unknown precision");
        Stream st;
        auto h = std::make_unique<vk_spmat>();
        h->precision = precision;
        static const int64_t zero = 0;
        vk::upload_pattern(a->rows, a->cols, a->rows > 0 ? a->row_offsets : &zero, a->col_indices, h->a, st.s);
        const int64_t nnz = h->a.nnz;
        vk::transpose_pattern(h->a, h->at, h->perm, st.s);
        vk::DevBuf<double> v(vk::padded(nnz));
        vk::stage_h2d(v.get(), a->values, nnz * sizeof(double), st.s);
        if (precision == VK_PREC_FP64) {
            h->vt64.reset(vk::padded(nnz));
            vk::gather_values<double, double>(h->perm.get(), v.get(), h->vt64.get(), nnz, st.s);
            h->v64 = std::move(v);
        } else {
            h->v32.reset(vk::padded(nnz));
            h->vt32.reset(vk::padded(nnz));
            vk::convert_values<float, double>(v.get(), h->v32.get(), nnz, st.s);
            vk::gather_values<float, double>(h->perm.get(), v.get(), h->vt32.get(), nnz, st.s);
        }
        if (precision == VK_PREC_FP64) {
            vk::autotune_pattern<double>(h->a, h->v64.get(), st.s);
            vk::autotune_pattern<double>(h->at, h->vt64.get(), st.s);
        } else {
            vk::autotune_pattern<float>(h->a, h->v32.get(), st.s);
            vk::autotune_pattern<float>(h->at, h->vt32.get(), st.s);
        }
        VK_CUDA(cudaStreamSynchronize(st.s));
        *out = h.release();
        return VK_OK;
    });
}

int vk_spmat_apply_device(vk_spmat *m, const void *x, void *y, int transpose, void *stream) {
    return guarded([&] {
        if (!m || !x || !y) return set_error(VK_ERR_INVALID, "null argument");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const vk::CsrPattern32 &p = transpose ? m->at : m->a;
        if (m->precision == VK_PREC_FP64) {
            PlainEpi<double> e;
            e.y = static_cast<double *>(y);
            vk::launch_tiles<double, double, 1, false>(vk::view(p, transpose ? m->vt64.get() : m->v64.get()),
                                                       vk::Gathers<double, 1>{{static_cast<const double *>(x)}}, e, s);
        } else {
            PlainEpi<float> e;
            e.y = static_cast<float *>(y);
            vk::launch_tiles<float, float, 1, false>(vk::view(p, transpose ? m->vt32.get() : m->v32.get()),
                                                     vk::Gathers<float, 1>{{static_cast<const float *>(x)}}, e, s);
        }
        return VK_OK;
    });
}

int vk_spmat_set_values(vk_spmat *m, const double *values, int64_t nnz) {
    return guarded([&] {
        if (!m || (nnz > 0 && !values)) return set_error(VK_ERR_INVALID, "null argument");
        if (nnz != m->a.nnz)
            return set_error(VK_ERR_INVALID, "set_values: values size " + std::to_string(nnz) + " != nnz " +
                                                 std::to_string(m->a.nnz));
        if (m->precision != VK_PREC_FP64) return set_error(VK_ERR_UNSUPPORTED, "set_values needs a float64 operator");
        if (nnz > 0) {
            VK_CUDA(cudaMemcpyAsync(m->v64.get(), values, nnz * sizeof(double), cudaMemcpyHostToDevice, nullptr));
            vk::gather_values<double, double>(m->perm.get(), m->v64.get(), m->vt64.get(), nnz, nullptr);
        }
        return VK_OK;
    });
}

int vk_spmat_multiply(vk_spmat *m, double alpha, const vk_dvec *x, double beta, vk_dvec *y, int transpose,
                      int spmv_order) {
    return guarded([&] {
        if (!m || !x || !y) return set_error(VK_ERR_INVALID, "null argument");
        if (m->precision != VK_PREC_FP64) return set_error(VK_ERR_UNSUPPORTED, "multiply needs a float64 operator");
        const vk::CsrPattern32 &p = transpose ? m->at : m->a; // p.rows = length of y, p.cols = length of x
        const char *op = transpose ? "multiply (Yes)" : "multiply (No)";
        if (vk::dvec_size(x) != p.cols)
            return set_error(VK_ERR_INVALID, std::string(op) + ": x size " + std::to_string(vk::dvec_size(x)) +
                                                 " != " + std::to_string(p.cols));
        if (vk::dvec_size(y) != p.rows)
            return set_error(VK_ERR_INVALID, std::string(op) + ": y size " + std::to_string(vk::dvec_size(y)) +
                                                 " != " + std::to_string(p.rows));
        const bool exact = spmv_order == VK_SPMV_SEQUENTIAL;
        const double *dx = vk::dvec_ptr(x);
        double *dy = vk::dvec_ptr(y);
        if (!transpose) {
            AxpbyEpi e;
            e.alpha = alpha;
            e.beta = beta;
            e.y = dy;
            auto M = vk::view(p, m->v64.get());
            if (exact)
                vk::launch_tiles<double, double, 1, true>(M, vk::Gathers<double, 1>{{dx}}, e, nullptr);
            else
                vk::launch_tiles<double, double, 1, false>(M, vk::Gathers<double, 1>{{dx}}, e, nullptr);
        } else {
            ScatterEpi e;
            e.alpha = alpha;
            e.beta = beta;
            e.y = dy;
            auto M = vk::view(p, m->vt64.get());
            if (exact)
                vk::launch_tiles<double, double, 1, true>(M, vk::Gathers<double, 1>{{dx}}, e, nullptr);
            else
                vk::launch_tiles<double, double, 1, false>(M, vk::Gathers<double, 1>{{dx}}, e, nullptr);
        }
        return VK_OK;
    });
}

int64_t vk_spmat_bytes(const vk_spmat *m, int transpose) {
    if (!m) return 0;
    const vk::CsrPattern32 &p = transpose ? m->at : m->a;
    const int64_t s = m->precision == VK_PREC_FP64 ? 8 : 4;
    return p.nnz * (s + 4) + 4 * (int64_t(p.rows) + 1) + int64_t(p.cols) * s + int64_t(p.rows) * s;
}

int vk_spmat_variant(const vk_spmat *m, int transpose) {
    if (!m) return -1;
    return transpose ? m->at.variant : m->a.variant;
}

int vk_spmat_set_variant(vk_spmat *m, int transpose, int variant) {
    if (!m || variant < 0 || variant >= vk::kFastVariants)
        return set_error(VK_ERR_INVALID, "variant out of range");
    (transpose ? m->at : m->a).variant = variant;
    return VK_OK;
}

int vk_vec_dot_device(const double *x, const double *y, int64_t n, double *result, void *stream) {
    return guarded([&] {
        if (!result || n < 0 || (n > 0 && (!x || !y))) return set_error(VK_ERR_INVALID, "invalid argument");
        double *partials = vk::reduction_scratch(std::max<int64_t>(1, vk::reduction_blocks(n)));
        vk::launch_dot(x, y, n, partials, result, static_cast<cudaStream_t>(stream));
        return VK_OK;
    });
}

int vk_vec_norm_inf_device(const double *x, int64_t n, double *result, void *stream) {
    return guarded([&] {
        if (!result || n < 0 || (n > 0 && !x)) return set_error(VK_ERR_INVALID, "invalid argument");
        double *partials = vk::reduction_scratch(std::max<int64_t>(1, vk::reduction_blocks(n)));
        vk::launch_norm_inf(x, n, partials, result, static_cast<cudaStream_t>(stream));
        return VK_OK;
    });
}

namespace {
// One CTA; thread 0 waits on an mbarrier that expects one arrival nobody makes,
// with the same bounded poll the pipelined sparse passes use for their staged
// copies; on timeout it records the code those passes record and returns.
__global__ void bounded_wait_probe_kernel(int *err, uint32_t polls, int *gave_up) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        vk::mbar_init(&bar, 1);
        vk::fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const bool done = vk::mbar_wait_bounded(&bar, 0, polls);
        if (!done) atomicCAS(err, 0, static_cast<int>(vk::kDevErrBarrierTimeout));
        *gave_up = done ? 0 : 1;
        asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(vk::smem_u32(&bar)) : "memory");
    }
}
} // namespace

int vk_diag_bounded_wait(int32_t polls) {
    return guarded([&] {
        if (polls < 1 || polls > (1 << 20)) return set_error(VK_ERR_INVALID, "polls must be in [1, 1048576]");
        Stream st;
        int *err = vk::device_error_flag();
        vk::DevBuf<int> gave_up(1);
        bounded_wait_probe_kernel<<<1, 32, 0, st.s>>>(err, static_cast<uint32_t>(polls), gave_up.get());
        VK_LAUNCH_CHECK();
        int h = 0;
        VK_CUDA(cudaMemcpyAsync(&h, gave_up.get(), sizeof(int), cudaMemcpyDeviceToHost, st.s));
        // reads and clears the device error flag; throws (-> VK_ERR_CUDA) when set
        vk::check_device_error(st.s);
        return h ? set_error(VK_ERR_INTERNAL, "the probe's wait gave up but no device error was recorded")
                 : set_error(VK_ERR_INTERNAL, "the probe's barrier completed although nothing arrived");
    });
}

void vk_spmat_destroy(vk_spmat *m) {
    try {
        delete m;
    } catch (...) {
    }
}

int vk_batch_solve(const vk_problem *problems, int32_t count, const vk_options *opts, vk_result *results) {
    return guarded([&] {
        if (!problems || !results || count <= 0) return set_error(VK_ERR_INVALID, "invalid argument");
        vk_options o;
        if (opts)
            o = *opts;
        else {
            vk_default_options(&o);
            o.algorithm = VK_ALGO_HALPERN;
        }
        vk::batch_solve(problems, count, o, results);
        return VK_OK;
    });
}

int vk_batch_solve_shared(const vk_problem *problem, int32_t count, const double *lower, const double *upper,
                          const double *warm, const vk_options *opts, vk_result *results) {
    return guarded([&] {
        if (!problem || !results || count <= 0) return set_error(VK_ERR_INVALID, "invalid argument");
        vk_options o;
        if (opts)
            o = *opts;
        else {
            vk_default_options(&o);
            o.algorithm = VK_ALGO_HALPERN;
        }
        vk::batch_solve_shared(*problem, count, lower, upper, warm, o, results);
        return VK_OK;
    });
}

int vk_batch_solve_together(const vk_problem *problem, int32_t node_count, const double *lower,
                            const double *upper, const double *warm, const vk_problem *problems, int32_t count,
                            const vk_options *opts, vk_result *node_results, vk_result *results) {
    return guarded([&] {
        if (!problem || !problems || !node_results || !results || node_count <= 0 || count <= 0)
            return set_error(VK_ERR_INVALID, "invalid argument");
        vk_options o;
        if (opts)
            o = *opts;
        else {
            vk_default_options(&o);
            o.algorithm = VK_ALGO_HALPERN;
        }
        vk::batch_solve_together(*problem, node_count, lower, upper, warm, problems, count, o, node_results,
                                 results);
        return VK_OK;
    });
}

void vk_default_adjoint_options(vk_adjoint_options *o) {
    if (!o) return;
    o->active_tolerance = 1e-6;
    o->solve_tolerance = 1e-10;
    o->iteration_limit = 20000;
    o->device = 0;
}

int vk_lp_adjoint(const vk_problem *problems, int32_t count, const double *x, const double *y, const double *dL_dx,
                  double dL_dobj, const vk_adjoint_options *opts, double *dL_dc, double *dL_db, double *dL_dA,
                  vk_adjoint_info *info) {
    return guarded([&] {
        if (!problems || count <= 0 || !x || !dL_dx) return set_error(VK_ERR_INVALID, "invalid argument");
        int64_t m = 0;
        for (int b = 0; b < count; ++b) m += problems[b].A.rows;
        if (m > 0 && !y) return set_error(VK_ERR_INVALID, "y is required when the problems have rows");
        vk_adjoint_options o;
        if (opts)
            o = *opts;
        else
            vk_default_adjoint_options(&o);
        static const double none = 0.0;
        vk::lp_adjoint(problems, count, x, y ? y : &none, dL_dx, dL_dobj, o, dL_dc, dL_db, dL_dA, info);
        return VK_OK;
    });
}

} // extern "C"
