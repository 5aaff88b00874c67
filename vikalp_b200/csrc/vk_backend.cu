// Device vectors and the vector primitives of the reference's ExecutionBackend
// contract (include/vikalp/contracts/ExecutionBackend.hpp:36-64 in VIKALP):
// create_vector, upload, download, fill, copy, axpby, dot, norm_inf,
// project_box. The C++ backend class that VIKALP's solver code holds
// (make_cuda_backend, vikalp_b200/host/backend.cpp) is built on these and on
// vk_spmat_multiply / vk_spmat_set_values (vk_capi.cu).
//
// Semantics follow the reference's CPU backend (src/backend/cpu_ops.cpp):
// axpby rounds alpha*x and beta*y separately and adds them (no FMA), so it is
// bit-identical to the CPU loop; project_box is std::min(std::max(x, lo), hi)
// (NaN in x passes through); norm_inf ignores NaN as std::max does; dot is a
// fixed-order tree sum (deterministic; equal to the CPU's sequential sum up to
// rounding). Size mismatches return VK_ERR_INVALID with the operation named.
// All work is on the legacy default stream of the calling thread's device;
// dot, norm_inf and download return after the device finished.
#include "vk_solver.h"
#include "vk_vec.cuh"

#include <string>

struct vk_dvec {
    int device = 0;
    int64_t n = 0;
    vk::DevBuf<double> d;
};

namespace vk {
int record_error(int code, const std::string &msg);
double *dvec_ptr(vk_dvec *v) { return v->d.get(); }
const double *dvec_ptr(const vk_dvec *v) { return v->d.get(); }
int64_t dvec_size(const vk_dvec *v) { return v->n; }
} // namespace vk

namespace {

__global__ void dvec_fill_kernel(double *__restrict__ y, int64_t n, double v) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        y[i] = v;
}

// y = alpha * x + beta * y, each product rounded on its own (cpu_ops.cpp axpby)
__global__ void dvec_axpby_kernel(double alpha, const double *__restrict__ x, double beta, double *__restrict__ y,
                                  int64_t n) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        y[i] = __dadd_rn(__dmul_rn(alpha, x[i]), __dmul_rn(beta, y[i]));
}

__global__ void dvec_project_kernel(double *__restrict__ x, const double *__restrict__ lo,
                                    const double *__restrict__ hi, int64_t n) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        x[i] = vk::clampbox(x[i], lo[i], hi[i]);
}

int grid_of(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return static_cast<int>(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

template <class F>
int guarded_dvec(F &&f) {
    try {
        return f();
    } catch (const vk::CudaFailure &e) {
        return vk::record_error(VK_ERR_CUDA, e.what());
    } catch (const std::exception &e) {
        return vk::record_error(VK_ERR_INTERNAL, e.what());
    } catch (...) {
        return vk::record_error(VK_ERR_INTERNAL, "unknown failure");
    }
}

// One device double per device for reduction results (allocated on first use,
// kept until exit; calls are ordered on the default stream).
double *result_slot() {
    static double *slots[64] = {nullptr};
    int dev = 0;
    VK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw vk::CudaFailure("device ordinal out of range");
    if (!slots[dev]) VK_CUDA(cudaMalloc(&slots[dev], sizeof(double)));
    return slots[dev];
}

int size_error(const char *op, int64_t a, int64_t b) {
    return vk::record_error(VK_ERR_INVALID, std::string(op) + ": size " + std::to_string(a) + " != size " +
                                                std::to_string(b));
}

} // namespace

extern "C" {

int vk_device_select(int32_t device) {
    return guarded_dvec([&] {
        VK_CUDA(cudaSetDevice(device));
        return VK_OK;
    });
}

int vk_device_synchronize(void) {
    return guarded_dvec([&] {
        VK_CUDA(cudaDeviceSynchronize());
        return VK_OK;
    });
}

int vk_dvec_create(int64_t n, vk_dvec **out) {
    return guarded_dvec([&] {
        if (!out) return vk::record_error(VK_ERR_INVALID, "null argument");
        *out = nullptr;
        if (n < 0) return vk::record_error(VK_ERR_INVALID, "vector size must be non-negative");
        auto v = std::make_unique<vk_dvec>();
        VK_CUDA(cudaGetDevice(&v->device));
        v->n = n;
        v->d.reset(static_cast<size_t>(n));
        if (n > 0) VK_CUDA(cudaMemsetAsync(v->d.get(), 0, n * sizeof(double), nullptr));
        *out = v.release();
        return VK_OK;
    });
}

void vk_dvec_destroy(vk_dvec *v) {
    try {
        delete v;
    } catch (...) {
    }
}

int64_t vk_dvec_size(const vk_dvec *v) { return v ? v->n : -1; }

int vk_dvec_upload(vk_dvec *v, const double *host, int64_t n) {
    return guarded_dvec([&] {
        if (!v || (n > 0 && !host)) return vk::record_error(VK_ERR_INVALID, "null argument");
        if (n != v->n) return size_error("upload", n, v->n);
        if (n > 0) VK_CUDA(cudaMemcpyAsync(v->d.get(), host, n * sizeof(double), cudaMemcpyHostToDevice, nullptr));
        return VK_OK;
    });
}

int vk_dvec_download(const vk_dvec *v, double *host, int64_t n) {
    return guarded_dvec([&] {
        if (!v || (n > 0 && !host)) return vk::record_error(VK_ERR_INVALID, "null argument");
        if (n != v->n) return size_error("download", n, v->n);
        if (n > 0) VK_CUDA(cudaMemcpyAsync(host, v->d.get(), n * sizeof(double), cudaMemcpyDeviceToHost, nullptr));
        VK_CUDA(cudaStreamSynchronize(nullptr));
        return VK_OK;
    });
}

int vk_dvec_fill(vk_dvec *v, double value) {
    return guarded_dvec([&] {
        if (!v) return vk::record_error(VK_ERR_INVALID, "null argument");
        if (v->n > 0) {
            dvec_fill_kernel<<<grid_of(v->n), 256>>>(v->d.get(), v->n, value);
            VK_LAUNCH_CHECK();
        }
        return VK_OK;
    });
}

int vk_dvec_copy(const vk_dvec *src, vk_dvec *dst) {
    return guarded_dvec([&] {
        if (!src || !dst) return vk::record_error(VK_ERR_INVALID, "null argument");
        if (src->n != dst->n) return size_error("copy", src->n, dst->n);
        if (src != dst && src->n > 0)
            VK_CUDA(cudaMemcpyAsync(dst->d.get(), src->d.get(), src->n * sizeof(double), cudaMemcpyDeviceToDevice,
                                    nullptr));
        return VK_OK;
    });
}

int vk_dvec_axpby(double alpha, const vk_dvec *x, double beta, vk_dvec *y) {
    return guarded_dvec([&] {
        if (!x || !y) return vk::record_error(VK_ERR_INVALID, "null argument");
        if (x->n != y->n) return size_error("axpby", x->n, y->n);
        if (y->n > 0) {
            dvec_axpby_kernel<<<grid_of(y->n), 256>>>(alpha, x->d.get(), beta, y->d.get(), y->n);
            VK_LAUNCH_CHECK();
        }
        return VK_OK;
    });
}

int vk_dvec_dot(const vk_dvec *x, const vk_dvec *y, double *result) {
    return guarded_dvec([&] {
        if (!x || !y || !result) return vk::record_error(VK_ERR_INVALID, "null argument");
        if (x->n != y->n) return size_error("dot", x->n, y->n);
        double *r = result_slot();
        double *partials = vk::reduction_scratch(vk::reduction_blocks(x->n));
        vk::launch_dot(x->d.get(), y->d.get(), x->n, partials, r, nullptr);
        VK_CUDA(cudaMemcpyAsync(result, r, sizeof(double), cudaMemcpyDeviceToHost, nullptr));
        VK_CUDA(cudaStreamSynchronize(nullptr));
        return VK_OK;
    });
}

int vk_dvec_norm_inf(const vk_dvec *x, double *result) {
    return guarded_dvec([&] {
        if (!x || !result) return vk::record_error(VK_ERR_INVALID, "null argument");
        double *r = result_slot();
        double *partials = vk::reduction_scratch(vk::reduction_blocks(x->n));
        vk::launch_norm_inf(x->d.get(), x->n, partials, r, nullptr);
        VK_CUDA(cudaMemcpyAsync(result, r, sizeof(double), cudaMemcpyDeviceToHost, nullptr));
        VK_CUDA(cudaStreamSynchronize(nullptr));
        return VK_OK;
    });
}

int vk_dvec_project_box(vk_dvec *x, const vk_dvec *lower, const vk_dvec *upper) {
    return guarded_dvec([&] {
        if (!x || !lower || !upper) return vk::record_error(VK_ERR_INVALID, "null argument");
        if (lower->n != x->n) return size_error("project_box (lower)", lower->n, x->n);
        if (upper->n != x->n) return size_error("project_box (upper)", upper->n, x->n);
        if (x->n > 0) {
            dvec_project_kernel<<<grid_of(x->n), 256>>>(x->d.get(), lower->d.get(), upper->d.get(), x->n);
            VK_LAUNCH_CHECK();
        }
        return VK_OK;
    });
}

} // extern "C"
