// make_cuda_backend(): VIKALP's ExecutionBackend contract
// (include/vikalp/contracts/ExecutionBackend.hpp) over this library's C ABI --
// device vectors (vk_dvec_*) and resident sparse operators with their
// pre-built transposes (vk_spmat_*). It replaces the reference's CUDA backend
// (cuda/cuda_ops.cu: cudaMalloc'ed vectors, cuSPARSE SpMV, five SIMT kernels,
// host-finished reductions) for callers that drive PDHG or other algorithms
// primitive by primitive; the fused solvers (vk_pdhg_*) do not go through it.
// solve_linear_system is BiCGSTAB composed of the backend's own primitives,
// step for step as the reference's CPU backend runs it
// (src/backend/cpu_ops.cpp:160-267).
#include "vikalp/backend/CudaBackend.hpp"
#include "vikalp_b200.h"

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

namespace vikalp {
namespace {

void check(int rc, const char *what) {
    if (rc == VK_OK) return;
    const std::string msg = std::string("CudaBackend: ") + what + ": " + vk_last_error();
    if (rc == VK_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

[[noreturn]] void dim_error(const std::string &msg) { throw std::invalid_argument("CudaBackend: " + msg); }

class DeviceVector final : public BackendVector {
public:
    explicit DeviceVector(Index n) {
        if (n < 0) dim_error("vector size must be non-negative");
        check(vk_dvec_create(n, &v_), "create_vector");
    }
    ~DeviceVector() override { vk_dvec_destroy(v_); }
    DeviceVector(const DeviceVector &) = delete;
    DeviceVector &operator=(const DeviceVector &) = delete;
    [[nodiscard]] Index size() const noexcept override { return vk_dvec_size(v_); }
    vk_dvec *get() const noexcept { return v_; }

private:
    vk_dvec *v_ = nullptr;
};

class DeviceMatrix final : public BackendMatrix {
public:
    explicit DeviceMatrix(const CsrPattern &p) : rows_(p.rows), cols_(p.columns) {
        if (p.rows < 0 || p.columns < 0) dim_error("matrix dimensions must be non-negative");
        if (p.row_offsets.size() != static_cast<std::size_t>(p.rows) + 1)
            dim_error("CsrPattern row_offsets size != rows+1");
        if (p.row_offsets.front() != 0 || p.row_offsets.back() != static_cast<Index>(p.column_indices.size()))
            dim_error("CsrPattern row_offsets do not describe column_indices");
        nnz_ = static_cast<Index>(p.column_indices.size());
        const std::vector<double> zeros(static_cast<std::size_t>(nnz_), 0.0);
        const vk_csr a{p.rows, p.columns, p.row_offsets.data(), p.column_indices.data(), zeros.data()};
        check(vk_spmat_create(&a, VK_PREC_FP64, &m_), "create_matrix");
    }
    ~DeviceMatrix() override { vk_spmat_destroy(m_); }
    DeviceMatrix(const DeviceMatrix &) = delete;
    DeviceMatrix &operator=(const DeviceMatrix &) = delete;
    [[nodiscard]] Index rows() const noexcept override { return rows_; }
    [[nodiscard]] Index columns() const noexcept override { return cols_; }
    Index nnz() const noexcept { return nnz_; }
    vk_spmat *get() const noexcept { return m_; }

private:
    Index rows_ = 0, cols_ = 0, nnz_ = 0;
    vk_spmat *m_ = nullptr;
};

DeviceVector &dev(BackendVector &v) {
    auto *p = dynamic_cast<DeviceVector *>(&v);
    if (!p) dim_error("BackendVector is not a CudaBackend vector");
    return *p;
}
const DeviceVector &dev(const BackendVector &v) {
    const auto *p = dynamic_cast<const DeviceVector *>(&v);
    if (!p) dim_error("BackendVector is not a CudaBackend vector");
    return *p;
}
const DeviceMatrix &dev(const BackendMatrix &m) {
    const auto *p = dynamic_cast<const DeviceMatrix *>(&m);
    if (!p) dim_error("BackendMatrix is not a CudaBackend matrix");
    return *p;
}
DeviceMatrix &dev(BackendMatrix &m) {
    auto *p = dynamic_cast<DeviceMatrix *>(&m);
    if (!p) dim_error("BackendMatrix is not a CudaBackend matrix");
    return *p;
}

class B200Backend final : public ExecutionBackend {
public:
    explicit B200Backend(CudaProductOrder order)
        : order_(order == CudaProductOrder::Sequential ? VK_SPMV_SEQUENTIAL : VK_SPMV_FAST) {
        check(vk_device_select(0), "device 0");
    }

    [[nodiscard]] std::unique_ptr<BackendVector> create_vector(Index size) override {
        return std::make_unique<DeviceVector>(size);
    }
    [[nodiscard]] std::unique_ptr<BackendMatrix> create_matrix(const CsrPattern &pattern) override {
        return std::make_unique<DeviceMatrix>(pattern);
    }
    void upload(std::span<const Scalar> source, BackendVector &target) override {
        check(vk_dvec_upload(dev(target).get(), source.data(), static_cast<int64_t>(source.size())), "upload");
    }
    void download(const BackendVector &source, std::span<Scalar> target) const override {
        check(vk_dvec_download(dev(source).get(), target.data(), static_cast<int64_t>(target.size())), "download");
    }
    void set_values(std::span<const Scalar> values, BackendMatrix &target) override {
        check(vk_spmat_set_values(dev(target).get(), values.data(), static_cast<int64_t>(values.size())),
              "set_values");
    }
    void fill(BackendVector &target, Scalar value) override { check(vk_dvec_fill(dev(target).get(), value), "fill"); }
    void copy(const BackendVector &source, BackendVector &target) override {
        check(vk_dvec_copy(dev(source).get(), dev(target).get()), "copy");
    }
    void axpby(Scalar alpha, const BackendVector &x, Scalar beta, BackendVector &y) override {
        check(vk_dvec_axpby(alpha, dev(x).get(), beta, dev(y).get()), "axpby");
    }
    [[nodiscard]] Scalar dot(const BackendVector &x, const BackendVector &y) override {
        double r = 0.0;
        check(vk_dvec_dot(dev(x).get(), dev(y).get(), &r), "dot");
        return r;
    }
    [[nodiscard]] Scalar norm_inf(const BackendVector &x) override {
        double r = 0.0;
        check(vk_dvec_norm_inf(dev(x).get(), &r), "norm_inf");
        return r;
    }
    void project_box(BackendVector &x, const BackendVector &lower, const BackendVector &upper) override {
        check(vk_dvec_project_box(dev(x).get(), dev(lower).get(), dev(upper).get()), "project_box");
    }
    void multiply(Scalar alpha, const BackendMatrix &matrix, const BackendVector &x, Scalar beta, BackendVector &y,
                  Transpose transpose) override {
        if (&x == &y) dim_error("multiply: x and y must be distinct vectors");
        check(vk_spmat_multiply(dev(matrix).get(), alpha, dev(x).get(), beta, dev(y).get(),
                                transpose == Transpose::Yes ? 1 : 0, order_),
              "multiply");
    }

    // BiCGSTAB from x = 0 with the reference's breakdown and stopping rules:
    // stop when |s| or |r| (infinity norm) <= tolerance, give up on a zero
    // rho, r_hat'v or t't, finish on omega == 0 (cpu_ops.cpp:160-267).
    [[nodiscard]] LinearSolveResult solve_linear_system(const BackendMatrix &matrix, const BackendVector &rhs,
                                                        BackendVector &solution, MatrixProperty,
                                                        Scalar tolerance, Index iteration_limit) override {
        const auto &A = dev(matrix);
        if (A.rows() != A.columns())
            dim_error("solve_linear_system: matrix must be square (" + std::to_string(A.rows()) + "x" +
                      std::to_string(A.columns()) + ")");
        if (rhs.size() != A.rows())
            dim_error("solve_linear_system: rhs size " + std::to_string(rhs.size()) + " != matrix rows " +
                      std::to_string(A.rows()));
        if (solution.size() != A.rows())
            dim_error("solve_linear_system: solution size " + std::to_string(solution.size()) + " != matrix rows " +
                      std::to_string(A.rows()));
        if (!std::isfinite(tolerance) || tolerance < 0.0)
            dim_error("solve_linear_system: tolerance must be finite and non-negative");
        if (iteration_limit < 0) dim_error("solve_linear_system: iteration_limit must be non-negative");
        const Index n = A.rows();
        auto &x = solution;
        fill(x, 0.0);
        DeviceVector r(n), r_hat(n), p(n), v(n), s(n), t(n);
        copy(rhs, r);
        copy(r, r_hat);
        Scalar rho_prev = 1.0, alpha = 1.0, omega = 1.0;
        Scalar r_hat_dot_r = dot(r_hat, r);
        const Scalar initial = norm_inf(r);
        if (initial <= tolerance) return LinearSolveResult{true, 0, initial};
        LinearSolveResult res;
        for (Index iter = 0; iter < iteration_limit; ++iter) {
            res.iterations = iter + 1;
            const Scalar rho = r_hat_dot_r;
            if (rho == 0.0) break;
            if (iter == 0) {
                copy(r, p);
            } else {
                const Scalar beta = (rho / rho_prev) * (alpha / omega);
                axpby(-omega, v, 1.0, p); // p - omega v
                axpby(1.0, r, beta, p);   // r + beta (p - omega v)
            }
            multiply(1.0, matrix, p, 0.0, v, Transpose::No);
            const Scalar denom = dot(r_hat, v);
            if (denom == 0.0) break;
            alpha = rho / denom;
            copy(r, s);
            axpby(-alpha, v, 1.0, s); // s = r - alpha v
            const Scalar norm_s = norm_inf(s);
            if (norm_s <= tolerance) {
                axpby(alpha, p, 1.0, x);
                return LinearSolveResult{true, iter + 1, norm_s};
            }
            multiply(1.0, matrix, s, 0.0, t, Transpose::No);
            const Scalar tt = dot(t, t);
            if (tt == 0.0) break;
            omega = dot(t, s) / tt;
            if (omega == 0.0) {
                axpby(alpha, p, 1.0, x);
                copy(s, r);
                break;
            }
            axpby(alpha, p, 1.0, x);
            axpby(omega, s, 1.0, x);
            copy(s, r);
            axpby(-omega, t, 1.0, r); // r = s - omega t
            const Scalar norm_r = norm_inf(r);
            if (norm_r <= tolerance) return LinearSolveResult{true, iter + 1, norm_r};
            r_hat_dot_r = dot(r_hat, r);
            rho_prev = rho;
        }
        // final residual |b - A x|
        multiply(1.0, matrix, x, 0.0, t, Transpose::No);
        axpby(1.0, rhs, -1.0, t);
        res.converged = false;
        res.residual = norm_inf(t);
        return res;
    }

    void synchronize() override { check(vk_device_synchronize(), "synchronize"); }

private:
    int order_;
};

} // namespace

std::unique_ptr<ExecutionBackend> make_cuda_backend() { return make_cuda_backend(CudaProductOrder::Fast); }

std::unique_ptr<ExecutionBackend> make_cuda_backend(CudaProductOrder order) {
    return std::make_unique<B200Backend>(order);
}

} // namespace vikalp
