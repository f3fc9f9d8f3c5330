// apxb200 replacement of the apxchol reference's GPU-resident PCG header,
// include/apxchol/solver/pcg_cuda.h (class cuda_pcg, pcg_cuda.h:56-452), used
// by apxchol::solve on APXCHOL_USE_CUDA builds (src/solve.cpp:687-729).
//
// setup(L, perm) builds the permuted full-symmetric operator on the device
// (pcg_cuda.h:68-152); solve(precond, b, x, tol, max_iter, iters, rnorm,
// laplacian) runs the whole PCG loop on the device -- one CUDA graph with a
// conditional WHILE node, no host round trip per iteration -- with the
// preconditioner's apxb200 factor (precond.trsv().handle(), the replacement
// cuda_sptrsv of this tree). The loop follows cpu_solver's semantics (stop
// rule, stagnation window, center-k centring, src/solve.cpp:478-654); the
// residual returned is the recurrence's, as the reference's.
#pragma once

#include <Eigen/Core>
#include <Eigen/Sparse>
#include <cuda_runtime.h>   // apxchol::solve reads cudaMemGetInfo after the solve (src/solve.cpp:722-724)

#include <cstdint>
#include <stdexcept>
#include <vector>

#include "apxchol/solver/sptrsv/cuda.h"

namespace apxchol {

class cuda_pcg {
public:
    cuda_pcg() = default;
    cuda_pcg(const cuda_pcg&) = delete;
    cuda_pcg& operator=(const cuda_pcg&) = delete;
    ~cuda_pcg() { destroy(); }

    // A = L (full symmetric, original ordering) and the factor's permutation
    // perm[original] = position.
    void setup(const Eigen::SparseMatrix<double>& L, const std::vector<node_index>& perm) {
        destroy();
        n_ = static_cast<int64_t>(L.rows());
        nnz_ = static_cast<int64_t>(L.nonZeros());
        if (static_cast<int64_t>(perm.size()) != n_) throw std::runtime_error("cuda_pcg::setup: perm size != n");
        if (!L.isCompressed()) throw std::runtime_error("cuda_pcg::setup: L must be compressed");
        eng_ = apxb::engine::shared(APXB_CURRENT_DEVICE);
        const std::vector<std::uint32_t> p(perm.begin(), perm.end());
        apxb::check(apxb_operator_create(eng_->get(), static_cast<std::uint32_t>(n_), L.outerIndexPtr(),
                                         L.innerIndexPtr(), L.valuePtr(), p.data(), &a_),
                    "cuda_pcg::setup");
    }

    template <class Precond>
    void solve(const Precond& precond, const Eigen::VectorXd& b_host, Eigen::VectorXd& x_host, double tol,
               int max_iter, int& iters_out, double& residual_out, bool laplacian) {
        if (!a_) throw std::runtime_error("cuda_pcg::solve: setup() not called");
        apxb_factor* f = precond.trsv().handle();
        if (!f) throw std::runtime_error("cuda_pcg::solve: the preconditioner has no device factor");
        apxb_factor_info inf{};
        apxb::check(apxb_factor_info_get(f, &inf), "cuda_pcg::solve");
        if (static_cast<int64_t>(inf.n) != n_) throw std::runtime_error("cuda_pcg::solve: factor and operator sizes differ");
        if (laplacian != (inf.sddm == 0)) throw std::runtime_error("cuda_pcg::solve: laplacian flag and factor differ");
        if (b_host.size() != n_) throw std::runtime_error("cuda_pcg::solve: b length != n");
        x_host.resize(n_);
        apxb_pcg_result r{};
        apxb::check(apxb_pcg(eng_->get(), f, a_, b_host.data(), x_host.data(), tol, max_iter, 0, 0, &r),
                    "cuda_pcg::solve");
        iters_out = r.iterations;
        residual_out = r.residual;
    }

    bool ready() const { return a_ != nullptr; }
    int64_t n() const { return n_; }
    int64_t nnz() const { return nnz_; }
    // The operator's values are stored in fp32 when every one is fp32-exact.
    bool fp32_operator() const {
        int v = 0;
        return a_ && apxb_operator_fp32(a_, &v) == APXB_OK && v != 0;
    }
    // Threads per row of the plain SpMV: the library picks them per row from
    // the average row length, so no single count applies; 1 is reported.
    int spmv_lanes() const { return 1; }

private:
    void destroy() {
        if (a_) apxb_operator_destroy(a_);
        a_ = nullptr;
    }
    std::shared_ptr<apxb::engine> eng_;
    apxb_operator* a_ = nullptr;
    int64_t n_ = 0, nnz_ = 0;
};

}  // namespace apxchol
