// apxb200.hpp -- header-only C++ drop-ins over the apxb200 C ABI.
//
// These classes keep the member surface and conventions of the reference's
// GPU solve-phase classes, so a maintainer can swap the type and keep the
// call sites:
//   apxb::cuda_sptrsv  for apxchol's cuda_sptrsv
//                      (include/apxchol/solver/sptrsv/cuda.h:164-900)
//   apxb::cuda_pcg     for apxchol's cuda_pcg
//                      (include/apxchol/solver/pcg_cuda.h:56-452)
// Errors are thrown as std::runtime_error carrying the library's message,
// as the reference does (cuda.h:36-39). Both classes are non-copyable and
// not safe for concurrent calls on one object (solve.h:96-97).
#ifndef APXB200_HPP
#define APXB200_HPP

#include <cstdint>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "apxb200.h"

namespace apxb {

inline void check(int rc, const char* where) {
    if (rc != APXB_OK) throw std::runtime_error(std::string(where) + ": " + apxb_last_error());
}

// One engine (device + stream + error word) per device and process, shared by
// the drop-ins (the reference classes all run on the current device's legacy
// stream).
class engine {
public:
    explicit engine(int device = 0) { check(apxb_engine_create(device, &h_), "apxb_engine_create"); }
    ~engine() { if (h_) apxb_engine_destroy(h_); }
    engine(const engine&) = delete;
    engine& operator=(const engine&) = delete;
    apxb_engine* get() const { return h_; }

    // The process's engine, created on first use on `device` (by default the
    // calling thread's current device); one device per process, as the
    // reference's classes. Thread-safe.
    static std::shared_ptr<engine> shared(int device = APXB_CURRENT_DEVICE) {
        static std::mutex mu;
        static std::shared_ptr<engine> e;
        std::lock_guard<std::mutex> lock(mu);
        if (!e) e = std::make_shared<engine>(device);
        return e;
    }

private:
    apxb_engine* h_ = nullptr;
};

// Drop-in for cuda_sptrsv. Csc is the reference's sparse_csc (or anything with
// rows(), outerIndexPtr(), innerIndexPtr(), valuePtr() over u32 / u32 / f32).
class cuda_sptrsv {
public:
    cuda_sptrsv() = default;
    ~cuda_sptrsv() { reset(); }
    cuda_sptrsv(const cuda_sptrsv&) = delete;
    cuda_sptrsv& operator=(const cuda_sptrsv&) = delete;

    // Per-round boundaries of the elimination (cumulative, bounds[0] = 0), as
    // apx_cholesky::install_factor hands them over (preconditioner.h:247-257).
    void set_round_bounds(std::vector<uint32_t> bounds) {
        rounds_.clear();
        for (size_t i = 1; i < bounds.size(); ++i) rounds_.push_back(bounds[i] - bounds[i - 1]);
    }

    // APXCHOL_SPTRSV_FP16, the reference's storage switch (cuda.h:186-205):
    // 1 = fp16 storage, 0 = not, anything else / unset = -1 (the default).
    static int fp16_env_tristate() {
        const char* e = std::getenv("APXCHOL_SPTRSV_FP16");
        if (!e) return -1;
        return std::string(e) == "1" ? 1 : (std::string(e) == "0" ? 0 : -1);
    }
    static bool fp16_from_env() { return fp16_env_tristate() == 1; }
    // The storage setup() picks by default. Unlike the reference (fp16 by
    // default on its own kernels), the default here is the fp64 sweep, which
    // reproduces the reference CPU backend bit for bit; =1 selects fp16.
    static bool fp16_resolved() { return fp16_env_tristate() == 1; }
    static int default_precision() { return fp16_resolved() ? APXB_PREC_FP16 : APXB_PREC_FP64; }

    // cuda_sptrsv::setup(const sparse_csc& L, node_index m) (cuda.h:233).
    // The sweeps run in the factor's permuted space, so no permutation is
    // needed here (identity); apply_perm() installs one for apply().
    template <class Csc>
    void setup(const Csc& L, uint32_t m, int precision = default_precision()) {
        const uint32_t n = static_cast<uint32_t>(L.rows());
        if (m != n && m + 1 != n) throw std::runtime_error("cuda_sptrsv::setup: m must be n or n-1");
        if (perm_.size() != n) {
            perm_.resize(n);
            for (uint32_t v = 0; v < n; ++v) perm_[v] = v;
        }
        reset();
        eng_ = engine::shared();
        check(apxb_factor_create(eng_->get(), n, reinterpret_cast<const uint32_t*>(L.outerIndexPtr()),
                                 reinterpret_cast<const uint32_t*>(L.innerIndexPtr()),
                                 reinterpret_cast<const float*>(L.valuePtr()), perm_.data(), m == n ? 1 : 0,
                                 rounds_.empty() ? nullptr : rounds_.data(),
                                 static_cast<uint32_t>(rounds_.size()), -1.0, precision, &f_),
              "cuda_sptrsv::setup");
        check(apxb_factor_info_get(f_, &info_), "cuda_sptrsv::setup");
    }
    // Elimination permutation (perm[original] = position) for apply().
    void apply_perm(std::vector<uint32_t> perm) { perm_ = std::move(perm); }

    // out = (L L^T)^-1 in over m entries; host pointers (cuda.h:464) / device pointers (cuda.h:480).
    void solve_LLt(const double* x_in, double* x_out) const {
        check(apxb_sweep_pair_host(eng_->get(), f_, x_in, x_out), "cuda_sptrsv::solve_LLt");
    }
    void solve_LLt_dev(const double* d_in, double* d_out) const {
        check(apxb_sweep_pair(eng_->get(), f_, d_in, d_out), "cuda_sptrsv::solve_LLt_dev");
    }
    // apx_cholesky::apply_core in the original ordering (preconditioner.h:403-529); returns b.z.
    double apply(const double* b, double* z, int flags = APXB_CENTER_SCHEDULE) const {
        double rz = 0.0;
        check(apxb_apply(eng_->get(), f_, b, z, flags, &rz), "apx_cholesky::apply");
        return rz;
    }
    void reset_apply_count() { check(apxb_factor_reset_apply_count(f_), "reset_apply_count"); }

    bool ready() const { return f_ != nullptr; }
    std::uint64_t stored_nnz() const { return info_.nnz_stored; }
    bool dataflow() const { return true; }
    const char* backend_name() const { return "dataflow"; }
    const char* backend_reason() const { return "apxb200 sync-free dataflow sweeps (sm_100a)"; }
    bool backend_forced() const { return false; }
    bool fp16() const { return info_.precision == APXB_PREC_FP16; }
    static constexpr std::size_t value_bytes = 4;
    std::size_t value_bytes_effective() const { return fp16() ? 2 : value_bytes; }
    std::uint64_t factor_device_bytes() const { return info_.device_bytes; }
    apxb_factor* handle() const { return f_; }
    apxb_engine* engine_handle() const { return eng_ ? eng_->get() : nullptr; }

private:
    void reset() {
        if (f_) apxb_factor_destroy(f_);
        f_ = nullptr;
    }
    std::shared_ptr<engine> eng_;
    apxb_factor* f_ = nullptr;
    apxb_factor_info info_{};
    std::vector<uint64_t> rounds_;
    std::vector<uint32_t> perm_;
};

// Drop-in for cuda_pcg. SpMat is Eigen::SparseMatrix<double> (column-major,
// int indices, compressed): the full symmetric operator in the original ordering.
class cuda_pcg {
public:
    cuda_pcg() = default;
    ~cuda_pcg() { if (a_) apxb_operator_destroy(a_); }
    cuda_pcg(const cuda_pcg&) = delete;
    cuda_pcg& operator=(const cuda_pcg&) = delete;

    // cuda_pcg::setup(L, perm) (pcg_cuda.h:68).
    template <class SpMat, class Index>
    void setup(const SpMat& L, const std::vector<Index>& perm) {
        if (a_) { apxb_operator_destroy(a_); a_ = nullptr; }
        eng_ = engine::shared();
        n_ = static_cast<int64_t>(L.rows());
        nnz_ = static_cast<int64_t>(L.nonZeros());
        std::vector<uint32_t> p(perm.begin(), perm.end());
        check(apxb_operator_create(eng_->get(), static_cast<uint32_t>(n_), L.outerIndexPtr(), L.innerIndexPtr(),
                                   L.valuePtr(), p.data(), &a_),
              "cuda_pcg::setup");
    }

    // cuda_pcg::solve (pcg_cuda.h:157). precond exposes its device factor as
    // precond.trsv_handle() (an apxb::cuda_sptrsv's handle()); the whole loop
    // runs on the device. The factor's own permutation is not used: the
    // operator's perm maps b into the factor's space. `laplacian` is implied by
    // the factor (m = n - 1) and only checked.
    template <class Precond, class Vec>
    void solve(const Precond& precond, const Vec& b_host, Vec& x_host, double tol, int max_iter, int& iters_out,
               double& residual_out, bool laplacian) {
        apxb_factor* f = precond.trsv_handle();
        apxb_factor_info inf{};
        check(apxb_factor_info_get(f, &inf), "cuda_pcg::solve");
        if (laplacian != (inf.sddm == 0)) throw std::runtime_error("cuda_pcg::solve: laplacian flag and factor differ");
        x_host.resize(b_host.size());
        apxb_pcg_result r{};
        check(apxb_pcg(eng_->get(), f, a_, b_host.data(), x_host.data(), tol, max_iter, 0, 0, &r), "cuda_pcg::solve");
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
    int spmv_lanes() const { return 1; }

private:
    std::shared_ptr<engine> eng_;
    apxb_operator* a_ = nullptr;
    int64_t n_ = 0, nnz_ = 0;
};

}  // namespace apxb

#endif
