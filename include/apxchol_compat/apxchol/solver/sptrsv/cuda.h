// apxb200 replacement of the apxchol reference's GPU SpTRSV header,
// include/apxchol/solver/sptrsv/cuda.h (class cuda_sptrsv, cuda.h:164-900).
//
// Put include/apxchol_compat first on the include path of a build of the
// reference with APXCHOL_USE_CUDA defined, link libapxb200, and the
// reference's unmodified sources -- preconditioner.h (`mutable cuda_sptrsv
// trsv_`, install_factor, apply_core) and src/solve.cpp (apxchol::solve, the
// banner) -- run the solve phase on apxb200's sm_100a kernels. The other
// headers of this tree replace pcg_cuda.h and cuda_context.h the same way.
//
// What the class keeps of the reference: every member its call sites and
// tests use, non-copyable and non-movable, errors as std::runtime_error
// carrying the library's message (cuda.h:36-39), host-pointer and
// device-pointer pair solves over the factor's m permuted rows.
// What differs:
//   * the sweeps are the library's fp64 dataflow sweeps, which reproduce the
//     reference CPU backend's arithmetic (the reference GPU backend sweeps in
//     fp32 over fp16 storage by default); APXCHOL_SPTRSV_FP16=1, the
//     reference's own switch, selects the fp16 storage with fp32 sweeps.
//     preconditioner.h hands no elimination rounds to the GPU class, so the
//     sweep levels are the factor's dependency levels (omp_sptrsv's
//     APXCHOL_ROUND_LEVELS=0 levels);
//   * backend_from_env() reads APXCHOL_GPU_SPTRSV as the reference does, but
//     there is one backend (cusparse_available() is false);
//   * device_bytes_delta() is the device memory the library allocated for the
//     factor (no cudaMemGetInfo granularity).
#pragma once

#include <cstdint>
#include <cstdlib>
#include <string>
#include <vector>

#include "apxb200.hpp"
#include "apxchol/lowprec.h"
#include "apxchol/sparse_csc.h"
#include "apxchol/solver/sptrsv/factor_drop.h"

namespace apxchol {

class cuda_sptrsv {
public:
    cuda_sptrsv() = default;
    ~cuda_sptrsv() { destroy(); }
    cuda_sptrsv(const cuda_sptrsv&) = delete;
    cuda_sptrsv& operator=(const cuda_sptrsv&) = delete;
    cuda_sptrsv(cuda_sptrsv&&) = delete;
    cuda_sptrsv& operator=(cuda_sptrsv&&) = delete;

    // Value type of the stored factor in the reference's fp32 layout.
    static constexpr std::size_t value_bytes = sizeof(sptrsv_value_t);
    static constexpr const char* value_name = "float (fp32)";

    // APXCHOL_SPTRSV_FP16 (lowprec.h): 1 on, 0 off, -1 unset.
    static int fp16_env_tristate() { return sptrsv_fp16_env_tristate(); }
    static bool fp16_from_env() { return fp16_env_tristate() == 1; }
    // The storage setup() uses: fp16 only when asked for; unset means the
    // fp64 sweeps (the reference GPU backend defaults to fp16).
    static bool fp16_resolved() { return fp16_env_tristate() == 1; }
    static constexpr bool cusparse_available() { return false; }
    // APXCHOL_GPU_SPTRSV: "dataflow" -> 1, "cusparse" -> -1, unset / other -> 0
    // (AUTO), the reference's reading of the variable (cuda.h:217-231).
    static int backend_from_env() {
        const char* be = std::getenv("APXCHOL_GPU_SPTRSV");
        if (!be) return 0;
        const std::string v(be);
        return v == "dataflow" ? 1 : (v == "cusparse" ? -1 : 0);
    }

    // cuda_sptrsv::setup(const sparse_csc& L, node_index m) (cuda.h:233): the
    // factor's L11 (m = n: SDDM; m = n - 1: Laplacian, the grounded last
    // row/column dropped), the compacting drop, both sweep plans, upload.
    void setup(const sparse_csc& L, node_index m) {
        const std::uint32_t n = static_cast<std::uint32_t>(L.rows());
        if (m != n && m + 1 != n) throw std::runtime_error("cuda_sptrsv::setup: m must be n or n - 1");
        destroy();
        const int be = backend_from_env();
        if (be < 0) throw std::runtime_error("cuda_sptrsv::setup: APXCHOL_GPU_SPTRSV=cusparse: not available here");
        backend_forced_ = be > 0;
        std::vector<std::uint32_t> outer;
        const std::uint32_t* colptr = reinterpret_cast<const std::uint32_t*>(L.outerIndexPtr());
        if constexpr (sizeof(edge_index) != sizeof(std::uint32_t)) {   // APXCHOL_64BIT_INDICES builds
            if (L.nonZeros() > 0xffffffffull) throw std::runtime_error("cuda_sptrsv::setup: factor exceeds 2^32 entries");
            outer.assign(L.outerIndexPtr(), L.outerIndexPtr() + n + 1);
            colptr = outer.data();
        }
        std::vector<std::uint32_t> ident(n);
        for (std::uint32_t v = 0; v < n; ++v) ident[v] = v;   // sweeps run in the permuted space
        eng_ = apxb::engine::shared(APXB_CURRENT_DEVICE);
        const std::uint64_t used0 = apxb_engine_memory_used(eng_->get());
        const int prec = fp16_resolved() ? APXB_PREC_FP16 : APXB_PREC_FP64;
        apxb::check(apxb_factor_create(eng_->get(), n, colptr, reinterpret_cast<const std::uint32_t*>(L.innerIndexPtr()),
                                       L.valuePtr(), ident.data(), m == n ? 1 : 0, nullptr, 0, -1.0, prec, &f_),
                    "cuda_sptrsv::setup");
        apxb::check(apxb_factor_info_get(f_, &info_), "cuda_sptrsv::setup");
        delta_ = apxb_engine_memory_used(eng_->get()) - used0;
        stats_ = factor_drop_stats{};
        stats_.rel = info_.drop_rel;
        stats_.nnz_factor = info_.nnz_factor;
        stats_.nnz_stored = info_.nnz_stored;
        stats_.dropped = info_.dropped;
        stats_.dropped_flush = info_.dropped_flush;
        stats_.dropped_threshold = info_.dropped - info_.dropped_flush;
        reason_ = backend_forced_ ? "dataflow (APXCHOL_GPU_SPTRSV=dataflow): apxb200 sync-free sweeps, sm_100a"
                                  : "dataflow (AUTO): apxb200 sync-free sweeps, sm_100a";
    }

    // out = (L L^T)^-1 in over the m permuted rows: host pointers
    // (cuda.h:464-473, staged through the engine's pinned buffers) and device
    // pointers (cuda.h:480-487). in and out may alias.
    void solve_LLt(const double* x_in, double* x_out) const {
        apxb::check(apxb_sweep_pair_host(eng_->get(), f_, x_in, x_out), "cuda_sptrsv::solve_LLt");
    }
    void solve_LLt_dev(const double* d_in, double* d_out) const {
        apxb::check(apxb_sweep_pair(eng_->get(), f_, d_in, d_out), "cuda_sptrsv::solve_LLt_dev");
    }

    bool ready() const { return f_ != nullptr; }
    const factor_drop_stats& drop_stats() const { return stats_; }
    std::uint64_t stored_nnz() const { return stats_.nnz_stored; }
    bool dataflow() const { return f_ != nullptr; }
    const char* backend_name() const { return "dataflow"; }
    int dataflow_grid() const { return f_ ? info_.sweep_grid : 0; }
    bool backend_forced() const { return backend_forced_; }
    const std::string& backend_reason() const { return reason_; }
    bool fp16() const { return f_ && info_.precision == APXB_PREC_FP16; }
    std::size_t value_bytes_effective() const { return fp16() ? 2 : value_bytes; }
    std::size_t factor_device_bytes() const { return f_ ? info_.device_bytes : 0; }
    std::size_t device_bytes_delta() const { return delta_; }
    std::size_t cusparse_buffer_bytes() const { return 0; }

    // apxb200 handles, for the replacement cuda_pcg (one GPU-resident loop).
    apxb_factor* handle() const { return f_; }
    apxb_engine* engine_handle() const { return eng_ ? eng_->get() : nullptr; }

private:
    void destroy() {
        if (f_) apxb_factor_destroy(f_);
        f_ = nullptr;
        info_ = apxb_factor_info{};
        delta_ = 0;
    }
    std::shared_ptr<apxb::engine> eng_;
    apxb_factor* f_ = nullptr;
    apxb_factor_info info_{};
    factor_drop_stats stats_{};
    std::size_t delta_ = 0;
    bool backend_forced_ = false;
    std::string reason_;
};

}  // namespace apxchol
