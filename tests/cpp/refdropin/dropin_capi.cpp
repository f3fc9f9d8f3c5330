// TEST INFRASTRUCTURE: the apxchol reference's own solve phase -- src/solve.cpp
// and include/apxchol/solver/preconditioner.h, unmodified -- compiled with
// APXCHOL_USE_CUDA against the replacement headers of include/apxchol_compat
// (cuda_sptrsv, cuda_pcg, cuda_ctx over libapxb200), so that the reference's
// call sites run on apxb200's kernels. C entry points for the tests:
//   dap_solve         apxchol::solve(L, b, opts)  (src/solve.cpp:681-737): the
//                     reference factorizes, then cuda_pcg runs the GPU loop
//   dap_solver_*      cpu_solver(L, F, opts) on a given factor
//                     (src/solve.cpp:295-318): apply() and solve() reach the
//                     GPU sweeps through apx_cholesky::trsv_ (a cuda_sptrsv)
// Built by the Makefile beside this file into _ref/libapxdropin.so.
#include "apxchol/solver/solve.h"

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
thread_local std::string g_err;

Eigen::SparseMatrix<double> make_matrix(int n, const int* colptr, const int* rowidx, const double* vals) {
    Eigen::SparseMatrix<double> A(n, n);
    A.resizeNonZeros(colptr[n]);
    std::memcpy(A.outerIndexPtr(), colptr, sizeof(int) * (static_cast<size_t>(n) + 1));
    std::memcpy(A.innerIndexPtr(), rowidx, sizeof(int) * static_cast<size_t>(colptr[n]));
    std::memcpy(A.valuePtr(), vals, sizeof(double) * static_cast<size_t>(colptr[n]));
    return A;
}

struct solver_handle {
    Eigen::SparseMatrix<double> A;
    apxchol::cpu_solver* slv = nullptr;
    ~solver_handle() { delete slv; }
};
}  // namespace

extern "C" {

const char* dap_last_error() { return g_err.c_str(); }

int dap_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
    return omp_get_max_threads();
#else
    (void)t;
    return 1;
#endif
}

// apxchol::solve on A (full symmetric CSC, int32) with factor seed `seed`.
// Outputs x[n], the iterations, the residual and the stored factor nnz the
// GPU SpTRSV reports through the reference's own banner-free API.
int dap_solve(int n, const int* a_colptr, const int* a_rowidx, const double* a_vals, const double* b, double tol,
              int max_iter, unsigned seed, double* x, int* iters, double* residual, double* vram_mb) {
    try {
        const Eigen::SparseMatrix<double> A = make_matrix(n, a_colptr, a_rowidx, a_vals);
        Eigen::VectorXd bv(n);
        std::memcpy(bv.data(), b, sizeof(double) * n);
        apxchol::solve_options opts;
        opts.tol = tol;
        opts.max_iter = max_iter;
        opts.factor_opts.seed = seed;
        const apxchol::solve_result r = apxchol::solve(A, bv, opts);
        std::memcpy(x, r.x.data(), sizeof(double) * n);
        *iters = static_cast<int>(r.iterations);
        *residual = r.residual;
        if (vram_mb) *vram_mb = r.solve_vram_mb;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// cpu_solver(L, F): the factor as apxchol::factorize produced it (CSC u32 /
// f32, perm[original] = position, sddm, per-round IS sizes).
int dap_solver_create(int n, const int* a_colptr, const int* a_rowidx, const double* a_vals,
                      const uint32_t* f_colptr, const uint32_t* f_rowidx, const float* f_vals,
                      const uint32_t* perm, int sddm, const uint64_t* rounds, uint32_t n_rounds, void** out) {
    try {
        auto* h = new solver_handle;
        h->A = make_matrix(n, a_colptr, a_rowidx, a_vals);
        apxchol::factorization F;
        F.L.resize(static_cast<uint32_t>(n), static_cast<uint32_t>(n));
        std::memcpy(F.L.outer_.data(), f_colptr, sizeof(uint32_t) * (static_cast<size_t>(n) + 1));
        F.L.resizeNonZeros(f_colptr[n]);
        std::memcpy(F.L.inner_.data(), f_rowidx, sizeof(uint32_t) * f_colptr[n]);
        std::memcpy(F.L.vals_.data(), f_vals, sizeof(float) * f_colptr[n]);
        F.perm.assign(perm, perm + n);
        F.sddm = sddm != 0;
        F.rounds.resize(n_rounds);
        for (uint32_t r = 0; r < n_rounds; ++r) F.rounds[r] = {0, static_cast<size_t>(rounds[r]), 0.0, 0, 0};
        apxchol::solve_options opts;
        try {
            h->slv = new apxchol::cpu_solver(h->A, std::move(F), opts, nullptr);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

void dap_solver_free(void* h) { delete static_cast<solver_handle*>(h); }

// cpu_solver::apply (the Eigen seam): z = M^-1 r, center-k counter reset first when `reset`.
int dap_apply(void* hv, const double* r, double* z, int reset) {
    try {
        auto* h = static_cast<solver_handle*>(hv);
        const Eigen::Index n = h->A.rows();
        if (reset) h->slv->preconditioner().reset_apply_count();
        Eigen::VectorXd rv(n);
        std::memcpy(rv.data(), r, sizeof(double) * n);
        const Eigen::VectorXd zv = h->slv->apply(rv);
        std::memcpy(z, zv.data(), sizeof(double) * n);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// cpu_solver::solve: the reference's host PCG, each preconditioner application on the GPU sweeps.
int dap_solver_solve(void* hv, const double* b, double* x, double tol, int max_iter, int* iters, double* residual) {
    try {
        auto* h = static_cast<solver_handle*>(hv);
        const Eigen::Index n = h->A.rows();
        Eigen::VectorXd bv(n), xv(n);
        std::memcpy(bv.data(), b, sizeof(double) * n);
        const apxchol::solve_result r = h->slv->solve(bv, Eigen::Ref<Eigen::VectorXd>(xv), tol, max_iter);
        std::memcpy(x, xv.data(), sizeof(double) * n);
        *iters = static_cast<int>(r.iterations);
        *residual = r.residual;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// What the GPU SpTRSV (the replacement cuda_sptrsv) reports through the
// reference's accessors after setup: stored nnz, dropped, grid, device bytes, fp16.
int dap_trsv_info(void* hv, uint64_t* stored, uint64_t* dropped, int* grid, uint64_t* dev_bytes, int* fp16) {
    try {
        const auto& t = static_cast<solver_handle*>(hv)->slv->preconditioner().trsv();
        *stored = t.stored_nnz();
        *dropped = t.drop_stats().dropped;
        *grid = t.dataflow_grid();
        *dev_bytes = t.factor_device_bytes();
        *fp16 = t.fp16() ? 1 : 0;
        return t.ready() ? 0 : -1;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

}  // extern "C"
