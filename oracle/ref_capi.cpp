// TEST INFRASTRUCTURE (oracle): C entry points over the apxchol reference's own
// CPU solve phase, compiled unchanged from the reference sources into
// oracle/_ref/libapxref.so by oracle/Makefile. Used by the tests to pin the C
// restatement (oracle/apxoracle.c) and by bench.py's CPU-baseline leg. The CUDA
// product never loads it.
//
// Wrapped reference symbols:
//   cpu_solver(L, F, opts) / solve / apply    src/solve.cpp:295-318, 478-679
//   apx_cholesky::apply_fused / reset_apply_count   preconditioner.h:317, 370-377
//   omp_sptrsv forward_solve / transpose_solve / csr_* / csc_*   sptrsv/omp.h:1048-1058, 1176-1189
#include "apxchol/solver/solve.h"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
thread_local std::string g_err;

struct solver_handle {
    Eigen::SparseMatrix<double> A;
    apxchol::cpu_solver* slv = nullptr;
    ~solver_handle() { delete slv; }
};

apxchol::factorization make_factor(uint32_t n, const uint32_t* colptr, const uint32_t* rowidx,
                                   const float* vals, const uint32_t* perm, int sddm,
                                   const uint64_t* rounds, uint32_t n_rounds) {
    apxchol::factorization F;
    F.L.resize(n, n);
    std::memcpy(F.L.outer_.data(), colptr, sizeof(uint32_t) * (static_cast<size_t>(n) + 1));
    F.L.resizeNonZeros(colptr[n]);
    std::memcpy(F.L.inner_.data(), rowidx, sizeof(uint32_t) * colptr[n]);
    std::memcpy(F.L.vals_.data(), vals, sizeof(float) * colptr[n]);
    F.perm.assign(perm, perm + n);
    F.sddm = sddm != 0;
    F.rounds.resize(n_rounds);
    for (uint32_t r = 0; r < n_rounds; ++r) F.rounds[r] = {0, static_cast<size_t>(rounds[r]), 0.0, 0, 0};
    return F;
}
}  // namespace

extern "C" {

const char* apxref_last_error() { return g_err.c_str(); }

int apxref_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
    return omp_get_max_threads();
#else
    (void)t;
    return 1;
#endif
}

// A: full symmetric CSC (int32) of the operator; the factor as produced by
// apxchol::factorize (CSC u32 / f32, perm, sddm, per-round IS sizes).
int apxref_solver_create(int n, const int* a_colptr, const int* a_rowidx, const double* a_vals,
                         const uint32_t* f_colptr, const uint32_t* f_rowidx, const float* f_vals,
                         const uint32_t* perm, int sddm, const uint64_t* rounds, uint32_t n_rounds,
                         int keep_factor, void** out) {
    try {
        auto* h = new solver_handle;
        h->A.resize(n, n);
        h->A.resizeNonZeros(a_colptr[n]);
        std::memcpy(h->A.outerIndexPtr(), a_colptr, sizeof(int) * (static_cast<size_t>(n) + 1));
        std::memcpy(h->A.innerIndexPtr(), a_rowidx, sizeof(int) * a_colptr[n]);
        std::memcpy(h->A.valuePtr(), a_vals, sizeof(double) * a_colptr[n]);
        apxchol::solve_options opts;
        opts.keep_factor_values = keep_factor != 0;
        try {
            h->slv = new apxchol::cpu_solver(
                h->A, make_factor(static_cast<uint32_t>(n), f_colptr, f_rowidx, f_vals, perm, sddm, rounds, n_rounds),
                opts, nullptr);
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

void apxref_solver_free(void* h) { delete static_cast<solver_handle*>(h); }

// cpu_solver::solve from x0 = 0. Returns the wall seconds of the call in *secs.
int apxref_solve(void* hv, const double* b, double* x, double tol, int max_iter, int* iters,
                 double* residual, double* secs) {
    try {
        auto* h = static_cast<solver_handle*>(hv);
        const Eigen::Index n = h->A.rows();
        Eigen::VectorXd bv(n);
        std::memcpy(bv.data(), b, sizeof(double) * n);
        Eigen::VectorXd xv(n);
        const auto t0 = std::chrono::steady_clock::now();
        apxchol::solve_result r = h->slv->solve(bv, Eigen::Ref<Eigen::VectorXd>(xv), tol, max_iter);
        const auto t1 = std::chrono::steady_clock::now();
        std::memcpy(x, xv.data(), sizeof(double) * n);
        *iters = static_cast<int>(r.iterations);
        *residual = r.residual;
        if (secs) *secs = std::chrono::duration<double>(t1 - t0).count();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// One preconditioner application through the Eigen seam (cpu_solver::apply ->
// apx_cholesky::_solve_impl). The center-k counter is reset first when
// `reset` is set.
int apxref_apply(void* hv, const double* r, double* z, int reset) {
    auto* h = static_cast<solver_handle*>(hv);
    const Eigen::Index n = h->A.rows();
    if (reset) h->slv->preconditioner().reset_apply_count();
    Eigen::VectorXd rv(n);
    std::memcpy(rv.data(), r, sizeof(double) * n);
    Eigen::VectorXd zv = h->slv->apply(rv);
    std::memcpy(z, zv.data(), sizeof(double) * n);
    return 0;
}

// apx_cholesky::apply_fused: z = M^-1 r with r.z returned (PCG entry).
double apxref_apply_fused(void* hv, const double* r, double r_sum, double* z, int reset) {
    auto* h = static_cast<solver_handle*>(hv);
    if (reset) h->slv->preconditioner().reset_apply_count();
    return h->slv->preconditioner().apply_fused(r, r_sum, z);
}

// Direct sweeps over the permuted factor dimension m.
void apxref_forward(void* hv, const double* in, double* out) {
    static_cast<solver_handle*>(hv)->slv->preconditioner().trsv().forward_solve(in, out);
}
void apxref_transpose(void* hv, const double* in, double* out) {
    static_cast<solver_handle*>(hv)->slv->preconditioner().trsv().transpose_solve(in, out);
}
double apxref_pair_seconds(void* hv, const double* in, double* tmp, double* out, int reps) {
    const auto& t = static_cast<solver_handle*>(hv)->slv->preconditioner().trsv();
    const auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < reps; ++k) { t.forward_solve(in, tmp); t.transpose_solve(tmp, out); }
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count() / reps;
}

// Sizes of the SpTRSV arrays: m, nnz_stored, forward / backward level counts.
void apxref_sptrsv_info(void* hv, uint32_t* m, uint64_t* nnz, int* fwd_levels, int* bck_levels) {
    const auto& t = static_cast<solver_handle*>(hv)->slv->preconditioner().trsv();
    *m = static_cast<uint32_t>(t.csr_row_ptr().size() - 1);
    *nnz = t.stored_nnz();
    *fwd_levels = t.num_fwd_levels();
    *bck_levels = t.num_bck_levels();
}

// Copy of the SpTRSV's CSR(L11) and CSC(L11) arrays (fp32 storage).
void apxref_sptrsv_arrays(void* hv, uint32_t* csr_ptr, uint32_t* csr_idx, float* csr_val,
                          uint32_t* csc_ptr, uint32_t* csc_idx, float* csc_val) {
    const auto& t = static_cast<solver_handle*>(hv)->slv->preconditioner().trsv();
    std::memcpy(csr_ptr, t.csr_row_ptr().data(), sizeof(uint32_t) * t.csr_row_ptr().size());
    std::memcpy(csr_idx, t.csr_col_idx().data(), sizeof(uint32_t) * t.csr_col_idx().size());
    std::memcpy(csr_val, t.csr_vals().data(), sizeof(float) * t.csr_vals().size());
    std::memcpy(csc_ptr, t.csc_col_ptr().data(), sizeof(uint32_t) * t.csc_col_ptr().size());
    std::memcpy(csc_idx, t.csc_row_idx().data(), sizeof(uint32_t) * t.csc_row_idx().size());
    std::memcpy(csc_val, t.csc_vals().data(), sizeof(float) * t.csc_vals().size());
}

// Per-level sizes of each direction (sizes[l] for l < levels).
void apxref_level_sizes(void* hv, int fwd, int* sizes) {
    const auto& t = static_cast<solver_handle*>(hv)->slv->preconditioner().trsv();
    std::vector<int> s;
    std::vector<long long> w;
    t.level_stats(fwd != 0, s, w);
    std::memcpy(sizes, s.data(), sizeof(int) * s.size());
}

}  // extern "C"
