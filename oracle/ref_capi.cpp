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
//   cuda_host:: build_L11_csc_int / column_scales / apply_factor_drop /
//     narrow_fp16_scaled / transpose_csr   sptrsv/cuda_host.h:66-258 (CUDA-free)
#include "apxchol/solver/solve.h"
#include "apxchol/solver/sptrsv/cuda_host.h"

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

// The reference GPU backend's host preparation with fp16 storage: what
// cuda_sptrsv::setup computes before its upload (cuda.h:276-372): L11 as int
// CSC, the pre-drop column scales, the drop with the fp16 keep predicate, the
// narrowing and the transpose carrying the 16-bit values. The scale fallback
// (cuda.h:295-301) sits inside the CUDA class, so its five lines are restated
// here. Call once with NULL arrays for *m_out / *nnz_out.
// stats[3] = {dropped, dropped_flush, flushed}.
int apxref_fp16_prep(uint32_t n, const uint32_t* colptr, const uint32_t* rowidx, const float* vals, int sddm,
                     double rel, uint32_t* m_out, uint64_t* nnz_out, int* lt_ptr, int* lt_idx, uint16_t* lt_val16,
                     int* l_ptr, int* l_idx, uint16_t* l_val16, float* diag, float* inv_scale, uint64_t* stats) {
    try {
        namespace ch = apxchol::cuda_host;
        std::vector<uint32_t> perm(n);
        for (uint32_t v = 0; v < n; ++v) perm[v] = v;
        const apxchol::factorization F = make_factor(n, colptr, rowidx, vals, perm.data(), sddm, nullptr, 0);
        const int64_t m = sddm ? n : n - 1;
        ch::csr_int<float> LT = ch::build_L11_csc_int<float>(F.L, m);
        std::vector<float> col_scale = ch::column_scales(LT);
        for (int64_t j = 0; j < m; ++j) {
            const float s = col_scale[static_cast<size_t>(j)];
            const float d = LT.vals[LT.ptr[static_cast<size_t>(j)]];
            if (!std::isfinite(1.0f / s) || !std::isfinite(d / s)) col_scale[static_cast<size_t>(j)] = 1.0f;
        }
        const apxchol::factor_drop_stats st = ch::apply_factor_drop(LT, col_scale, rel, true);
        ch::fp16_scaled_arrays h16 = ch::narrow_fp16_scaled(LT, col_scale);
        *m_out = static_cast<uint32_t>(m);
        *nnz_out = static_cast<uint64_t>(LT.nnz);
        if (!lt_ptr) return 0;
        const size_t nnz = static_cast<size_t>(LT.nnz);
        std::memcpy(lt_ptr, LT.ptr.data(), sizeof(int) * (static_cast<size_t>(m) + 1));
        std::memcpy(lt_idx, LT.idx.get(), sizeof(int) * nnz);
        std::memcpy(lt_val16, h16.vals.get(), 2 * nnz);
        std::memcpy(diag, h16.diag.data(), 4 * static_cast<size_t>(m));
        std::memcpy(inv_scale, h16.inv_scale.data(), 4 * static_cast<size_t>(m));
        ch::csr_int<uint16_t> LT16;
        LT16.m = LT.m; LT16.nnz = LT.nnz; LT16.ptr = LT.ptr;
        LT16.idx = std::move(LT.idx);
        LT16.vals = std::move(h16.vals);
        const ch::csr_int<uint16_t> L16 = ch::transpose_csr(LT16);
        std::memcpy(l_ptr, L16.ptr.data(), sizeof(int) * (static_cast<size_t>(m) + 1));
        std::memcpy(l_idx, L16.idx.get(), sizeof(int) * nnz);
        std::memcpy(l_val16, L16.vals.get(), 2 * nnz);
        stats[0] = st.dropped; stats[1] = st.dropped_flush; stats[2] = h16.flushed;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

}  // extern "C"
