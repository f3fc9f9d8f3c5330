// C entry points around the apxchol reference's own seeded factorization
// (src/factorization.cpp, include/apxchol/solver/factorization.h:201-204), compiled
// unchanged from the reference sources. The solve phase consumes the factor it
// produces; this library is the setup phase, not part of the measured path.
//
// The factorization is deterministic for a fixed (matrix, seed, thread count),
// so every call pins its OpenMP team to `threads` and restores the previous
// setting afterwards.
#include "apxchol/solver/factorization.h"

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
thread_local std::string g_err;

struct factor_handle {
    apxchol::factorization F;
};
}  // namespace

extern "C" {

const char* apxref_setup_last_error() { return g_err.c_str(); }

// Factorize the n x n symmetric matrix given as a full (both triangles) CSC with
// int32 indices, rows ascending within each column. storage: 0 vec, 1
// forward_star, 2 bstr, 3 vec_pool (the reference default).
int apxref_factorize(int n, const int* colptr, const int* rowidx, const double* vals,
                     unsigned seed, int threads, int storage, void** out) {
    try {
        Eigen::SparseMatrix<double> A(n, n);
        A.resizeNonZeros(colptr[n]);
        std::memcpy(A.outerIndexPtr(), colptr, sizeof(int) * (static_cast<size_t>(n) + 1));
        std::memcpy(A.innerIndexPtr(), rowidx, sizeof(int) * static_cast<size_t>(colptr[n]));
        std::memcpy(A.valuePtr(), vals, sizeof(double) * static_cast<size_t>(colptr[n]));
        apxchol::factor_options opts;
        opts.seed = seed;
#ifdef _OPENMP
        const int prev = omp_get_max_threads();
        if (threads > 0) omp_set_num_threads(threads);
#endif
        auto* h = new factor_handle;
        try {
            h->F = apxchol::factorize(A, static_cast<apxchol::graph_storage>(storage), opts, nullptr);
        } catch (...) {
            delete h;
#ifdef _OPENMP
            omp_set_num_threads(prev);
#endif
            throw;
        }
#ifdef _OPENMP
        omp_set_num_threads(prev);
#endif
        *out = h;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

int apxref_factor_info(void* hv, uint32_t* n, uint64_t* nnz, int* sddm, uint32_t* n_rounds,
                       int64_t* lumped) {
    auto* h = static_cast<factor_handle*>(hv);
    *n = h->F.L.rows();
    *nnz = h->F.L.nonZeros();
    *sddm = h->F.sddm ? 1 : 0;
    *n_rounds = static_cast<uint32_t>(h->F.rounds.size());
    *lumped = static_cast<int64_t>(h->F.lumped_offdiag);
    return 0;
}

// Copy the factor out: CSC colptr[n+1], rowidx[nnz], vals[nnz] (fp32), perm[n]
// and the per-round independent-set sizes (rounds[n_rounds]).
int apxref_factor_copy(void* hv, uint32_t* colptr, uint32_t* rowidx, float* vals, uint32_t* perm,
                       uint64_t* round_is_size) {
    auto* h = static_cast<factor_handle*>(hv);
    const auto& L = h->F.L;
    const size_t n = L.rows();
    std::memcpy(colptr, L.outerIndexPtr(), sizeof(uint32_t) * (n + 1));
    std::memcpy(rowidx, L.innerIndexPtr(), sizeof(uint32_t) * L.nonZeros());
    std::memcpy(vals, L.valuePtr(), sizeof(float) * L.nonZeros());
    std::memcpy(perm, h->F.perm.data(), sizeof(uint32_t) * n);
    for (size_t r = 0; r < h->F.rounds.size(); ++r) round_is_size[r] = h->F.rounds[r].is_size;
    return 0;
}

void apxref_factor_free(void* hv) { delete static_cast<factor_handle*>(hv); }

}  // extern "C"
