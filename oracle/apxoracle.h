/* TEST INFRASTRUCTURE (oracle). Plain-C restatement of the apxchol reference's
 * CPU solve phase, used only by the tests, smoke() and the CPU-baseline leg of
 * bench.py to check the CUDA product. Nothing in the product links it.
 *
 * Parity pin: the tests check every function here byte-for-byte against the
 * reference itself compiled from its sources (oracle/_ref/libapxref.so).
 *
 * Arithmetic: every product and sum is rounded on its own (built with
 * -ffp-contract=off), the order of every sum follows the cited reference line,
 * and reductions reproduce the reference's OpenMP static-chunk partials for a
 * given team size `nt` (preconditioner.h:61-125).
 */
#ifndef APXORACLE_H
#define APXORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Host prep: L11 extraction, compacting drop, CSC->CSR transpose.
 * (sptrsv/omp.h:505-805, factor_drop.h:90-211, transpose.h:116-246)
 * Inputs: the factor CSC (n columns, u32 / f32), m = n or n-1, drop rel.
 * Outputs (caller-allocated with nnz(L) capacity): CSR(L11) and CSC(L11).
 * Returns nnz_stored, or -1 on a malformed factor. */
int64_t ora_prepare(uint32_t n, uint32_t m, const uint32_t* colptr, const uint32_t* rowidx,
                    const float* vals, double rel,
                    uint32_t* csr_ptr, uint32_t* csr_idx, float* csr_val,
                    uint32_t* csc_ptr, uint32_t* csc_idx, float* csc_val);

/* Level of every row in each sweep direction (sptrsv/omp.h:865-975): from the
 * per-round IS sizes when n_rounds > 0 (round-as-level), else the topological
 * depth. Writes fwd_level[m], bck_level[m]; returns the number of levels
 * (forward, and via *n_bck backward). */
int32_t ora_levels(uint32_t m, const uint32_t* csr_ptr, const uint32_t* csr_idx,
                   const uint32_t* csc_ptr, const uint32_t* csc_idx,
                   const uint64_t* rounds, uint32_t n_rounds,
                   int32_t* fwd_level, int32_t* bck_level, int32_t* n_bck);

/* Per-row sum mode: 1 = "thin" level (4-way split sum, omp.h:1343-1357), 0 =
 * "fat" level (single serial sum, omp.h:1434-1439). threshold = 1024
 * (kSpTRSVOMPThreshold, omp.h:32). */
void ora_thin_flags(uint32_t m, const int32_t* level, int32_t n_levels, uint32_t threshold,
                    uint8_t* thin);

/* One sweep (omp.h:1094-1119, 1425-1445). dir 0: forward on CSR(L11),
 * diagonal last; dir 1: backward on CSC(L11), diagonal first. */
void ora_sweep(int dir, uint32_t m, const uint32_t* ptr, const uint32_t* idx, const float* val,
               const uint8_t* thin, const double* in, double* out);

/* One sweep over an fp16-stored factor, in fp64: the reference test's
 * independent host sweep (tests/test_sptrsv_drop.cpp:1100-1127) over the
 * storage of cuda_host.h:16-34. Rows in order (dir 0, CSR(L11)) or in reverse
 * (dir 1, CSC(L11)); out[i] = (rhs[i] * (in_scale ? in_scale[i] : 1)
 * - sum_{j != i} value(val16[p]) * out[j]) / diag[i], the sum in storage order. */
void ora_sweep16(int dir, uint32_t m, const uint32_t* ptr, const uint32_t* idx, const uint16_t* val16,
                 const float* diag, const double* in_scale, const double* rhs, double* out);

typedef struct ora_system {
    /* operator: full symmetric CSR (== CSC for a symmetric matrix), int32 */
    uint32_t n;
    const int32_t* a_ptr;
    const int32_t* a_idx;
    const double* a_val;
    /* preconditioner */
    uint32_t m;
    int32_t sddm;
    const uint32_t* perm;
    const uint32_t* csr_ptr; const uint32_t* csr_idx; const float* csr_val;
    const uint32_t* csc_ptr; const uint32_t* csc_idx; const float* csc_val;
    const uint8_t* fwd_thin; const uint8_t* bck_thin;
    /* reduction team size and the center-k period (env_knobs.h:72-73) */
    int32_t nt;
    int32_t center_k;
    /* center-k application counter (preconditioner.h:393-397) */
    uint64_t apply_count;
} ora_system;

/* apx_cholesky::apply_core (preconditioner.h:403-529). `center` decided by the
 * caller. Returns b.z when want_rz. */
double ora_apply_core(ora_system* s, const double* b, double b_sum, int center, double* z, int want_rz);
/* apply_fused (preconditioner.h:370-377): advances the center-k counter. */
double ora_apply_fused(ora_system* s, const double* r, double r_sum, double* z);
/* _solve_impl (preconditioner.h:344-353): the Eigen-seam application. */
void ora_apply(ora_system* s, const double* b, double* z);

/* cpu_solver::solve_impl from x0 = 0 (src/solve.cpp:478-654): stagnation
 * window 50. Returns 0. */
int ora_pcg(ora_system* s, const double* b, double tol, int max_iter, double* x,
            int* iters, double* residual);

#ifdef __cplusplus
}
#endif
#endif
