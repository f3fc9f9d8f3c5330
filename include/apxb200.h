/* apxb200 -- the apxchol solve phase on NVIDIA B200 (sm_100a), as a C ABI.
 *
 * Replaces, behind plain pointers and sizes, the reference's GPU solve-phase
 * classes and the CPU preconditioner application they back:
 *   cuda_sptrsv::setup / solve_LLt / solve_LLt_dev
 *       include/apxchol/solver/sptrsv/cuda.h:233-487
 *   apx_cholesky::apply_core / apply_fused / _solve_impl / reset_apply_count
 *       include/apxchol/solver/preconditioner.h:317, 344-529
 *   cuda_pcg::setup / solve (GPU-resident PCG)
 *       include/apxchol/solver/pcg_cuda.h:68-261
 *   cpu_solver::solve / apxchol::solve (the PCG semantics followed)
 *       src/solve.cpp:478-654, 681-737
 * The factor is the reference factorization's own output
 * (apxchol::factorization, include/apxchol/solver/factorization.h:22-56),
 * uploaded once.
 *
 * Conventions: every call returns an int status (APXB_OK = 0, negative on
 * failure) and never throws; apxb_last_error() gives the message of the last
 * failure on the calling thread. Pointers flagged as device pointers must be
 * device memory of the engine's GPU; all others are host memory. Calls on one
 * engine are not thread-safe (as the reference: solve.h:96-97).
 */
#ifndef APXB200_H
#define APXB200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define APXB_OK               0
#define APXB_ERR_INVALID     -1  /* bad argument or malformed input */
#define APXB_ERR_CUDA        -2  /* a CUDA runtime call failed */
#define APXB_ERR_OOM         -3  /* device allocation failed */
#define APXB_ERR_TIMEOUT     -4  /* a device wait ran out of its spin budget */
#define APXB_ERR_BAD_FACTOR  -5  /* factor violates the storage contract */
#define APXB_ERR_NONFINITE   -6  /* NaN / Inf met where a finite value is required */
#define APXB_ERR_BUDGET      -7  /* the engine's device-memory budget is exhausted */
#define APXB_ERR_BUSY        -8  /* no free slot (serving) */

/* ---- sweep precisions ---- */
#define APXB_PREC_FP64  0  /* fp32-stored factor, fp64 sweeps: the reference's CPU arithmetic */
#define APXB_PREC_FP32  1  /* fp32 factor and sweeps, fp32 accumulation (mixed precision) */
#define APXB_PREC_FP16  2  /* fp16 per-column-scaled factor storage, fp32 sweeps: the reference GPU
                            * backend's default storage (cuda_sptrsv with APXCHOL_SPTRSV_FP16,
                            * cuda.h:131-163); 6 instead of 8 bytes per stored entry */

/* ---- apply flags ---- */
#define APXB_DEVICE_PTRS      1  /* b / z are device pointers */
#define APXB_CENTER_SCHEDULE  0  /* Laplacian centring per the center-k counter (default) */
#define APXB_CENTER_ALWAYS    2
#define APXB_CENTER_NEVER     4
#define APXB_TRUE_RESIDUAL    8  /* batch solve: recompute ||b - A x|| / ||b|| per slot in fp64 */

typedef struct apxb_engine apxb_engine;
typedef struct apxb_factor apxb_factor;
typedef struct apxb_operator apxb_operator;
typedef struct apxb_batch apxb_batch;

typedef struct apxb_factor_info {
    uint32_t n;              /* operator dimension */
    uint32_t m;              /* factor dimension: n (SDDM) or n-1 (Laplacian) */
    uint64_t nnz_factor;     /* nnz of L11 before the drop */
    uint64_t nnz_stored;     /* nnz each sweep direction stores (after the drop) */
    uint64_t dropped;        /* off-diagonals removed by the drop */
    int32_t  fwd_levels;     /* level count of each direction (row sum modes) */
    int32_t  bck_levels;
    int32_t  precision;      /* APXB_PREC_* */
    int32_t  sddm;
    uint64_t device_bytes;   /* device memory held by the factor */
    uint64_t apply_count;    /* center-k application counter */
    double   drop_rel;       /* drop threshold in effect (factor_drop.h: rel) */
    uint64_t dropped_flush;  /* of `dropped`: off-diagonals fp16 storage would store as zero */
    int32_t  sweep_grid;     /* blocks of the resident sweep grid of this factor's sweeps */
    int32_t  reserved;
} apxb_factor_info;

typedef struct apxb_pcg_result {
    int32_t  iterations;
    int32_t  status;         /* 0 converged, 1 max_iter, 2 stagnated, 3 pAp <= 0, 4 non-finite */
    double   residual;       /* recurrence relative residual sqrt(r.r)/||b|| at exit */
    double   true_residual;  /* ||b - A x|| / ||b|| recomputed in fp64 (when requested) */
    double   seconds;        /* device time of the solve (CUDA events) */
} apxb_pcg_result;

const char* apxb_last_error(void);
const char* apxb_version(void);

/* ---- engine: one GPU, one stream, an error word and workspaces ----
 * device: a CUDA device index, or APXB_CURRENT_DEVICE for the calling
 * thread's current device (where the reference's classes run). */
#define APXB_CURRENT_DEVICE (-1)
int apxb_engine_create(int device, apxb_engine** out);
/* With factors or operators still alive the engine is only marked closed; the
 * last of them to be destroyed releases it. */
int apxb_engine_destroy(apxb_engine* e);
int apxb_engine_sync(apxb_engine* e);
/* The engine's CUDA stream (cudaStream_t), for callers that order their own work around it. */
void* apxb_engine_stream(apxb_engine* e);
/* Spin budget of every device wait, in nanoseconds (default 2e9). */
int apxb_engine_set_spin_budget(apxb_engine* e, uint64_t ns);
/* Blocks of the persistent sweep launches (0 = the resident grid). Any value
 * gives the same bytes; tests use it to show the result is schedule-free.
 * Batches read it when they are created. */
int apxb_engine_set_sweep_grid(apxb_engine* e, int blocks);
/* Device-memory budget for factors and operators created on this engine (0 = unlimited). */
int apxb_engine_set_memory_budget(apxb_engine* e, uint64_t bytes);
uint64_t apxb_engine_memory_used(apxb_engine* e);

/* ---- factor (replaces cuda_sptrsv::setup, cuda.h:233-459) ----
 * colptr[n+1], rowidx[nnz], vals[nnz]: the factor CSC, each column starting
 * with its diagonal, rows ascending (u32 / f32). perm[n]: perm[v] = position.
 * sddm: full-rank (m = n) vs Laplacian (m = n-1, row/column n-1 dropped).
 * rounds[n_rounds]: per-round independent-set sizes (factorization.h:43-51);
 * they fix the sum order of each row exactly as the reference CPU sweep
 * (n_rounds = 0 uses topological levels, as the reference without rounds).
 * drop_rel: compacting drop threshold (< 0 = the reference default 1e-4,
 * 0 = off). precision: APXB_PREC_*. */
int apxb_factor_create(apxb_engine* e, uint32_t n, const uint32_t* colptr, const uint32_t* rowidx,
                       const float* vals, const uint32_t* perm, int sddm,
                       const uint64_t* rounds, uint32_t n_rounds, double drop_rel, int precision,
                       apxb_factor** out);
int apxb_factor_destroy(apxb_factor* f);
int apxb_factor_info_get(const apxb_factor* f, apxb_factor_info* info);
/* Host copies of the prepared sweep arrays (CSR(L11), CSC(L11)); any pointer may be NULL. */
int apxb_factor_arrays(const apxb_factor* f, uint32_t* csr_ptr, uint32_t* csr_idx, float* csr_val,
                       uint32_t* csc_ptr, uint32_t* csc_idx, float* csc_val,
                       uint8_t* fwd_thin, uint8_t* bck_thin);
/* apx_cholesky::reset_apply_count (preconditioner.h:317). */
int apxb_factor_reset_apply_count(apxb_factor* f);
/* Host-only preparation (no GPU): the arrays apxb_factor_create would upload.
 * Call once with NULL arrays to get *m and *nnz_stored, then with buffers of
 * m+1 / nnz_stored / m entries. levels[2] receives the level counts. */
int apxb_prepare_host(uint32_t n, const uint32_t* colptr, const uint32_t* rowidx, const float* vals,
                      const uint32_t* perm, int sddm, const uint64_t* rounds, uint32_t n_rounds,
                      double drop_rel, uint32_t* m, uint64_t* nnz_stored, int32_t* levels,
                      uint32_t* csr_ptr, uint32_t* csr_idx, float* csr_val,
                      uint32_t* csc_ptr, uint32_t* csc_idx, float* csc_val,
                      uint8_t* fwd_thin, uint8_t* bck_thin);

/* Host-only fp16 storage (no GPU): what apxb_factor_create(..., APXB_PREC_FP16)
 * uploads. Replaces the reference GPU backend's host preparation with fp16
 * storage: cuda_host::apply_factor_drop with the fp16 keep predicate and
 * cuda_host::narrow_fp16_scaled (cuda_host.h:120-232), after the scale
 * fallback of cuda_sptrsv::setup (cuda.h:287-301). Call once with NULL arrays
 * for *m and *nnz_stored. csc_*: CSC(L11) = CSR(L11^T) with binary16 values;
 * csr_*: CSR(L11) carrying the same bit patterns; diag[m] = fp32 L_jj / s_j
 * plus the column's rounding residual; inv_scale[m] = fp32 1 / s_j;
 * stats[3] = {dropped, dropped only because fp16 flushes them, stored
 * off-diagonals flushed to zero}. */
int apxb_prepare_host_fp16(uint32_t n, const uint32_t* colptr, const uint32_t* rowidx, const float* vals,
                           const uint32_t* perm, int sddm, const uint64_t* rounds, uint32_t n_rounds,
                           double drop_rel, uint32_t* m, uint64_t* nnz_stored,
                           uint32_t* csc_ptr, uint32_t* csc_idx, uint16_t* csc_val16,
                           uint32_t* csr_ptr, uint32_t* csr_idx, uint16_t* csr_val16,
                           float* diag, float* inv_scale, uint64_t* stats);

/* ---- sweeps, permuted space, m entries (cuda_sptrsv::solve_LLt_dev, cuda.h:480-487) ---- */
/* dir 0: forward L y = x; dir 1: backward L^T z = y. Device pointers; fp64.
 * fp32 / fp16 factors sweep in fp32 (input narrowed, output widened); an fp16
 * factor's sweeps are those of the stored, column-scaled factor: the forward
 * returns D y and the backward reads its input times D^-2 (D = diag(s_j)), so
 * only the pair applies (L L^T)^-1. */
int apxb_sweep(apxb_engine* e, apxb_factor* f, int dir, const double* d_in, double* d_out);
/* Both sweeps: out = (L L^T)^-1 in. Device pointers (in and out may alias). */
int apxb_sweep_pair(apxb_engine* e, apxb_factor* f, const double* d_in, double* d_out);
/* apxb_sweep_pair without any device allocation in the call. No counterpart
 * in the reference. For callers that cannot allocate device memory when they
 * apply the preconditioner: hosts that reserve the GPU's memory for their own
 * pool and forbid allocations outside it, and latency-bound loops that cannot
 * take the device-wide synchronisation cudaMalloc / cudaFree may cause.
 * Same result as apxb_sweep_pair, bit for bit. The intermediate vectors live in
 * one fixed array of device memory owned by the library, 1 MiB + 256 B on every
 * GPU that loads it, held until the process exits; so the factor's m must be
 * at most 65,536 (larger: APXB_ERR_INVALID, with the limit in the message),
 * and the factor must be fp64. The engine and the factor are created (and
 * allocate) beforehand. The first call on a device looks up the array's
 * device address on it: make that first call before any stream capture.
 * That address is kept for the life of the process; after cudaDeviceReset it
 * is stale, so do not call this on a device that has been reset. Every call
 * returns after the engine stream has finished its sweeps (it reads the
 * engine's error word).
 * Every call re-arms the array, but all calls on one device share it: calls
 * whose work overlaps on the GPU (other engines' streams, other host threads)
 * race and corrupt each other's results. */
int apxb_sweep_pair_noalloc(apxb_engine* e, apxb_factor* f, const double* d_in, double* d_out);
/* The same with host pointers (cuda_sptrsv::solve_LLt, cuda.h:464-473). */
int apxb_sweep_pair_host(apxb_engine* e, apxb_factor* f, const double* in, double* out);
/* reps back-to-back pairs on the engine stream, timed with CUDA events; *seconds = per pair. */
int apxb_sweep_pair_timed(apxb_engine* e, apxb_factor* f, const double* d_in, double* d_out, int reps,
                          double* seconds);
/* k right-hand sides at once, row-interleaved in[i*k + s] (device pointers).
 * The sweeps are fp32 (fp16-stored factors: over their binary16 values)
 * whatever the factor's precision; k in {1, 2, 4, 8, 16}. */
int apxb_sweep_pair_multi(apxb_engine* e, apxb_factor* f, int k, const double* d_in, double* d_out);

/* ---- preconditioner application in the original ordering (apply_core) ----
 * z = P^T (L L^T)^-1 P (b - mean) (- mean), see preconditioner.h:403-529.
 * flags: APXB_DEVICE_PTRS | APXB_CENTER_*; rz_out (may be NULL) receives b.z. */
int apxb_apply(apxb_engine* e, apxb_factor* f, const double* b, double* z, int flags, double* rz_out);

/* ---- the reference's raw dataflow sweep (cuda_dataflow.h:160-208) ----
 * apxchol::dataflow_solve / dataflow_solve_fp16 / dataflow_grid_size /
 * dataflow_prefetch_depth are C++ functions of this library, declared by the
 * replacement header apxchol/solver/sptrsv/cuda_dataflow.h (include/apxchol_compat).
 * They report nothing themselves (the reference's return void): a launch whose
 * wait made no progress for one second (a plan or epoch that breaks the
 * contract) stops and records it, once per device. apxb_dataflow_status
 * returns the current device's record (APXB_ERR_TIMEOUT or APXB_ERR_INVALID
 * with apxb_last_error set, else APXB_OK) and clears it; it synchronizes with
 * that device. */
int apxb_dataflow_status(void);

/* ---- operator: A in the factor's permuted ordering (cuda_pcg::setup, pcg_cuda.h:68-152) ----
 * colptr[n+1], rowidx[nnz], vals[nnz]: full symmetric CSC (int32, rows ascending).
 * Values are stored in fp32 when every one round-trips fp32 (v == (double)(float)v),
 * else in fp64 (the reference's rule, pcg_cuda.h:100-111); the SpMV widens each
 * value to fp64, so an fp32-stored exact operator gives the same results. The
 * environment variable APXCHOL_GPU_FP32_OPERATOR, read at creation, overrides:
 * "0" keeps fp64, any other non-empty value forces fp32 (values rounded). */
int apxb_operator_create(apxb_engine* e, uint32_t n, const int32_t* colptr, const int32_t* rowidx,
                         const double* vals, const uint32_t* perm, apxb_operator** out);
int apxb_operator_destroy(apxb_operator* a);
/* *fp32 = 1 when the operator's values are stored in fp32, else 0
 * (cuda_pcg::fp32_operator, pcg_cuda.h:267). */
int apxb_operator_fp32(const apxb_operator* a, int* fp32);
/* y = A x in the original ordering (host pointers), for residual checks. */
int apxb_operator_matvec(apxb_engine* e, apxb_operator* a, const double* x, double* y);

/* ---- GPU-resident PCG (apxchol::solve on the device; cpu_solver semantics) ----
 * b, x in the original ordering; host pointers unless APXB_DEVICE_PTRS.
 * The stop rule, stagnation window (50) and center-k schedule follow
 * src/solve.cpp:478-654. want_true_residual: recompute ||b - A x||/||b||. */
int apxb_pcg(apxb_engine* e, apxb_factor* f, apxb_operator* a, const double* b, double* x,
             double tol, int max_iter, int flags, int want_true_residual, apxb_pcg_result* res);

/* ---- batched solves: mixed precision, many right-hand sides, uneven instances ----
 * A batch binds S instances (factor + operator pairs of any sizes, solved as
 * one block-diagonal system in a single set of launches) and k right-hand-side
 * slots per instance (k = 1, 2, 4, 8, 16, 32, 64 or 128). The preconditioner runs fp32
 * sweeps with fp32 accumulation; SpMV, residuals, dots and centring are fp64.
 * Each slot is an independent PCG with the semantics of apxb_pcg. No
 * counterpart in the reference (its GPU PCG solves one right-hand side). */
int apxb_batch_create(apxb_engine* e, int n_inst, apxb_factor* const* factors, apxb_operator* const* ops, int k,
                      apxb_batch** out);
int apxb_batch_destroy(apxb_batch* b);
int apxb_batch_size(const apxb_batch* b, int* n_inst, int* k, uint32_t* n_total);
/* B, X: for instance i (row offset off_i, size n_i, original ordering) and
 * column c, entries at [k * off_i + c * n_i, ... + n_i). nrhs[i] (NULL = all
 * k) columns of instance i are used; the others return x = 0. res receives
 * one result per slot (instance-major). flags: APXB_DEVICE_PTRS,
 * APXB_TRUE_RESIDUAL. */
int apxb_batch_solve(apxb_batch* b, const double* B, double* X, const int* nrhs, double tol, int max_iter,
                     int flags, apxb_pcg_result* res);
/* Periodic true-residual refresh (fp64): every `every` iterations of a slot
 * (its own count, so a slot's arithmetic does not depend on the other
 * slots) its residual is recomputed as b - A x before the x/r update, which
 * keeps the fp64 recurrence from drifting away from the true residual. The
 * same refresh confirms convergence: a slot whose recurrence residual drops
 * below its tolerance in an iteration that did not start with a refresh runs
 * one more iteration that does, and stops only if the residual taken from the
 * recomputed b - A x is below its tolerance (so a converged slot's fp64
 * relative residual ||b - A x|| / ||b|| meets its tolerance, up to the rounding
 * of one update). At max_iter the recurrence alone decides. Default 25; 0 turns
 * off both (the stop then follows the recurrence, as apxb_pcg). Only while no
 * slot is admitted (else APXB_ERR_BUSY). */
int apxb_batch_set_refresh(apxb_batch* b, int every);

/* Host-only (no GPU): builds and checks the batch sweep plans apxb_batch_create
 * would build for this factor and k (column lanes, oldest-dependency-first
 * entries, chunked claims); n_items[2] / n_chunks[2] receive their sizes per
 * direction. */
int apxb_batch_plan_host(uint32_t n, const uint32_t* colptr, const uint32_t* rowidx, const float* vals,
                         const uint32_t* perm, int sddm, const uint64_t* rounds, uint32_t n_rounds, double drop_rel,
                         int k, uint32_t* n_items, uint32_t* n_chunks);

/* ---- continuous batching (the serving form; no counterpart in the reference) ----
 * Slots are admitted and retired one at a time while the other slots keep
 * iterating. Slot s belongs to instance s / k; a new batch has every slot idle.
 * Every call below only enqueues work on the engine stream, in call order, and
 * returns without waiting, so the host can keep iterations queued while it
 * admits and retires slots.
 *  admit:   load rhs (the instance's n values, original ordering) into an idle
 *           slot, with its own tolerance; the slot joins at the next iteration
 *           enqueued after the call. Pageable host memory is staged before the
 *           call returns; pinned host or device memory is read later, in stream
 *           order, and must stay unchanged until then. max_iter can change
 *           only while no slot is admitted (else APXB_ERR_BUSY).
 *  step:    enqueue `iterations` iterations of every live slot, then a copy of
 *           the slot states; *step_id names the step.
 *  query:   *ready = 1 once step step_id has finished (non-blocking).
 *  slots:   the slot states after step step_id (waits for it): done (finished
 *           and not re-admitted since), iterations, status (as
 *           apxb_pcg_result.status) and recurrence residual; any pointer may be
 *           NULL. The states of a step stay readable until two later steps are
 *           enqueued (the library keeps two copies).
 *  retire:  enqueue the copy of a finished slot's x (original ordering;
 *           Laplacian instances centred) to x; the slot is idle at once and can
 *           be admitted again (the new right-hand side is ordered after the copy).
 *  retired: *ready = 1 once the last retire of that slot has written x.
 * A slot's arithmetic does not depend on the other slots, so a right-hand side
 * gives the same bits alone and in any mix. apxb_batch_solve refuses while
 * slots are admitted. */
int apxb_batch_admit(apxb_batch* b, int slot, const double* rhs, double tol, int max_iter, int flags);
int apxb_batch_step(apxb_batch* b, int iterations, int64_t* step_id);
int apxb_batch_query(apxb_batch* b, int64_t step_id, int* ready);
int apxb_batch_slots(const apxb_batch* b, int64_t step_id, int* done, int* iterations, int* status, double* residual);
int apxb_batch_retire(apxb_batch* b, int slot, double* x, int flags);
int apxb_batch_retired(apxb_batch* b, int slot, int* ready);
/* Times the batch's forward and backward fp32 sweeps (all k columns) on the
 * right-hand sides of its last iteration: seconds per sweep, mean of reps. */
int apxb_batch_sweep_timed(apxb_batch* b, int reps, double* fwd_seconds, double* bck_seconds);

/* ---- failure detection test hook ----
 * Runs one forward sweep whose first 32 rows are never solved (the work
 * counter starts past them), so every row that depends on them waits on a
 * value nothing writes. Each wait gives up after budget_ns, the kernel records
 * APXB_ERR_TIMEOUT and drains; the call returns that status and leaves the
 * engine usable. Used by the tests to show a stalled wait ends in an error,
 * not a hang. */
int apxb_test_stalled_sweep(apxb_engine* e, apxb_factor* f, uint64_t budget_ns);

/* ---- device preparation test hook ----
 * apxb_factor_create prepares factors with round sizes and fp32 / fp64
 * storage on the device (the reference does this work on the host:
 * cuda.h:280-420, cuda_host.h:66-558). This hook prepares the given factor
 * both ways and compares every array: CSC(L11) and CSR(L11) after the drop,
 * levels, row sum modes, both directions' sweep plans, the batch plans for
 * k right-hand sides (k > 0) and, when the operator is given (full symmetric
 * CSC, int32), its permutation P A P^T (pcg_cuda.h:304-404). APXB_OK when
 * all are identical (or both preparations reject the input with the same
 * message); else APXB_ERR_INVALID naming the first array that differs. */
int apxb_test_prep_compare(apxb_engine* e, uint32_t n, const uint32_t* colptr, const uint32_t* rowidx,
                           const float* vals, const uint32_t* perm, int sddm, const uint64_t* rounds,
                           uint32_t n_rounds, double drop_rel, int k, const int32_t* a_colptr,
                           const int32_t* a_rowidx, const double* a_vals);

#ifdef __cplusplus
}
#endif
#endif
