// Launch interfaces of the solve-phase kernels (implemented in sweep.cu and pcg.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "device.cuh"

namespace apxb {

// Work-claim counters of one persistent sweep launch; the last warp to leave
// resets both, so a launch always starts from zero.
struct sweep_ctl {
    unsigned ticket;
    unsigned done;
};

// One sync-free sweep over a prepared direction of the factor (forward:
// L y = x over CSR(L11); backward: L^T z = y over CSC(L11)), driven by the
// direction's plan (host_prep.hpp, sweep_plan).
// `out` must hold the not-yet-solved marker in rows [0, m) on entry; the
// kernel writes the marker into `reset` (when given) at every row it solves,
// which re-arms the buffer the other direction writes next.
template <class T>
struct sweep_args {
    uint32_t m;
    uint32_t n_items;                 // work items of the plan
    const uint32_t* info;             // per item: count | log2(G) << 8 | thin << 16
    const uint32_t* ord;              // per position (32 per item): row or ~0
    const uint32_t* ptr;              // per position: entry range in idx / val (diagonal last)
    const uint32_t* idx;
    const float* val;
    // serial segment (see sweep_plan): rows [seg_first, seg_first + seg_rows)
    uint32_t seg_first, seg_rows, seg_levels;
    const uint32_t* seg_row;
    const uint32_t* seg_lvl;
    const uint32_t* seg_ptr;
    const uint32_t* seg_idx;
    const float* seg_val;
    const T* in;                      // right-hand side, row-major [row][k]
    const double* rhs_sub;            // nullable: device scalar(s) subtracted from every rhs
    T* out;                           // tracked solution [row][k]
    T* reset;                         // nullable: re-armed at every solved row
    T* copy_out;                      // nullable: untracked copy of the solution
    sweep_ctl* ctl;
    dev_error* err;
    const int* skip;                  // nullable: the launch is a no-op when *skip != 0
    unsigned long long budget_ns;     // spin budget of every wait
    int k;                            // right-hand sides per row (fp32 multi-RHS sweep)
    // batch plans (host_prep.hpp, build_batch_plan): claim units over the items
    const uint32_t* chunk;            // chunk c = items [chunk[c], chunk[c + 1])
    uint32_t n_chunks;
    // fp16 factor storage (fp32 sweeps only; prepared_factor::fp16): entry
    // weights are the binary16 values val16 (val is not read), a row's
    // diagonal is diag16[row] (its plan slot is not read), and, when
    // in_scale2 is given, the fp32 right-hand side is multiplied by
    // in_scale2[row] in fp64 and rounded once (the backward sweep's D^-2).
    const uint16_t* val16;
    const float* diag16;
    const double* in_scale2;
};

// fp64 sweep reproducing the reference CPU arithmetic (exact sum order).
void launch_sweep64(int dir, const sweep_args<double>& a, int grid, cudaStream_t s);
// fp32 sweep, fp32 accumulation, k in {1, 2, 4, 8, 16} right-hand sides
// (fp16-stored factors when a.val16 is set).
void launch_sweep32(int dir, const sweep_args<float>& a, int grid, cudaStream_t s);
// The same with the right-hand side read from fp64 (minus rhs_sub[s] when given).
void launch_sweep32_from64(int dir, const sweep_args<float>& a, const double* in64, int grid, cudaStream_t s);
// Batched fp32 sweep over a batch plan (column lanes, chunked claims), k in
// {1, 2, 4, 8, 16, 32, 64, 128}: a.k, a.chunk and a.n_chunks must be set; over
// binary16 plan values when a.val16 is set (a.diag16 and, backward,
// a.in_scale2 too).
void launch_sweep32_batch(int dir, const sweep_args<float>& a, int grid, cudaStream_t s);
// Resident grid (blocks) of the persistent sweeps.
int sweep_grid64(int num_sms);
int sweep_grid32(int k, int num_sms);
int sweep_grid32_batch(int k, int num_sms);
constexpr int kSweepThreads = 256;

void launch_fill64(double* p, size_t n, double v, cudaStream_t s);
void launch_fill32(float* p, size_t n, float v, cudaStream_t s);
void launch_fill_sent64(double* p, size_t n, cudaStream_t s);
void launch_fill_sent32(float* p, size_t n, cudaStream_t s);

// ---- PCG / apply kernels (pcg.cu) ----

// Device-resident PCG state (one solve); see pcg.cu for the field meanings.
struct pcg_state {
    double rz, pAp, alpha, beta, rr, rs, bnorm, rnorm, prev_check, mean_in, shift, tol, xmean;
    int iters, max_iter, done, status, center, laplacian, pmode, stag_window, center_k, pad;
    unsigned long long apply_count;
    unsigned n, m;
};

// An operator value: the fp32 copy when the operator is stored in fp32 (every
// value fp32-exact, so the widened value is the fp64 one), else the fp64 array.
__device__ __forceinline__ double op_val(const double* val, const float* valf, int64_t k) {
    return valf ? static_cast<double>(__ldg(valf + k)) : __ldg(val + k);
}

struct reduce_ws {
    double* partials;   // [grid * 4]
    unsigned* counter;  // one per reduction site
};

struct pcg_ptrs {
    // operator (permuted ordering)
    const int32_t* a_ptr; const int32_t* a_idx; const double* a_val;
    const float* a_valf;   // non-null: values stored in fp32 (a_val unused)
    const uint32_t* perm;
    // vectors, permuted ordering
    double* x; double* r; double* p; double* Ap; const double* z;
    // original-ordering input / output
    const double* b_orig; double* x_orig;
    pcg_state* st;
    dev_error* err;
    double* partials;
    unsigned* counters;   // [8]
    unsigned n;
    int grid;
    int spmv_lanes;       // 1: a thread per row (short rows), else lanes per row
    // rows longer than kLongRowPlain nonzeros: long row i is lr_row[i], its
    // chunks [lr_first[i], lr_first[i+1]) cover entries [ch_lo[c], ch_hi[c])
    const uint32_t* lr_row; const uint32_t* lr_first; const uint32_t* ch_lo; const uint32_t* ch_hi;
    unsigned n_long, n_chunks;
    double* ch_part;
};
constexpr uint32_t kLongRowPlain = 128;
constexpr uint32_t kChunkNnzPlain = 512;

void launch_pcg_init(const pcg_ptrs& p, cudaStream_t s);
void launch_pcg_zsum(const pcg_ptrs& p, cudaStream_t s);
void launch_pcg_rz(const pcg_ptrs& p, cudaStream_t s);
void launch_pcg_update_p(const pcg_ptrs& p, cudaStream_t s, unsigned long long cond_handle, int use_cond);
void launch_pcg_spmv(const pcg_ptrs& p, cudaStream_t s);
void launch_pcg_update_xr(const pcg_ptrs& p, cudaStream_t s);
void launch_pcg_finish(const pcg_ptrs& p, cudaStream_t s);

// apply in the original ordering: permute-in (with optional centring), gather-out.
struct apply_ptrs {
    const uint32_t* perm;
    const double* b;        // original ordering
    double* zp;             // permuted rhs buffer [n]
    const double* zsol;     // permuted solution (tracked buffer) [n], zsol[m] = 0 for a Laplacian
    double* z;              // original ordering output
    double* scal;           // [0] = b mean, [1] = z shift, [2] = b.z (device)
    int center;             // Laplacian centring on this application
    double* partials;
    unsigned* counters;
    unsigned n;
    int grid;
};
void launch_apply_bsum(const apply_ptrs& a, cudaStream_t s);      // scal[0] = sum(b)/n if center
void launch_apply_permute(const apply_ptrs& a, cudaStream_t s);   // zp[perm[v]] = b[v] - scal[0]
void launch_apply_zsum(const apply_ptrs& a, cudaStream_t s);      // scal[1] = sum(zsol)/n if center
void launch_apply_gather(const apply_ptrs& a, cudaStream_t s);    // z[v] = zsol[perm[v]] - scal[1]; scal[2] = b.z

// y = A x over the permuted operator with permute / unpermute (residual checks);
// values from valf when it is given (fp32 storage), else from val.
void launch_spmv_plain(const int32_t* ptr, const int32_t* idx, const double* val, const float* valf, const double* x,
                       double* y, unsigned n, int grid, cudaStream_t s);

}  // namespace apxb
