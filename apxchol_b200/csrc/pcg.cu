// GPU-resident PCG and the preconditioner application's vector passes.
//
// The loop follows the reference CPU solver's semantics
// (cpu_solver::solve_impl, src/solve.cpp:478-654): stop when
// sqrt(r.r)/||b|| < tol right after the x/r update, break on p.Ap <= 0, a
// stagnation check every 50 iterations, center-k centring of the
// preconditioner's input and output on every K-th application of a Laplacian
// solve (preconditioner.h:393-397, 488-524), and the min-norm centring of x at
// the end (solve.cpp:265-269, 631-634). It runs in the factor's permuted
// ordering (like the reference's cuda_pcg, pcg_cuda.h:157-261), so the
// preconditioner is the two sweeps alone; b is permuted in once and x
// unpermuted once.
//
// Every scalar (p.Ap, alpha, r.r, beta, ...) is produced on the device by the
// last block of the kernel that reduces it, from per-block partials summed in
// block order over a fixed grid: results are bit-identical run to run, and no
// scalar crosses to the host inside the loop. Kernels read `done` first and
// return, so an iteration launched after convergence does nothing.
#include "kernels.cuh"

namespace apxb {

namespace {

constexpr int kThreads = 256;
enum counter_slot { kCInit = 0, kCZsum, kCRz, kCSpmv, kCXr, kCXsum, kCApply0, kCApply1 };

__device__ __forceinline__ bool stopped(const pcg_state* st, const dev_error* err) {
    return st->done != 0 || err->code != 0;
}

__global__ void __launch_bounds__(kThreads) k_pcg_init(pcg_ptrs p) {
    pcg_state* st = p.st;
    double v[2] = {0.0, 0.0};
    const unsigned n = p.n;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double bi = p.b_orig[i];
        p.r[p.perm[i]] = bi;
        p.x[i] = 0.0;
        v[0] = fma(bi, bi, v[0]);
        v[1] += bi;
    }
    double tot[2];
    if (grid_sum<2>(v, p.partials, p.counters + kCInit, tot)) {
        st->rr = tot[0];
        st->rs = tot[1];
        st->bnorm = sqrt(tot[0]);
        st->iters = 0;
        st->rnorm = 1.0;
        st->prev_check = 1.0;
        st->status = 1;
        st->done = 0;
        st->shift = 0.0;
        st->pmode = 1;
        st->xmean = 0.0;
        if (st->bnorm == 0.0) {
            st->done = 1;
            st->status = 0;
            st->rnorm = 0.0;
        } else {
            st->apply_count = 1;
            st->center = st->laplacian && (1ull % static_cast<unsigned long long>(st->center_k)) == 0;
            st->mean_in = st->center ? tot[1] / static_cast<double>(n) : 0.0;
        }
    }
}

// shift = mean(z) on a centring application (z[m] = 0 for a Laplacian).
__global__ void __launch_bounds__(kThreads) k_pcg_zsum(pcg_ptrs p) {
    pcg_state* st = p.st;
    if (stopped(st, p.err) || !st->center) return;
    double v[1] = {0.0};
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x) v[0] += p.z[i];
    double tot[1];
    if (grid_sum<1>(v, p.partials, p.counters + kCZsum, tot)) st->shift = tot[0] / static_cast<double>(p.n);
}

// rz = r.(z - shift); beta = rz_new / rz (preconditioner.h:423-447 fused dot, solve.cpp:620-629).
__global__ void __launch_bounds__(kThreads) k_pcg_rz(pcg_ptrs p) {
    pcg_state* st = p.st;
    if (stopped(st, p.err)) return;
    const double shift = st->shift;
    double v[1] = {0.0};
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x)
        v[0] = fma(p.r[i], p.z[i] - shift, v[0]);
    double tot[1];
    if (grid_sum<1>(v, p.partials, p.counters + kCRz, tot)) {
        if (st->pmode == 1) {
            st->beta = 0.0;
        } else {
            st->beta = tot[0] / st->rz;
        }
        st->rz = tot[0];
    }
}

// p = (z - shift) + beta p (first application: p = z - shift). Sets the while
// condition of a graph-resident loop.
__global__ void __launch_bounds__(kThreads) k_pcg_update_p(pcg_ptrs p, unsigned long long handle, int use_cond) {
    pcg_state* st = p.st;
    if (use_cond && blockIdx.x == 0 && threadIdx.x == 0)
        cudaGraphSetConditional(static_cast<cudaGraphConditionalHandle>(handle), stopped(st, p.err) ? 0u : 1u);
    if (stopped(st, p.err)) return;
    const double shift = st->shift, beta = st->beta;
    const bool copy = st->pmode == 1;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x) {
        const double zi = p.z[i] - shift;
        p.p[i] = copy ? zi : fma(beta, p.p[i], zi);
    }
}

// Ap = A p with p.Ap fused (src/solve.cpp:122-161). G lanes per row, lanes
// stride the row's entries, fixed xor-butterfly inside the group.
template <int G>
__global__ void __launch_bounds__(kThreads) k_pcg_spmv(pcg_ptrs p) {
    pcg_state* st = p.st;
    if (stopped(st, p.err)) return;
    constexpr unsigned kRowsPerWarp = 32 / G;
    const unsigned lane = threadIdx.x & (G - 1);
    const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
    double v[1] = {0.0};
    // Warp-uniform trip count: every lane reaches the shuffles.
    for (unsigned base = warp * kRowsPerWarp; base < p.n; base += nwarps * kRowsPerWarp) {
        const unsigned row = base + ((threadIdx.x & 31) / G);
        double s = 0.0;
        bool is_long = false;
        if (row < p.n) {
            const int b = __ldg(p.a_ptr + row), e = __ldg(p.a_ptr + row + 1);
            is_long = static_cast<uint32_t>(e - b) > kLongRowPlain;   // summed by the chunk kernels
            if (!is_long)
                for (int k = b + static_cast<int>(lane); k < e; k += G)
                    s = fma(op_val(p.a_val, p.a_valf, k), p.p[__ldg(p.a_idx + k)], s);
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o, G);
        if (lane == 0 && row < p.n) {
            if (is_long) s = p.Ap[row];
            else p.Ap[row] = s;
            v[0] = fma(p.p[row], s, v[0]);
        }
    }
    double tot[1];
    if (grid_sum<1>(v, p.partials, p.counters + kCSpmv, tot)) {
        st->pAp = tot[0];
        st->pmode = 0;
        if (tot[0] <= 0.0) {
            st->done = 1;
            st->status = 3;
        } else {
            st->alpha = st->rz / tot[0];
        }
    }
}

// The same for short rows: a thread per row, the row's entries summed in CSR
// order, their gathers issued 8 at a time.
__global__ void __launch_bounds__(kThreads) k_pcg_spmv_rows(pcg_ptrs p) {
    pcg_state* st = p.st;
    if (stopped(st, p.err)) return;
    constexpr int kE = 8;
    double v[1] = {0.0};
    for (unsigned row = blockIdx.x * blockDim.x + threadIdx.x; row < p.n; row += gridDim.x * blockDim.x) {
        const int b = __ldg(p.a_ptr + row), e = __ldg(p.a_ptr + row + 1);
        if (static_cast<uint32_t>(e - b) > kLongRowPlain) {   // summed by the chunk kernels
            v[0] = fma(p.p[row], p.Ap[row], v[0]);
            continue;
        }
        double s = 0.0, own = 0.0;
        bool have_own = false;
        for (int k0 = b; k0 < e; k0 += kE) {
            int col[kE];
            double w[kE], x[kE];
#pragma unroll
            for (int j = 0; j < kE; ++j)
                if (k0 + j < e) { col[j] = __ldg(p.a_idx + k0 + j); w[j] = op_val(p.a_val, p.a_valf, k0 + j); }
#pragma unroll
            for (int j = 0; j < kE; ++j)
                if (k0 + j < e) x[j] = p.p[col[j]];
#pragma unroll
            for (int j = 0; j < kE; ++j)
                if (k0 + j < e) {
                    s = fma(w[j], x[j], s);
                    if (col[j] == static_cast<int>(row)) { own = x[j]; have_own = true; }
                }
        }
        p.Ap[row] = s;
        if (!have_own) own = p.p[row];
        v[0] = fma(own, s, v[0]);
    }
    double tot[1];
    if (grid_sum<1>(v, p.partials, p.counters + kCSpmv, tot)) {
        st->pAp = tot[0];
        st->pmode = 0;
        if (tot[0] <= 0.0) {
            st->done = 1;
            st->status = 3;
        } else {
            st->alpha = st->rz / tot[0];
        }
    }
}

// x += alpha p; r -= alpha Ap; r.r and sum(r) (src/solve.cpp:169-208), then
// the stop rules (solve.cpp:600-615) and the next application's centring.
__global__ void __launch_bounds__(kThreads) k_pcg_update_xr(pcg_ptrs p) {
    pcg_state* st = p.st;
    if (stopped(st, p.err)) return;
    const double alpha = st->alpha;
    double v[2] = {0.0, 0.0};
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x) {
        p.x[i] = fma(alpha, p.p[i], p.x[i]);
        const double ri = fma(-alpha, p.Ap[i], p.r[i]);
        p.r[i] = ri;
        v[0] = fma(ri, ri, v[0]);
        v[1] += ri;
    }
    double tot[2];
    if (grid_sum<2>(v, p.partials, p.counters + kCXr, tot)) {
        st->rr = tot[0];
        st->rs = tot[1];
        const double rnorm = sqrt(tot[0]) / st->bnorm;
        st->rnorm = rnorm;
        st->iters += 1;
        int done = 0, status = 1;
        if (rnorm < st->tol) { done = 1; status = 0; }
        else if (!isfinite(rnorm)) { done = 1; status = 4; }
        else if (st->stag_window > 0 && st->iters % st->stag_window == 0) {
            if (rnorm > st->prev_check * 0.5) { done = 1; status = 2; }
            else st->prev_check = rnorm;
        }
        if (!done && st->iters >= st->max_iter) { done = 1; status = 1; }
        st->status = status;
        st->done = done;
        if (!done) {
            st->apply_count += 1;
            st->center = st->laplacian &&
                         (st->apply_count % static_cast<unsigned long long>(st->center_k)) == 0;
            st->mean_in = st->center ? tot[1] / static_cast<double>(p.n) : 0.0;
            st->shift = 0.0;
        }
    }
}

// xmean = mean(x) for a Laplacian (min-norm solution), computed on the permuted x.
__global__ void __launch_bounds__(kThreads) k_pcg_xsum(pcg_ptrs p) {
    pcg_state* st = p.st;
    if (!st->laplacian || st->bnorm == 0.0 || p.err->code != 0) return;
    double v[1] = {0.0};
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x) v[0] += p.x[i];
    double tot[1];
    if (grid_sum<1>(v, p.partials, p.counters + kCXsum, tot)) st->xmean = tot[0] / static_cast<double>(p.n);
}

__global__ void __launch_bounds__(kThreads) k_pcg_gather_x(pcg_ptrs p) {
    const double mean = p.st->xmean;
    for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < p.n; v += gridDim.x * blockDim.x)
        p.x_orig[v] = p.x[p.perm[v]] - mean;
}

// ---- apply in the original ordering ----

__global__ void __launch_bounds__(kThreads) k_apply_bsum(apply_ptrs a) {
    if (!a.center) return;
    double v[1] = {0.0};
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) v[0] += a.b[i];
    double tot[1];
    if (grid_sum<1>(v, a.partials, a.counters + kCApply0, tot)) a.scal[0] = tot[0] / static_cast<double>(a.n);
}

__global__ void __launch_bounds__(kThreads) k_apply_permute(apply_ptrs a) {
    const bool center = a.center != 0;
    const double mean = center ? a.scal[0] : 0.0;
    for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < a.n; v += gridDim.x * blockDim.x)
        a.zp[a.perm[v]] = center ? a.b[v] - mean : a.b[v];
}

__global__ void __launch_bounds__(kThreads) k_apply_zsum(apply_ptrs a) {
    if (!a.center) return;
    double v[1] = {0.0};
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) v[0] += a.zsol[i];
    double tot[1];
    if (grid_sum<1>(v, a.partials, a.counters + kCApply0, tot)) a.scal[1] = tot[0] / static_cast<double>(a.n);
}

__global__ void __launch_bounds__(kThreads) k_apply_gather(apply_ptrs a) {
    const double shift = a.center ? a.scal[1] : 0.0;
    double v[1] = {0.0};
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const double zi = a.zsol[a.perm[i]] - shift;
        a.z[i] = zi;
        v[0] = fma(a.b[i], zi, v[0]);
    }
    double tot[1];
    if (grid_sum<1>(v, a.partials, a.counters + kCApply1, tot)) a.scal[2] = tot[0];
}

__global__ void __launch_bounds__(kThreads) k_spmv_plain(const int32_t* ptr, const int32_t* idx, const double* val,
                                                         const float* valf, const double* x, double* y, unsigned n) {
    constexpr int G = 8;
    constexpr unsigned kRowsPerWarp = 32 / G;
    const unsigned lane = threadIdx.x & (G - 1);
    const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
    for (unsigned base = warp * kRowsPerWarp; base < n; base += nwarps * kRowsPerWarp) {
        const unsigned row = base + ((threadIdx.x & 31) / G);
        double s = 0.0;
        if (row < n) {
            const int b = ptr[row], e = ptr[row + 1];
            for (int k = b + static_cast<int>(lane); k < e; k += G) s = fma(op_val(val, valf, k), x[idx[k]], s);
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o, G);
        if (lane == 0 && row < n) y[row] = s;
    }
}

}  // namespace

void launch_pcg_init(const pcg_ptrs& p, cudaStream_t s) { k_pcg_init<<<p.grid, kThreads, 0, s>>>(p); }
void launch_pcg_zsum(const pcg_ptrs& p, cudaStream_t s) { k_pcg_zsum<<<p.grid, kThreads, 0, s>>>(p); }
void launch_pcg_rz(const pcg_ptrs& p, cudaStream_t s) { k_pcg_rz<<<p.grid, kThreads, 0, s>>>(p); }
void launch_pcg_update_p(const pcg_ptrs& p, cudaStream_t s, unsigned long long h, int use_cond) {
    k_pcg_update_p<<<p.grid, kThreads, 0, s>>>(p, h, use_cond);
}
// Long rows: chunk sums (one block per chunk, fixed block tree), then each
// row's chunks added in order into Ap.
__global__ void __launch_bounds__(kThreads) k_pcg_spmv_chunks(pcg_ptrs p) {
    if (stopped(p.st, p.err)) return;
    __shared__ double red[32];
    for (unsigned ch = blockIdx.x; ch < p.n_chunks; ch += gridDim.x) {
        double a = 0.0;
        for (uint32_t q = p.ch_lo[ch] + threadIdx.x; q < p.ch_hi[ch]; q += blockDim.x)
            a = fma(op_val(p.a_val, p.a_valf, q), p.p[__ldg(p.a_idx + q)], a);
        double v[1] = {a};
        block_sum<1>(v, red);
        if (threadIdx.x == 0) p.ch_part[ch] = v[0];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads) k_pcg_spmv_long(pcg_ptrs p) {
    if (stopped(p.st, p.err)) return;
    for (unsigned r = blockIdx.x * blockDim.x + threadIdx.x; r < p.n_long; r += gridDim.x * blockDim.x) {
        double sum = 0.0;
        for (uint32_t ch = p.lr_first[r]; ch < p.lr_first[r + 1]; ++ch) sum += p.ch_part[ch];
        p.Ap[p.lr_row[r]] = sum;
    }
}

void launch_pcg_spmv(const pcg_ptrs& p, cudaStream_t s) {
    if (p.n_long) {
        k_pcg_spmv_chunks<<<std::min<unsigned>(p.n_chunks, 4u * static_cast<unsigned>(p.grid)), kThreads, 0, s>>>(p);
        k_pcg_spmv_long<<<p.grid, kThreads, 0, s>>>(p);
    }
    if (p.spmv_lanes == 1) k_pcg_spmv_rows<<<p.grid, kThreads, 0, s>>>(p);
    else if (p.spmv_lanes == 8) k_pcg_spmv<8><<<p.grid, kThreads, 0, s>>>(p);
    else k_pcg_spmv<32><<<p.grid, kThreads, 0, s>>>(p);
}
void launch_pcg_update_xr(const pcg_ptrs& p, cudaStream_t s) { k_pcg_update_xr<<<p.grid, kThreads, 0, s>>>(p); }
void launch_pcg_finish(const pcg_ptrs& p, cudaStream_t s) {
    k_pcg_xsum<<<p.grid, kThreads, 0, s>>>(p);
    k_pcg_gather_x<<<p.grid, kThreads, 0, s>>>(p);
}

void launch_apply_bsum(const apply_ptrs& a, cudaStream_t s) { k_apply_bsum<<<a.grid, kThreads, 0, s>>>(a); }
void launch_apply_permute(const apply_ptrs& a, cudaStream_t s) { k_apply_permute<<<a.grid, kThreads, 0, s>>>(a); }
void launch_apply_zsum(const apply_ptrs& a, cudaStream_t s) { k_apply_zsum<<<a.grid, kThreads, 0, s>>>(a); }
void launch_apply_gather(const apply_ptrs& a, cudaStream_t s) { k_apply_gather<<<a.grid, kThreads, 0, s>>>(a); }

void launch_spmv_plain(const int32_t* ptr, const int32_t* idx, const double* val, const float* valf, const double* x,
                       double* y, unsigned n, int grid, cudaStream_t s) {
    k_spmv_plain<<<grid, kThreads, 0, s>>>(ptr, idx, val, valf, x, y, n);
}

}  // namespace apxb

namespace apxb {

namespace {

__global__ void k_cast32to64(const float* in, double* out, size_t n) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<double>(in[i]);
}

__global__ void k_cast64to32(const double* in, float* out, size_t n) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<float>(in[i]);
}

__global__ void k_perm_in(const uint32_t* perm, const double* src, double* dst, unsigned n) {
    for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) dst[perm[v]] = src[v];
}

__global__ void k_perm_out(const uint32_t* perm, const double* src, double* dst, unsigned n) {
    for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) dst[v] = src[perm[v]];
}

// scal[4] = ||b - y||^2, scal[5] = ||b||^2 with y in the permuted ordering.
__global__ void __launch_bounds__(256) k_resid(const uint32_t* perm, const double* b_orig, const double* y_perm,
                                               double* scal, double* partials, unsigned* counter, unsigned n) {
    double v[2] = {0.0, 0.0};
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double bi = b_orig[i];
        const double d = bi - y_perm[perm[i]];
        v[0] = fma(d, d, v[0]);
        v[1] = fma(bi, bi, v[1]);
    }
    double tot[2];
    if (grid_sum<2>(v, partials, counter, tot)) {
        scal[4] = tot[0];
        scal[5] = tot[1];
    }
}

int grid_for(size_t n) {
    const size_t b = (n + 255) / 256;
    return static_cast<int>(b < 4096 ? (b ? b : 1) : 4096);
}

}  // namespace

void launch_cast32to64(const float* in, double* out, size_t n, cudaStream_t s) {
    if (n) k_cast32to64<<<grid_for(n), 256, 0, s>>>(in, out, n);
}
void launch_cast64to32(const double* in, float* out, size_t n, cudaStream_t s) {
    if (n) k_cast64to32<<<grid_for(n), 256, 0, s>>>(in, out, n);
}
void launch_perm_in(const uint32_t* perm, const double* src, double* dst, unsigned n, int grid, cudaStream_t s) {
    k_perm_in<<<grid, 256, 0, s>>>(perm, src, dst, n);
}
void launch_perm_out(const uint32_t* perm, const double* src, double* dst, unsigned n, int grid, cudaStream_t s) {
    k_perm_out<<<grid, 256, 0, s>>>(perm, src, dst, n);
}
void launch_resid(const uint32_t* perm, const double* b_orig, const double* y_perm, double* scal, double* partials,
                  unsigned* counter, unsigned n, int grid, cudaStream_t s) {
    k_resid<<<grid, 256, 0, s>>>(perm, b_orig, y_perm, scal, partials, counter, n);
}

}  // namespace apxb
