// Batched solve engine: many right-hand sides of one or several systems per
// launch (the mixed-precision form).
//
//  * A batch holds S instances (each a factor + operator pair, block-diagonal
//    in one combined permuted index space) and K right-hand-side slots per
//    instance; vectors are row-interleaved [row][K], so every factor and
//    operator entry is read once for all K columns.
//  * Preconditioner: the fp32 sweeps with fp32 accumulation over a combined
//    work plan (items of all instances, level by level: uneven instances share
//    one launch). Everything else -- SpMV, residual update, dots, centring,
//    the final true residual -- is fp64.
//  * Each slot runs its own PCG (the reference cpu_solver's semantics,
//    src/solve.cpp:478-654): per-slot scalars live on the device and are
//    produced by one finalize kernel per reduction from per-tile partials
//    summed in tile order (deterministic). A slot is "fresh" for one
//    iteration after admission: that iteration's x/r update is skipped and
//    its reductions initialise the slot, so a new right-hand side can join a
//    running batch at any iteration boundary (continuous batching).
//  * The iteration is a CUDA graph; a full solve runs it under a conditional
//    WHILE node until every slot is done.
#include <algorithm>

#include "objects.hpp"

namespace {

constexpr uint32_t kTile = 2048;   // rows per reduction tile
constexpr int kBT = 256;           // threads per block of the vector kernels
constexpr int kSd = 14;            // per-slot double arrays (bp::rz .. bp::tol)
// SpMV rows longer than kLongRow nonzeros (power-law hubs) are cut into
// chunks of kChunkNnz, each summed by one block; the row's chunks are then
// added in order (deterministic). Other rows stay with the row kernels.
constexpr uint32_t kLongRow = 128;
constexpr uint32_t kChunkNnz = 512;

enum fin_mode : int { kFinSpmv = 0, kFinXr = 1, kFinZsum = 2, kFinRz = 3, kFinResid = 4, kFinVerify = 5 };

// Device pointers and settings of a batch.
struct bp {
    int K;
    unsigned S, n_tot, n_tiles;
    const unsigned* tile_inst; const unsigned* tile_lo; const unsigned* tile_hi;
    const unsigned* inst_t0; const unsigned* inst_t1;
    const unsigned* inst_off; const unsigned* inst_n; const int* inst_lap;
    const int32_t* a_ptr; const int32_t* a_idx; const double* a_val;
    const float* a_valf;       // non-null: the operator's values in fp32 (a_val unused)
    // long SpMV rows: long row i is lr_row[i], its chunks [lr_first[i], lr_first[i+1]);
    // chunk c covers entries [ch_lo[c], ch_hi[c]); its partial sums go to ch_part[c][K]
    const uint32_t* lr_row; const uint32_t* lr_first; const uint32_t* ch_lo; const uint32_t* ch_hi;
    unsigned n_long, n_sp_chunks;
    double* ch_part;
    const uint32_t* gperm;     // original (global) index -> permuted position
    const uint32_t* inst_of;   // original (global) index -> instance
    double *x, *r, *p, *Ap, *b;
    float* rhs32;
    const float* z;
    // per slot [S*K]
    double *rz, *pAp, *alpha, *beta, *rr, *rs, *bnorm, *rnorm, *prev, *mean, *shift, *xmean, *tres, *tol;
    int *iters, *done, *status, *pmode, *center, *fresh;
    double* xa;                // per slot: the alpha this iteration's x and r updates use (0: no update)
    int* verify;               // per slot: converged on the recurrence, to be confirmed after a refresh
    unsigned long long* applies;
    int* all_done;
    int* any_center;           // some live slot centres its next preconditioner input
    int* refresh_due;          // some live slot refreshes its residual this iteration
    int refresh_every;         // a slot's residual is recomputed as b - A x every this many of its iterations (0: never)
    int max_iter, stag, center_k;
    double* partials;          // [n_tiles][K][2]
    double* sub_partials;      // [n_tiles][K/2][K]: p.Ap of every SpMV sub-tile (K >= 4)
    unsigned* sub_count;       // [n_tiles]: sub-tiles of the tile summed so far (0 between launches)
    apxb::dev_error* err;
};

// Block-level deterministic sum of NV values, result stored to partials[t][*].
template <int NV>
__device__ __forceinline__ void tile_store(double (&v)[NV], double* dst) {
    __shared__ double red[NV * 32];
    apxb::block_sum<NV>(v, red);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) dst[k] = v[k];
    __syncthreads();
}

// Per-column deterministic block reduction of the flat [row][K] kernels: a
// thread owns the column pair (c0, c0 + 1) (both column 0 when K == 1);
// lanes with the same columns combine by a fixed butterfly, then thread
// v * K + c adds the warps in order. dst[v * K + c] = total of value v, column c.
template <int K, int NV>
__device__ __forceinline__ void col_store(double (&a)[NV][2], double* dst) {
    constexpr int H = K >= 2 ? K / 2 : 1;
    __shared__ double red[kBT / 32][NV][K];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        if (K == 1) a[v][0] += a[v][1];
#pragma unroll
        for (int e = 0; e < (K == 1 ? 1 : 2); ++e)
#pragma unroll
            for (int o = H; o < 32; o <<= 1) a[v][e] += __shfl_xor_sync(apxb::kFull, a[v][e], o);
    }
    if (lane < static_cast<unsigned>(H)) {
        // the thread's pair (2 * threadIdx.x) % K: 2 * lane for K <= 64; warp w holds columns
        // [64 w % K, 64 w % K + 64) for K = 128
        const int c0 = K == 1 ? 0 : static_cast<int>((2u * threadIdx.x) % static_cast<unsigned>(K));
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            red[warp][v][c0] = a[v][0];
            if (K > 1) red[warp][v][c0 + 1] = a[v][1];
        }
    }
    __syncthreads();
    if (threadIdx.x < static_cast<unsigned>(K * NV)) {
        const int v = threadIdx.x / K, c = threadIdx.x % K;
        double s = 0.0;
        for (int w = 0; w < kBT / 32; ++w)
            if (K <= 64 || (64 * w) % K == (c & ~63)) s += red[w][v][c];   // the warps holding column c
        dst[v * K + c] = s;
    }
    __syncthreads();
}

// Flat walk of a tile's [row][K] block in pairs: element q = 2 * (tid + j * kBT)
// from the tile base; the thread's column pair is fixed (kBT * 2 % K == 0).
// Pairs are accessed as double2 / float2, so they must start at an even
// element: for K == 1 a tile starts at its instance's row offset, which can be
// odd, and then thread 0 takes the first element alone (two == false) and the
// pairs start one element later. (For K >= 2 the base is always even.)
#define FLAT_PAIRS(t, ...)                                                                    \
    {                                                                                          \
        const size_t lo_ = static_cast<size_t>(P.tile_lo[t]) * K;                             \
        const size_t end_ = static_cast<size_t>(P.tile_hi[t]) * K;                            \
        if ((lo_ & 1u) && threadIdx.x == 0 && lo_ < end_) {                                   \
            const size_t q = lo_;                                                              \
            const bool two = false;                                                            \
            __VA_ARGS__                                                                        \
        }                                                                                      \
        const size_t base_ = lo_ + (lo_ & 1u);                                                 \
        for (size_t q = base_ + 2 * threadIdx.x; q < end_; q += 2 * kBT) {                   \
            const bool two = q + 1 < end_;                                                     \
            __VA_ARGS__                                                                        \
        }                                                                                      \
    }

// The same walk for K >= 2 (the tile's [row][K] block starts and ends on an
// even element, so every access is a pair), kU pairs per thread per step: the
// step's loads are all issued (LOAD, for pair j at q = q_[j] while ok_[j])
// before its arithmetic and stores (the rest, in the walk's order, so every sum
// runs in the same order as FLAT_PAIRS).
constexpr int kU = 4;
#define FLAT_PAIRS_U(t, LOAD, ...)                                                           \
    {                                                                                          \
        const size_t lo_ = static_cast<size_t>(P.tile_lo[t]) * K;                             \
        const size_t end_ = static_cast<size_t>(P.tile_hi[t]) * K;                            \
        for (size_t s_ = lo_ + 2 * threadIdx.x; s_ < end_; s_ += 2 * kBT * kU) {             \
            size_t q_[kU];                                                                     \
            bool ok_[kU];                                                                      \
            _Pragma("unroll") for (int j = 0; j < kU; ++j) {                                  \
                q_[j] = s_ + static_cast<size_t>(j) * 2 * kBT;                                 \
                ok_[j] = q_[j] < end_;                                                         \
            }                                                                                  \
            _Pragma("unroll") for (int j = 0; j < kU; ++j) if (ok_[j]) { const size_t q = q_[j]; LOAD } \
            _Pragma("unroll") for (int j = 0; j < kU; ++j) if (ok_[j]) { const size_t q = q_[j]; (void)q; __VA_ARGS__ } \
        }                                                                                      \
    }

// fp32-stored operator values widened into a combined fp64 array.
__global__ void __launch_bounds__(kBT) k_b_widen(const float* src, double* dst, uint64_t n) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        dst[i] = static_cast<double>(src[i]);
}

// x = 0, r = b = P B (fresh slots only); B in the caller's layout: instance i,
// column c, original local index v at B[K * off_i + c * n_i + v]. Columns
// >= nrhs[i] are zero (their slots finish at once). Walks the original order
// (coalesced reads of B) and scatters each row's K values.
template <int K>
__global__ void __launch_bounds__(kBT) k_b_admit(bp P, const double* B, const int* nrhs) {
    for (unsigned g = blockIdx.x * blockDim.x + threadIdx.x; g < P.n_tot; g += gridDim.x * blockDim.x) {
        const unsigned i = P.inst_of[g], off = P.inst_off[i], ni = P.inst_n[i];
        const unsigned v = g - off;
        const size_t row = static_cast<size_t>(P.gperm[g]) * K;
#pragma unroll
        for (int c = 0; c < K; ++c) {
            const unsigned sl = i * K + c;
            if (!P.fresh[sl]) continue;
            const double bv = c < nrhs[i] ? B[static_cast<size_t>(K) * off + static_cast<size_t>(c) * ni + v] : 0.0;
            P.b[row + c] = bv; P.r[row + c] = bv; P.x[row + c] = 0.0; P.p[row + c] = 0.0;
        }
    }
}

// Ap = A p with per-slot p.Ap partials (mode 0), or Y = A X (mode 1). One
// thread per row, the K columns of every operand row read as 16-byte pairs.
template <int K>
__global__ void __launch_bounds__(kBT) k_b_spmv(bp P, const double* X, double* Y, int mode) {
    if (*P.all_done && mode == 0) return;
    if (mode == 2 && !*P.refresh_due) return;   // the residual refresh's A x, only when due
    for (unsigned t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
        double part[K];
#pragma unroll
        for (int c = 0; c < K; ++c) part[c] = 0.0;
        for (unsigned g = P.tile_lo[t] + threadIdx.x; g < P.tile_hi[t]; g += blockDim.x) {
            const unsigned row = __ldg(P.gperm + g);   // rows in the operator's own order (see k_b_spmv_pairs)
            double acc[K];
#pragma unroll
            for (int c = 0; c < K; ++c) acc[c] = 0.0;
            const int e = __ldg(P.a_ptr + row + 1);
            const int b0 = __ldg(P.a_ptr + row);
            if (static_cast<uint32_t>(e - b0) > kLongRow) {
                // a long row: its sums were made by the chunk kernels
                if (mode == 0)
#pragma unroll
                    for (int c = 0; c < K; ++c)
                        part[c] = fma(X[static_cast<size_t>(row) * K + c], Y[static_cast<size_t>(row) * K + c], part[c]);
                continue;
            }
#pragma unroll 2
            for (int k = b0; k < e; ++k) {
                const double w = apxb::op_val(P.a_val, P.a_valf, k);
                const double* src = X + static_cast<size_t>(__ldg(P.a_idx + k)) * K;
                if constexpr (K == 1) {
                    acc[0] = fma(w, src[0], acc[0]);
                } else {
#pragma unroll
                    for (int c = 0; c < K; c += 2) {
                        const double2 v = *reinterpret_cast<const double2*>(src + c);
                        acc[c] = fma(w, v.x, acc[c]);
                        acc[c + 1] = fma(w, v.y, acc[c + 1]);
                    }
                }
            }
            double* dst = Y + static_cast<size_t>(row) * K;
            const double* xr = X + static_cast<size_t>(row) * K;
            if constexpr (K == 1) {
                dst[0] = acc[0];
                if (mode == 0) part[0] = fma(xr[0], acc[0], part[0]);
            } else {
#pragma unroll
                for (int c = 0; c < K; c += 2) {
                    *reinterpret_cast<double2*>(dst + c) = make_double2(acc[c], acc[c + 1]);
                    if (mode == 0) {
                        const double2 xv = *reinterpret_cast<const double2*>(xr + c);
                        part[c] = fma(xv.x, acc[c], part[c]);
                        part[c + 1] = fma(xv.y, acc[c + 1], part[c + 1]);
                    }
                }
            }
        }
        if (mode == 0) tile_store<K>(part, P.partials + static_cast<size_t>(t) * K * 2);
    }
}

// The same for k >= 2 with the flat pair layout: a row's k columns are held by
// k/2 consecutive threads, two columns each, so every nonzero's operand row is
// read as one coalesced k*8-byte access; p.Ap partials through col_store. The
// row's own p (for p.Ap) is taken from the diagonal's gather when the row
// stores its diagonal.
// Both SpMV row kernels visit the rows in the operator's ORIGINAL order (row
// gperm[g] for g = tile_lo..tile_hi) while the vectors stay in elimination
// order. Elimination order lists each round's vertices together, so a
// vertex's neighbours sit in other rounds' segments and, visited in storage
// order, an operand row is re-read long after its first read. Visited in the
// original order, the neighbours of the rows in flight lie in one window of
// the mesh, and every operand row is reused while it is in L2. Each row's sum
// is unchanged; only the rows that share a p.Ap tile partial differ.
// That window is the rows all blocks have in flight at once. A tile is cut
// into K/2 sub-tiles of 8 block passes (16 * kBT / K rows) and the blocks
// stride over sub-tiles, so the window holds gridDim.x * 16 * kBT * 8 bytes of
// operand rows whatever K is (19 MB at 592 blocks), well inside L2; a block per
// tile would hold gridDim.x whole tiles (620 MB at K = 64). Each sub-tile
// stores its p.Ap partial; the block that completes a tile's last sub-tile
// (a per-tile counter) adds the tile's sub-partials in sub-tile order into the
// tile partial and clears the counter, so the tile partial does not depend on
// which blocks ran which sub-tiles.
template <int K>
__global__ void __launch_bounds__(kBT, 4) k_b_spmv_pairs(bp P, const double* X, double* Y, int mode) {
    if (*P.all_done && mode == 0) return;
    if (mode == 2 && !*P.refresh_due) return;   // the residual refresh's A x, only when due
    constexpr unsigned kRows = 2 * kBT / K;      // rows per pass of the block
    constexpr unsigned kNS = K >= 4 ? K / 2 : 1; // sub-tiles per tile
    constexpr unsigned kSubRows = kTile / kNS;   // 8 passes (kTile rows when K == 2)
    constexpr int kE = 4;                        // nonzeros whose gathers are in flight together
    static_assert(kSubRows % kRows == 0, "a sub-tile is whole passes");
    __shared__ int s_last;
    const unsigned c0 = (2 * threadIdx.x) % K, rsub = (2 * threadIdx.x) / K;
    for (unsigned u = blockIdx.x; u < P.n_tiles * kNS; u += gridDim.x) {
        const unsigned t = u / kNS;
        const unsigned lo = P.tile_lo[t] + (u % kNS) * kSubRows;
        const unsigned hi = min(P.tile_hi[t], lo + kSubRows);
        double acc[1][2] = {{0.0, 0.0}};
        for (unsigned g = lo + rsub; g < hi; g += kRows) {
            const unsigned row = __ldg(P.gperm + g);
            double a0 = 0.0, a1 = 0.0;
            double2 own = make_double2(0.0, 0.0);
            bool have_own = false;
            const int e = __ldg(P.a_ptr + row + 1);
            const int b0 = __ldg(P.a_ptr + row);
            if (static_cast<uint32_t>(e - b0) > kLongRow) {
                // a long row: its sums were made by the chunk kernels
                const double2 y = *reinterpret_cast<const double2*>(Y + static_cast<size_t>(row) * K + c0);
                if (mode == 0) {
                    own = *reinterpret_cast<const double2*>(X + static_cast<size_t>(row) * K + c0);
                    acc[0][0] = fma(own.x, y.x, acc[0][0]);
                    acc[0][1] = fma(own.y, y.y, acc[0][1]);
                }
                continue;
            }
            for (int k0 = b0; k0 < e; k0 += kE) {
                // indices and weights of the next kE nonzeros, then all their gathers, then the fmas
                // in CSR order
                unsigned col[kE];
                double w[kE];
                double2 v[kE];
#pragma unroll
                for (int j = 0; j < kE; ++j)
                    if (k0 + j < e) { col[j] = static_cast<unsigned>(__ldg(P.a_idx + k0 + j)); w[j] = apxb::op_val(P.a_val, P.a_valf, k0 + j); }
#pragma unroll
                for (int j = 0; j < kE; ++j)
                    if (k0 + j < e) v[j] = *reinterpret_cast<const double2*>(X + static_cast<size_t>(col[j]) * K + c0);
#pragma unroll
                for (int j = 0; j < kE; ++j)
                    if (k0 + j < e) {
                        a0 = fma(w[j], v[j].x, a0);
                        a1 = fma(w[j], v[j].y, a1);
                        if (col[j] == row) { own = v[j]; have_own = true; }
                    }
            }
            *reinterpret_cast<double2*>(Y + static_cast<size_t>(row) * K + c0) = make_double2(a0, a1);
            if (mode == 0) {
                if (!have_own) own = *reinterpret_cast<const double2*>(X + static_cast<size_t>(row) * K + c0);
                acc[0][0] = fma(own.x, a0, acc[0][0]);
                acc[0][1] = fma(own.y, a1, acc[0][1]);
            }
        }
        if (mode != 0) continue;
        if constexpr (kNS == 1) {
            col_store<K, 1>(acc, P.partials + static_cast<size_t>(t) * K * 2);
        } else {
            col_store<K, 1>(acc, P.sub_partials + static_cast<size_t>(u) * K);
            __threadfence();   // this block's sub-partial before its count
            __syncthreads();
            if (threadIdx.x == 0) {
                const unsigned before = atomicAdd(P.sub_count + t, 1u);
                s_last = before == kNS - 1;
                if (s_last) __threadfence();   // the other blocks' sub-partials before the reads below
            }
            __syncthreads();
            if (s_last) {
                if (threadIdx.x < static_cast<unsigned>(K)) {
                    const double* src = P.sub_partials + static_cast<size_t>(t) * kNS * K + threadIdx.x;
                    double sum = 0.0;
#pragma unroll 8
                    for (unsigned q = 0; q < kNS; ++q) sum += __ldcg(src + static_cast<size_t>(q) * K);
                    P.partials[static_cast<size_t>(t) * K * 2 + threadIdx.x] = sum;
                }
                if (threadIdx.x == 0) P.sub_count[t] = 0u;
            }
        }
    }
}

// Long SpMV rows, step 1: every chunk's partial sums (one block per chunk). For
// K >= 2 a thread holds a column pair and an entry lane; the entry lanes'
// sums are added in lane order. For K == 1 a fixed block tree.
template <int K>
__global__ void __launch_bounds__(kBT) k_b_spmv_chunks(bp P, const double* X, int mode) {
    if (*P.all_done && mode == 0) return;
    if (mode == 2 && !*P.refresh_due) return;   // the residual refresh's A x, only when due
    __shared__ double red[2 * kBT];
    for (unsigned ch = blockIdx.x; ch < P.n_sp_chunks; ch += gridDim.x) {
        const uint32_t lo = P.ch_lo[ch], hi = P.ch_hi[ch];
        double a0 = 0.0, a1 = 0.0;
        if constexpr (K == 1) {
            for (uint32_t q = lo + threadIdx.x; q < hi; q += kBT)
                a0 = fma(apxb::op_val(P.a_val, P.a_valf, q), X[__ldg(P.a_idx + q)], a0);
            double v[1] = {a0};
            apxb::block_sum<1>(v, red);
            if (threadIdx.x == 0) P.ch_part[ch] = v[0];
        } else {
            constexpr unsigned kLanes = 2 * kBT / K;   // entry lanes
            const unsigned c0 = (2 * threadIdx.x) % K, el = (2 * threadIdx.x) / K;
            for (uint32_t q = lo + el; q < hi; q += kLanes) {
                const double w = apxb::op_val(P.a_val, P.a_valf, q);
                const double2 v = *reinterpret_cast<const double2*>(X + static_cast<size_t>(__ldg(P.a_idx + q)) * K + c0);
                a0 = fma(w, v.x, a0);
                a1 = fma(w, v.y, a1);
            }
            red[2 * threadIdx.x] = a0;
            red[2 * threadIdx.x + 1] = a1;
            __syncthreads();
            if (threadIdx.x < static_cast<unsigned>(K)) {
                // column c: thread (lane * K/2 + c/2), component c % 2, lanes in order
                const unsigned c = threadIdx.x;
                double sum = 0.0;
                for (unsigned l = 0; l < kLanes; ++l) sum += red[2 * (l * (K / 2) + c / 2) + (c & 1u)];
                P.ch_part[static_cast<size_t>(ch) * K + c] = sum;
            }
        }
        __syncthreads();
    }
}

// Long SpMV rows, step 2: each row's chunk sums in chunk order -> Y.
template <int K>
__global__ void __launch_bounds__(kBT) k_b_spmv_long(bp P, double* Y, int mode) {
    if (*P.all_done && mode == 0) return;
    if (mode == 2 && !*P.refresh_due) return;   // the residual refresh's A x, only when due
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n_long * K; i += gridDim.x * blockDim.x) {
        const unsigned r = i / K, c = i % K;
        double sum = 0.0;
        for (uint32_t ch = P.lr_first[r]; ch < P.lr_first[r + 1]; ++ch) sum += P.ch_part[static_cast<size_t>(ch) * K + c];
        Y[static_cast<size_t>(P.lr_row[r]) * K + c] = sum;
    }
}

// Whether slot sl refreshes its residual at the start of this iteration: every
// refresh_every of its own completed iterations, and in the iteration after its
// recurrence residual first dropped below its tolerance (verify: the stop is
// then confirmed on a residual recomputed from x), so a slot's arithmetic does
// not depend on the other slots.
__device__ __forceinline__ bool refresh_slot(const bp& P, unsigned sl) {
    const int it = P.iters[sl];
    return P.refresh_every > 0 && !P.done[sl] && !P.fresh[sl] && it > 0 &&
           (it % P.refresh_every == 0 || P.verify[sl]);
}

// True-residual refresh (fp64): r = b - A x for the due slots, with A x in Ap
// from the mode-2 SpMV just before, and r.r partials for kFinVerify (which
// stops the slots whose convergence this refresh confirms). The iteration's
// x/r update then continues from the recomputed residual.
template <int K>
__global__ void __launch_bounds__(kBT) k_b_refresh(bp P) {
    if (!*P.refresh_due) return;
    const int c0 = K == 1 ? 0 : static_cast<int>((2 * threadIdx.x) % K), c1 = K == 1 ? 0 : c0 + 1;
    for (unsigned t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
        const unsigned i = P.tile_inst[t];
        const bool w0 = refresh_slot(P, i * K + c0), w1 = refresh_slot(P, i * K + c1);
        double acc[1][2] = {{0.0, 0.0}};
        if (w0 || w1) {
            FLAT_PAIRS(t, {
                if (w0) {
                    const double r = P.b[q] - P.Ap[q];
                    P.r[q] = r;
                    acc[0][0] = fma(r, r, acc[0][0]);
                }
                if (two && w1) {
                    const double r = P.b[q + 1] - P.Ap[q + 1];
                    P.r[q + 1] = r;
                    acc[0][1] = fma(r, r, acc[0][1]);
                }
            })
        }
        col_store<K, 1>(acc, P.partials + static_cast<size_t>(t) * K * 2);   // every thread of the block
    }
}

// Whether slot sl's next preconditioner application centres its input (the
// center-k schedule of kFinXr: application count + 1, or 1 for a fresh slot).
__device__ __forceinline__ bool centres_next(const bp& P, unsigned i, unsigned sl) {
    const unsigned long long ap = P.fresh[sl] ? 1ull : P.applies[sl] + 1ull;
    return P.inst_lap[i] && (ap % static_cast<unsigned long long>(P.center_k)) == 0;
}

// r -= alpha Ap with the iteration's per-slot alpha (xa: 0 for fresh and done
// slots); r.r and sum(r) partials. x += alpha p is left to k_b_up, which reads p
// anyway. Slots whose next preconditioner input is not centred get it here, as
// fp32 r (k_b_prep writes the centred ones).
template <int K>
__global__ void __launch_bounds__(kBT) k_b_xr(bp P) {
    if (*P.all_done) return;
    const int c0 = K == 1 ? 0 : static_cast<int>((2 * threadIdx.x) % K), c1 = K == 1 ? 0 : c0 + 1;
    for (unsigned t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
        const unsigned i = P.tile_inst[t];
        const unsigned s0 = i * K + c0, s1 = i * K + c1;
        const double a0 = P.xa[s0], a1 = P.xa[s1];
        const bool w0 = !centres_next(P, i, s0), w1 = !centres_next(P, i, s1);
        double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
        if constexpr (K >= 2) {
            double2 rv[kU], av[kU];
            FLAT_PAIRS_U(t, {
                rv[j] = *reinterpret_cast<const double2*>(P.r + q);
                av[j] = *reinterpret_cast<const double2*>(P.Ap + q);
            }, {
                double2 r = rv[j];
                r.x = fma(-a0, av[j].x, r.x); r.y = fma(-a1, av[j].y, r.y);
                *reinterpret_cast<double2*>(P.r + q) = r;
                if (w0 && w1) {
                    *reinterpret_cast<float2*>(P.rhs32 + q) = make_float2(static_cast<float>(r.x), static_cast<float>(r.y));
                } else {
                    if (w0) P.rhs32[q] = static_cast<float>(r.x);
                    if (w1) P.rhs32[q + 1] = static_cast<float>(r.y);
                }
                acc[0][0] = fma(r.x, r.x, acc[0][0]); acc[0][1] = fma(r.y, r.y, acc[0][1]);
                acc[1][0] += r.x; acc[1][1] += r.y;
            })
            col_store<K, 2>(acc, P.partials + static_cast<size_t>(t) * K * 2);
            continue;
        }
        FLAT_PAIRS(t, {
            if (two) {
                double2 r = *reinterpret_cast<const double2*>(P.r + q);
                const double2 ap = *reinterpret_cast<const double2*>(P.Ap + q);
                r.x = fma(-a0, ap.x, r.x); r.y = fma(-a1, ap.y, r.y);
                *reinterpret_cast<double2*>(P.r + q) = r;
                if (w0 && w1) {
                    *reinterpret_cast<float2*>(P.rhs32 + q) = make_float2(static_cast<float>(r.x), static_cast<float>(r.y));
                } else {
                    if (w0) P.rhs32[q] = static_cast<float>(r.x);
                    if (w1) P.rhs32[q + 1] = static_cast<float>(r.y);
                }
                acc[0][0] = fma(r.x, r.x, acc[0][0]); acc[0][1] = fma(r.y, r.y, acc[0][1]);
                acc[1][0] += r.x; acc[1][1] += r.y;
            } else {
                const double r = fma(-a0, P.Ap[q], P.r[q]);
                P.r[q] = r;
                if (w0) P.rhs32[q] = static_cast<float>(r);
                acc[0][0] = fma(r, r, acc[0][0]);
                acc[1][0] += r;
            }
        })
        col_store<K, 2>(acc, P.partials + static_cast<size_t>(t) * K * 2);
    }
}

// fp32 preconditioner input r - mean of the slots that centre it this
// application (the center-k input centring); the others got theirs in k_b_xr.
template <int K>
__global__ void __launch_bounds__(kBT) k_b_prep(bp P) {
    if (*P.all_done || !*P.any_center) return;
    const int c0 = K == 1 ? 0 : static_cast<int>((2 * threadIdx.x) % K), c1 = K == 1 ? 0 : c0 + 1;
    for (unsigned t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
        const unsigned i = P.tile_inst[t];
        const unsigned s0 = i * K + c0, s1 = i * K + c1;
        const bool w0 = P.center[s0] && !P.done[s0], w1 = P.center[s1] && !P.done[s1];
        if (!w0 && !w1) continue;
        const double m0 = P.mean[s0], m1 = P.mean[s1];
        FLAT_PAIRS(t, {
            if (two) {
                const double2 r = *reinterpret_cast<const double2*>(P.r + q);
                if (w0) P.rhs32[q] = static_cast<float>(r.x - m0);
                if (w1) P.rhs32[q + 1] = static_cast<float>(r.y - m1);
            } else if (w0) {
                P.rhs32[q] = static_cast<float>(P.r[q] - m0);
            }
        })
    }
}

// sum(z) partials (Laplacian instances; z = 0 at the grounded row).
template <int K>
__global__ void __launch_bounds__(kBT) k_b_zsum(bp P) {
    if (*P.all_done) return;
    for (unsigned t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
        double acc[1][2] = {{0.0, 0.0}};
        if (P.inst_lap[P.tile_inst[t]]) {
            FLAT_PAIRS(t, {
                if (two) {
                    const float2 z = *reinterpret_cast<const float2*>(P.z + q);
                    acc[0][0] += static_cast<double>(z.x); acc[0][1] += static_cast<double>(z.y);
                } else {
                    acc[0][0] += static_cast<double>(P.z[q]);
                }
            })
        }
        col_store<K, 1>(acc, P.partials + static_cast<size_t>(t) * K * 2);
    }
}

// r.(z - shift) partials.
template <int K>
__global__ void __launch_bounds__(kBT) k_b_rz(bp P) {
    if (*P.all_done) return;
    const int c0 = K == 1 ? 0 : static_cast<int>((2 * threadIdx.x) % K), c1 = K == 1 ? 0 : c0 + 1;
    for (unsigned t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
        const unsigned i = P.tile_inst[t];
        const double h0 = P.shift[i * K + c0], h1 = P.shift[i * K + c1];
        double acc[1][2] = {{0.0, 0.0}};
        if constexpr (K >= 2) {
            double2 rv[kU];
            float2 zv[kU];
            FLAT_PAIRS_U(t, {
                rv[j] = *reinterpret_cast<const double2*>(P.r + q);
                zv[j] = *reinterpret_cast<const float2*>(P.z + q);
            }, {
                acc[0][0] = fma(rv[j].x, static_cast<double>(zv[j].x) - h0, acc[0][0]);
                acc[0][1] = fma(rv[j].y, static_cast<double>(zv[j].y) - h1, acc[0][1]);
            })
            col_store<K, 1>(acc, P.partials + static_cast<size_t>(t) * K * 2);
            continue;
        }
        FLAT_PAIRS(t, {
            if (two) {
                const double2 r = *reinterpret_cast<const double2*>(P.r + q);
                const float2 z = *reinterpret_cast<const float2*>(P.z + q);
                acc[0][0] = fma(r.x, static_cast<double>(z.x) - h0, acc[0][0]);
                acc[0][1] = fma(r.y, static_cast<double>(z.y) - h1, acc[0][1]);
            } else {
                acc[0][0] = fma(P.r[q], static_cast<double>(P.z[q]) - h0, acc[0][0]);
            }
        })
        col_store<K, 1>(acc, P.partials + static_cast<size_t>(t) * K * 2);
    }
}

// x += alpha p (the iteration's step, with the old p; xa from k_b_fin), then
// p = (z - shift) + beta p for live slots; first application of a slot:
// p = z - shift. A slot that converged this iteration still takes its x step.
// Sets the graph's WHILE condition.
template <int K>
__global__ void __launch_bounds__(kBT) k_b_up(bp P, unsigned long long handle, int use_cond) {
    const bool fault = P.err->code != 0;
    const bool live = *P.all_done == 0;
    if (use_cond && blockIdx.x == 0 && threadIdx.x == 0)
        cudaGraphSetConditional(static_cast<cudaGraphConditionalHandle>(handle), (live && !fault) ? 1u : 0u);
    if (fault) return;
    const int c0 = K == 1 ? 0 : static_cast<int>((2 * threadIdx.x) % K), c1 = K == 1 ? 0 : c0 + 1;
    for (unsigned t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
        const unsigned i = P.tile_inst[t];
        const unsigned s0 = i * K + c0, s1 = i * K + c1;
        const double xa0 = P.xa[s0], xa1 = P.xa[s1];
        const bool l0 = live && !P.done[s0], l1 = live && !P.done[s1];
        const bool xs = xa0 != 0.0 || xa1 != 0.0;
        if (!l0 && !l1 && !xs) continue;
        const double h0 = P.shift[s0], h1 = P.shift[s1], b0 = P.beta[s0], b1 = P.beta[s1];
        const bool cp0 = P.pmode[s0] == 1, cp1 = P.pmode[s1] == 1;
        if constexpr (K >= 2) {
            double2 pv[kU], xv[kU];
            float2 zv[kU];
            FLAT_PAIRS_U(t, {
                pv[j] = *reinterpret_cast<const double2*>(P.p + q);
                if (xs) xv[j] = *reinterpret_cast<const double2*>(P.x + q);
                if (l0 || l1) zv[j] = *reinterpret_cast<const float2*>(P.z + q);
            }, {
                double2 p = pv[j];
                if (xs) {
                    double2 x = xv[j];
                    x.x = fma(xa0, p.x, x.x); x.y = fma(xa1, p.y, x.y);
                    *reinterpret_cast<double2*>(P.x + q) = x;
                }
                if (l0 || l1) {
                    const double z0 = static_cast<double>(zv[j].x) - h0, z1 = static_cast<double>(zv[j].y) - h1;
                    if (l0) p.x = cp0 ? z0 : fma(b0, p.x, z0);
                    if (l1) p.y = cp1 ? z1 : fma(b1, p.y, z1);
                    *reinterpret_cast<double2*>(P.p + q) = p;
                }
            })
            continue;
        }
        FLAT_PAIRS(t, {
            if (two) {
                double2 p = *reinterpret_cast<const double2*>(P.p + q);
                if (xs) {
                    double2 x = *reinterpret_cast<const double2*>(P.x + q);
                    x.x = fma(xa0, p.x, x.x); x.y = fma(xa1, p.y, x.y);
                    *reinterpret_cast<double2*>(P.x + q) = x;
                }
                if (l0 || l1) {
                    const float2 z = *reinterpret_cast<const float2*>(P.z + q);
                    const double z0 = static_cast<double>(z.x) - h0, z1 = static_cast<double>(z.y) - h1;
                    if (l0) p.x = cp0 ? z0 : fma(b0, p.x, z0);
                    if (l1) p.y = cp1 ? z1 : fma(b1, p.y, z1);
                    *reinterpret_cast<double2*>(P.p + q) = p;
                }
            } else {
                const double pq = P.p[q];
                if (xa0 != 0.0) P.x[q] = fma(xa0, pq, P.x[q]);
                if (l0) {
                    const double z0 = static_cast<double>(P.z[q]) - h0;
                    P.p[q] = cp0 ? z0 : fma(b0, pq, z0);
                }
            }
        })
    }
}

// Per-slot scalars from the tile partials, then the PCG state machine of the
// reduction that produced them. One warp per slot: lanes stride the
// instance's tiles in order, then a fixed butterfly (deterministic).
__device__ __forceinline__ void slot_sums(const bp& P, unsigned sl, int nv, double& s0, double& s1) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned i = sl / P.K, c = sl % P.K;
    s0 = 0.0; s1 = 0.0;
    // unrolled so the loads overlap; the additions stay in tile order
#pragma unroll 8
    for (unsigned t = P.inst_t0[i] + lane; t < P.inst_t1[i]; t += 32) {
        const double* src = P.partials + static_cast<size_t>(t) * P.K * 2;
        s0 += src[c];
        if (nv == 2) s1 += src[P.K + c];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(apxb::kFull, s0, o);
        s1 += __shfl_xor_sync(apxb::kFull, s1, o);
    }
}

constexpr int kFinThreads = 1024;   // one warp per slot, up to 32 slots at a time

__global__ void __launch_bounds__(kFinThreads) k_b_fin(bp P, int mode) {
    if (mode == kFinVerify && !*P.refresh_due) return;   // no refresh this iteration (uniform over the block)
    __shared__ int any_live, any_cen;
    if (threadIdx.x == 0) { any_live = 0; any_cen = 0; }
    __syncthreads();
    const unsigned nslots = P.S * P.K;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (!(*P.all_done) || mode == kFinResid) {
        for (unsigned sl = warp; sl < nslots; sl += nw) {
            const int nv = (mode == kFinXr || mode == kFinResid) ? 2 : 1;
            double s0, s1;
            slot_sums(P, sl, nv, s0, s1);
            if (lane != 0) continue;
            const unsigned i = sl / P.K;
            const double ni = static_cast<double>(P.inst_n[i]);
            if (mode == kFinResid) {
                P.tres[sl] = s1 > 0.0 ? sqrt(s0) / sqrt(s1) : 0.0;
                continue;
            }
            if (P.done[sl] && !P.fresh[sl]) continue;
            switch (mode) {
                case kFinSpmv:
                    P.pAp[sl] = s0;
                    if (!P.fresh[sl]) {
                        P.pmode[sl] = 0;
                        if (s0 <= 0.0) { P.done[sl] = 1; P.status[sl] = 3; }
                        else P.alpha[sl] = P.rz[sl] / s0;
                    }
                    break;
                case kFinXr: {
                    P.rr[sl] = s0;
                    P.rs[sl] = s1;
                    bool fin = false;
                    if (P.fresh[sl]) {
                        // initial residual r = b (src/solve.cpp:543-551)
                        P.bnorm[sl] = sqrt(s0);
                        P.iters[sl] = 0;
                        P.prev[sl] = 1.0;
                        P.pmode[sl] = 1;
                        P.applies[sl] = 0;
                        P.verify[sl] = 0;
                        if (P.bnorm[sl] == 0.0) { P.done[sl] = 1; P.status[sl] = 0; P.rnorm[sl] = 0.0; fin = true; }
                        else { P.rnorm[sl] = 1.0; P.status[sl] = 1; P.done[sl] = 0; }
                    } else {
                        const double rn = sqrt(s0) / P.bnorm[sl];
                        P.rnorm[sl] = rn;
                        const int it = ++P.iters[sl];
                        int status = 1;
                        if (rn < P.tol[sl]) {
                            // below tol on the recurrence: the next iteration recomputes b - A x from this x
                            // and kFinVerify stops the slot if that is below tol. With refreshes off, or at
                            // the iteration limit, the recurrence decides (apxb_pcg's rule).
                            if (P.refresh_every == 0 || it >= P.max_iter) { fin = true; status = 0; }
                            else P.verify[sl] = 1;
                        }
                        else if (!isfinite(rn)) { fin = true; status = 4; }
                        else if (P.stag > 0 && it % P.stag == 0) {
                            if (rn > P.prev[sl] * 0.5) { fin = true; status = 2; }
                            else P.prev[sl] = rn;
                        }
                        if (!fin && it >= P.max_iter) { fin = true; status = 1; }
                        P.status[sl] = status;
                        if (fin) P.done[sl] = 1;
                    }
                    if (!fin) {
                        const unsigned long long ap = ++P.applies[sl];
                        const int cen = P.inst_lap[i] && (ap % static_cast<unsigned long long>(P.center_k)) == 0;
                        P.center[sl] = cen;
                        P.mean[sl] = cen ? s1 / ni : 0.0;
                        P.shift[sl] = 0.0;
                    } else {
                        P.mean[sl] = 0.0;
                    }
                    break;
                }
                case kFinZsum:
                    P.shift[sl] = P.center[sl] ? s0 / ni : 0.0;
                    break;
                case kFinVerify:
                    // the refreshed residual of a slot whose recurrence fell below tol: its x stands
                    // when ||b - A x|| / ||b|| < tol (the rest of the iteration leaves a done slot alone)
                    if (P.verify[sl] && refresh_slot(P, sl)) {
                        const double rn = sqrt(s0) / P.bnorm[sl];
                        P.verify[sl] = 0;
                        if (rn < P.tol[sl]) { P.rnorm[sl] = rn; P.done[sl] = 1; P.status[sl] = 0; }
                    }
                    break;
                case kFinRz:
                    P.beta[sl] = P.pmode[sl] == 1 ? 0.0 : s0 / P.rz[sl];
                    P.rz[sl] = s0;
                    P.fresh[sl] = 0;
                    break;
                default:
                    break;
            }
        }
    }
    __syncthreads();
    if (mode == kFinRz) {   // the next iteration's residual refresh
        for (unsigned sl = threadIdx.x; sl < nslots; sl += blockDim.x)
            if (refresh_slot(P, sl)) any_cen = 1;
        __syncthreads();
        if (threadIdx.x == 0) *P.refresh_due = any_cen;
    }
    if (mode == kFinSpmv)   // the step this iteration's x and r updates take (0: fresh or done)
        for (unsigned sl = threadIdx.x; sl < nslots; sl += blockDim.x)
            P.xa[sl] = (!P.done[sl] && !P.fresh[sl]) ? P.alpha[sl] : 0.0;
    if (mode == kFinXr || mode == kFinSpmv || mode == kFinVerify) {
        for (unsigned sl = threadIdx.x; sl < nslots; sl += blockDim.x)
            if (!P.done[sl]) {
                any_live = 1;
                if (mode == kFinXr && P.center[sl]) any_cen = 1;
            }
        __syncthreads();
        if (threadIdx.x == 0) {
            *P.all_done = any_live ? 0 : 1;
            if (mode == kFinXr) *P.any_center = any_cen;
        }
    }
}

// x out to the caller's layout, minus the slot's mean for Laplacian instances
// (min-norm solution, src/solve.cpp:631-634); xmean from k_b_xsum.
template <int K>
__global__ void __launch_bounds__(kBT) k_b_xsum(bp P) {
    for (unsigned t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
        double acc[1][2] = {{0.0, 0.0}};
        FLAT_PAIRS(t, {
            if (two) {
                const double2 x = *reinterpret_cast<const double2*>(P.x + q);
                acc[0][0] += x.x; acc[0][1] += x.y;
            } else {
                acc[0][0] += P.x[q];
            }
        })
        col_store<K, 1>(acc, P.partials + static_cast<size_t>(t) * K * 2);
    }
}

__global__ void __launch_bounds__(kBT) k_b_xmean(bp P) {
    const unsigned nslots = P.S * P.K;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (unsigned sl = warp; sl < nslots; sl += nw) {
        double s, dummy;
        slot_sums(P, sl, 1, s, dummy);
        const unsigned i = sl / P.K;
        if (lane == 0)
            P.xmean[sl] = (P.inst_lap[i] && P.bnorm[sl] > 0.0) ? s / static_cast<double>(P.inst_n[i]) : 0.0;
    }
}

template <int K>
__global__ void __launch_bounds__(kBT) k_b_out(bp P, double* X) {
    for (unsigned g = blockIdx.x * blockDim.x + threadIdx.x; g < P.n_tot; g += gridDim.x * blockDim.x) {
        const unsigned i = P.inst_of[g], off = P.inst_off[i], ni = P.inst_n[i];
        const size_t row = static_cast<size_t>(P.gperm[g]) * K;
#pragma unroll
        for (int c = 0; c < K; ++c)
            X[static_cast<size_t>(K) * off + static_cast<size_t>(c) * ni + (g - off)] = P.x[row + c] - P.xmean[i * K + c];
    }
}

// ||b - A x||^2 and ||b||^2 partials with A x in Ap.
template <int K>
__global__ void __launch_bounds__(kBT) k_b_resid(bp P) {
    for (unsigned t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
        double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};   // [0]: ||b - A x||^2, [1]: ||b||^2
        FLAT_PAIRS(t, {
            if (two) {
                const double2 b = *reinterpret_cast<const double2*>(P.b + q);
                const double2 y = *reinterpret_cast<const double2*>(P.Ap + q);
                const double d0 = b.x - y.x, d1 = b.y - y.y;
                acc[0][0] = fma(d0, d0, acc[0][0]); acc[0][1] = fma(d1, d1, acc[0][1]);
                acc[1][0] = fma(b.x, b.x, acc[1][0]); acc[1][1] = fma(b.y, b.y, acc[1][1]);
            } else {
                const double d = P.b[q] - P.Ap[q];
                acc[0][0] = fma(d, d, acc[0][0]);
                acc[1][0] = fma(P.b[q], P.b[q], acc[1][0]);
            }
        })
        col_store<K, 2>(acc, P.partials + static_cast<size_t>(t) * K * 2);
    }
}

__global__ void k_b_zero_rows(float* z, const uint32_t* rows, unsigned n, int K) {
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n * static_cast<unsigned>(K); i += gridDim.x * blockDim.x)
        z[static_cast<size_t>(rows[i / K]) * K + (i % K)] = 0.0f;
}

// Continuous batching: x = 0, r = b = P b for one slot (b in original order).
template <int K>
__global__ void __launch_bounds__(kBT) k_b_admit_one(bp P, unsigned sl, const double* b) {
    const unsigned i = sl / K, c = sl % K, off = P.inst_off[i], ni = P.inst_n[i];
    for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < ni; v += gridDim.x * blockDim.x) {
        const size_t q = static_cast<size_t>(P.gperm[off + v]) * K + c;
        const double bv = b[v];
        P.b[q] = bv; P.r[q] = bv; P.x[q] = 0.0; P.p[q] = 0.0;
    }
}

// x of one slot in the original order minus the slot's mean (k_b_xsum +
// k_b_xmean: the same sums a whole-batch solve takes, so a request's result
// does not depend on the batch it ran in).
template <int K>
__global__ void __launch_bounds__(kBT) k_b_slot_out(bp P, unsigned sl, double* out) {
    const unsigned i = sl / K, c = sl % K, off = P.inst_off[i], ni = P.inst_n[i];
    const double mean = P.xmean[sl];
    for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < ni; v += gridDim.x * blockDim.x)
        out[v] = P.x[static_cast<size_t>(P.gperm[off + v]) * K + c] - mean;
}

// Slot state of an admission: fresh (its first iteration initialises it), not
// done, its tolerance; the batch is live again.
__global__ void k_b_mark_admit(bp P, unsigned sl, double tol) {
    if (threadIdx.x == 0) {
        P.fresh[sl] = 1;
        P.done[sl] = 0;
        P.verify[sl] = 0;
        P.tol[sl] = tol;
        *P.all_done = 0;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side.

struct apxb_batch {
    apxb_engine* e = nullptr;
    int S = 0, K = 0;
    uint32_t n_tot = 0;
    std::vector<uint32_t> off, n;
    std::vector<int> lap;
    std::vector<std::pair<void*, size_t>> owned;
    // batch sweep plan per direction (column lanes for this k; chunked claims)
    uint32_t n_items[2] = {0, 0};
    const uint32_t *info[2] = {nullptr, nullptr}, *ord[2] = {nullptr, nullptr}, *ptr[2] = {nullptr, nullptr};
    const uint32_t* idx[2] = {nullptr, nullptr};
    const float* val[2] = {nullptr, nullptr};
    const uint32_t* chunk[2] = {nullptr, nullptr};
    uint32_t n_chunks[2] = {0, 0};
    // fp16 factors (every instance's): binary16 plan values, per-row diagonal
    // and (backward input) inverse scale squared, in the batch's row numbering
    bool fp16 = false;
    const uint16_t* val16[2] = {nullptr, nullptr};
    const float* diag16 = nullptr;
    const double* inv_scale2 = nullptr;
    apxb::sweep_ctl* ctl = nullptr;
    int grid32 = 0;
    // operator (combined, permuted) and permutation
    const int32_t *a_ptr = nullptr, *a_idx = nullptr;
    const double* a_val = nullptr;
    const float* a_valf = nullptr;   // fp32 storage (every instance's operator fp32)
    // long SpMV rows (bp::lr_row ...)
    uint32_t n_long = 0, n_sp_chunks = 0;
    uint32_t *lr_row = nullptr, *lr_first = nullptr, *ch_lo = nullptr, *ch_hi = nullptr;
    double* ch_part = nullptr;
    uint32_t* gperm = nullptr;
    uint32_t* inst_of = nullptr;
    // tiles
    uint32_t n_tiles = 0;
    uint32_t *tile_inst = nullptr, *tile_lo = nullptr, *tile_hi = nullptr, *inst_t0 = nullptr, *inst_t1 = nullptr;
    uint32_t *inst_off = nullptr, *inst_n = nullptr;
    int* inst_lap = nullptr;
    int* nrhs = nullptr;
    // vectors and state
    double *x = nullptr, *r = nullptr, *p = nullptr, *Ap = nullptr, *b = nullptr;
    float *rhs32 = nullptr, *Yf = nullptr, *Zf = nullptr;
    bool y_armed = false;
    double* sd = nullptr;   // kSd double arrays of S*K
    int* si = nullptr;      // 6 int arrays of S*K, all_done, any_center, refresh_due
    double* xa = nullptr;   // per slot (bp::xa)
    int* verify = nullptr;  // per slot (bp::verify)
    int refresh_every = 25; // periodic fp64 residual refresh (bp::refresh_every)
    unsigned long long* applies = nullptr;
    double* partials = nullptr;
    double* sub_partials = nullptr;   // SpMV sub-tile partials (bp::sub_partials)
    unsigned* sub_count = nullptr;
    double* d_B = nullptr;  // staging of right-hand sides / solutions in the caller layout
    // graphs (max_iter is baked into them; tolerances are per slot on the device)
    cudaGraphExec_t loop = nullptr;
    cudaGraphExec_t one = nullptr;
    bool loop_cond = false;
    int graph_max = -1;
    // continuous batching: two state mirrors (steps alternate), per-slot
    // admission flags and retirement events
    int64_t steps_launched = 0;
    cudaEvent_t step_ev[2] = {nullptr, nullptr};
    double* m_sd[2] = {nullptr, nullptr};
    int* m_si[2] = {nullptr, nullptr};
    apxb::dev_error* m_err[2] = {nullptr, nullptr};
    std::vector<char> slot_busy;
    std::vector<cudaEvent_t> slot_ev;
    // pinned host mirrors
    double* h_sd = nullptr;
    int* h_si = nullptr;

    template <class T>
    int dalloc(T** q, size_t count) {
        const size_t bytes = count * sizeof(T);
        const int rc = e->alloc(reinterpret_cast<void**>(q), bytes);
        if (rc) return rc;
        owned.emplace_back(*q, bytes);
        return APXB_OK;
    }
    ~apxb_batch() {
        for (int j = 0; j < 2; ++j) {
            if (step_ev[j]) cudaEventDestroy(step_ev[j]);
            if (m_sd[j]) cudaFreeHost(m_sd[j]);
            if (m_si[j]) cudaFreeHost(m_si[j]);
            if (m_err[j]) cudaFreeHost(m_err[j]);
        }
        for (auto ev : slot_ev)
            if (ev) cudaEventDestroy(ev);
        if (loop) cudaGraphExecDestroy(loop);
        if (one) cudaGraphExecDestroy(one);
        for (auto& [q, bytes] : owned) e->release(q, bytes);
        if (h_sd) cudaFreeHost(h_sd);
        if (h_si) cudaFreeHost(h_si);
    }
    size_t slots() const { return static_cast<size_t>(S) * K; }
    // plan, buffers and counters of one sweep direction
    void sweep_dir(int dir, apxb::sweep_args<float>& a) const {
        a.n_items = n_items[dir]; a.info = info[dir]; a.ord = ord[dir]; a.ptr = ptr[dir];
        a.idx = idx[dir]; a.val = val[dir]; a.ctl = ctl + dir;
        a.chunk = chunk[dir]; a.n_chunks = n_chunks[dir];
        a.val16 = val16[dir]; a.diag16 = diag16; a.in_scale2 = dir == 1 ? inv_scale2 : nullptr;
        if (dir == 0) { a.in = rhs32; a.out = Yf; a.reset = Zf; }
        else { a.in = Yf; a.out = Zf; a.reset = Yf; }
    }
    // Markers into the forward output; the forward sweep re-arms the backward
    // output's factor rows itself, and Zf's grounded rows stay 0.
    void arm(cudaStream_t s) {
        apxb::launch_fill_sent32(Yf, static_cast<size_t>(n_tot) * K, s);
        y_armed = true;
    }
    bp params(int max_iter) const {
        bp P{};
        P.K = K; P.S = S; P.n_tot = n_tot; P.n_tiles = n_tiles;
        P.tile_inst = tile_inst; P.tile_lo = tile_lo; P.tile_hi = tile_hi; P.inst_t0 = inst_t0; P.inst_t1 = inst_t1;
        P.inst_off = inst_off; P.inst_n = inst_n; P.inst_lap = inst_lap;
        P.a_ptr = a_ptr; P.a_idx = a_idx; P.a_val = a_val; P.a_valf = a_valf; P.gperm = gperm; P.inst_of = inst_of;
        P.lr_row = lr_row; P.lr_first = lr_first; P.ch_lo = ch_lo; P.ch_hi = ch_hi;
        P.n_long = n_long; P.n_sp_chunks = n_sp_chunks; P.ch_part = ch_part;
        P.x = x; P.r = r; P.p = p; P.Ap = Ap; P.b = b; P.rhs32 = rhs32; P.z = Zf;
        const size_t ns = slots();
        double* d = sd;
        P.rz = d; P.pAp = d + ns; P.alpha = d + 2 * ns; P.beta = d + 3 * ns; P.rr = d + 4 * ns; P.rs = d + 5 * ns;
        P.bnorm = d + 6 * ns; P.rnorm = d + 7 * ns; P.prev = d + 8 * ns; P.mean = d + 9 * ns; P.shift = d + 10 * ns;
        P.xmean = d + 11 * ns; P.tres = d + 12 * ns; P.tol = d + 13 * ns;
        int* s = si;
        P.iters = s; P.done = s + ns; P.status = s + 2 * ns; P.pmode = s + 3 * ns; P.center = s + 4 * ns;
        P.fresh = s + 5 * ns; P.all_done = s + 6 * ns; P.any_center = s + 6 * ns + 1; P.refresh_due = s + 6 * ns + 2;
        P.refresh_every = refresh_every;
        P.applies = applies;
        P.xa = xa; P.verify = verify;
        P.max_iter = max_iter; P.stag = 50; P.center_k = e->center_k;
        P.partials = partials; P.sub_partials = sub_partials; P.sub_count = sub_count; P.err = e->d_err;
        return P;
    }
};

namespace {

// Batch plan of each direction (host_prep.hpp, build_batch_plan) for the
// batch's column lanes; several instances: their items merged level by level,
// rows and columns shifted to the combined index space, then re-chunked.
void batch_plan(const std::vector<const apxb_factor*>& fs, const std::vector<uint32_t>& off, int dir,
                uint32_t col_lanes, apxb::sweep_plan& out) {
    if (fs.size() == 1) {
        apxb::build_batch_plan(fs[0]->h, dir, col_lanes, out);
        return;
    }
    std::vector<apxb::sweep_plan> pl(fs.size());
    struct src_item { uint32_t inst, item; int32_t level; };
    std::vector<src_item> all;
    for (uint32_t i = 0; i < fs.size(); ++i) {
        apxb::build_batch_plan(fs[i]->h, dir, col_lanes, pl[i]);
        for (uint32_t c = 0; c < pl[i].n_items; ++c) all.push_back({i, c, pl[i].item_level[c]});
    }
    std::stable_sort(all.begin(), all.end(), [](const src_item& a, const src_item& b) { return a.level < b.level; });
    out = apxb::sweep_plan{};
    out.n_items = static_cast<uint32_t>(all.size());
    out.info.resize(all.size());
    out.item_level.resize(all.size());
    out.ord.assign(all.size() * 32, apxb::kNoRow);
    out.ptr.assign(all.size() * 32 + 1, 0);
    uint32_t e = 0;
    for (size_t c = 0; c < all.size(); ++c) {
        const auto& sit = all[c];
        const apxb::sweep_plan& p = pl[sit.inst];
        out.info[c] = p.info[sit.item];
        out.item_level[c] = sit.level;
        for (uint32_t s = 0; s < 32; ++s) {
            const size_t sp = static_cast<size_t>(sit.item) * 32 + s, dp = c * 32 + s;
            out.ptr[dp] = e;
            if (p.ord[sp] == apxb::kNoRow) continue;
            out.ord[dp] = p.ord[sp] + off[sit.inst];
            for (uint32_t q = p.ptr[sp]; q < p.ptr[sp + 1]; ++q) {
                out.idx.push_back(p.idx[q] + off[sit.inst]);
                out.val.push_back(p.val[q]);
                if (!p.val16.empty()) out.val16.push_back(p.val16[q]);
                ++e;
            }
        }
    }
    out.ptr[all.size() * 32] = e;
    apxb::chunk_plan(out);
}

template <int K>
int launch_iteration_k(apxb_batch* bt, const bp& P, cudaStream_t s, unsigned long long h, int use_cond) {
    const int g = bt->e->vec_grid;
    if (bt->refresh_every > 0) {   // r = b - A x for the slots due (every launch exits at once otherwise)
        if (bt->n_long) {
            k_b_spmv_chunks<K><<<std::min<unsigned>(bt->n_sp_chunks, 4u * g), kBT, 0, s>>>(P, P.x, 2);
            k_b_spmv_long<K><<<g, kBT, 0, s>>>(P, P.Ap, 2);
        }
        if constexpr (K == 1) k_b_spmv<K><<<g, kBT, 0, s>>>(P, P.x, P.Ap, 2);
        else k_b_spmv_pairs<K><<<g, kBT, 0, s>>>(P, P.x, P.Ap, 2);
        k_b_refresh<K><<<g, kBT, 0, s>>>(P);
        k_b_fin<<<1, kFinThreads, 0, s>>>(P, kFinVerify);
    }
    if (bt->n_long) {
        k_b_spmv_chunks<K><<<std::min<unsigned>(bt->n_sp_chunks, 4u * g), kBT, 0, s>>>(P, P.p, 0);
        k_b_spmv_long<K><<<g, kBT, 0, s>>>(P, P.Ap, 0);
    }
    if constexpr (K == 1) k_b_spmv<K><<<g, kBT, 0, s>>>(P, P.p, P.Ap, 0);
    else k_b_spmv_pairs<K><<<g, kBT, 0, s>>>(P, P.p, P.Ap, 0);
    k_b_fin<<<1, kFinThreads, 0, s>>>(P, kFinSpmv);
    k_b_xr<K><<<g, kBT, 0, s>>>(P);
    k_b_fin<<<1, kFinThreads, 0, s>>>(P, kFinXr);
    k_b_prep<K><<<g, kBT, 0, s>>>(P);
    apxb::sweep_args<float> a{};
    a.k = K; a.err = bt->e->d_err; a.budget_ns = bt->e->budget_ns; a.skip = P.all_done;
    a.m = bt->n_tot;
    for (int dir = 0; dir < 2; ++dir) {
        bt->sweep_dir(dir, a);
        apxb::launch_sweep32_batch(dir, a, bt->grid32, s);
    }
    k_b_zsum<K><<<g, kBT, 0, s>>>(P);
    k_b_fin<<<1, kFinThreads, 0, s>>>(P, kFinZsum);
    k_b_rz<K><<<g, kBT, 0, s>>>(P);
    k_b_fin<<<1, kFinThreads, 0, s>>>(P, kFinRz);
    k_b_up<K><<<g, kBT, 0, s>>>(P, h, use_cond);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return fail(APXB_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(err));
    return APXB_OK;
}

int launch_iteration(apxb_batch* bt, const bp& P, cudaStream_t s, unsigned long long h, int use_cond) {
    switch (bt->K) {
        case 1: return launch_iteration_k<1>(bt, P, s, h, use_cond);
        case 2: return launch_iteration_k<2>(bt, P, s, h, use_cond);
        case 4: return launch_iteration_k<4>(bt, P, s, h, use_cond);
        case 8: return launch_iteration_k<8>(bt, P, s, h, use_cond);
        case 16: return launch_iteration_k<16>(bt, P, s, h, use_cond);
        case 32: return launch_iteration_k<32>(bt, P, s, h, use_cond);
        case 64: return launch_iteration_k<64>(bt, P, s, h, use_cond);
        default: return launch_iteration_k<128>(bt, P, s, h, use_cond);
    }
}

template <int K>
void launch_finish_k(apxb_batch* bt, const bp& P, double* X, bool resid, cudaStream_t s) {
    const int g = bt->e->vec_grid;
    k_b_xsum<K><<<g, kBT, 0, s>>>(P);
    k_b_xmean<<<1, kBT, 0, s>>>(P);
    k_b_out<K><<<g, kBT, 0, s>>>(P, X);
    if (resid) {
        if (bt->n_long) {
            k_b_spmv_chunks<K><<<std::min<unsigned>(bt->n_sp_chunks, 4u * g), kBT, 0, s>>>(P, P.x, 1);
            k_b_spmv_long<K><<<g, kBT, 0, s>>>(P, P.Ap, 1);
        }
        if constexpr (K == 1) k_b_spmv<K><<<g, kBT, 0, s>>>(P, P.x, P.Ap, 1);
        else k_b_spmv_pairs<K><<<g, kBT, 0, s>>>(P, P.x, P.Ap, 1);
        k_b_resid<K><<<g, kBT, 0, s>>>(P);
        k_b_fin<<<1, kFinThreads, 0, s>>>(P, kFinResid);
    }
}

void launch_finish(apxb_batch* bt, const bp& P, double* X, bool resid, cudaStream_t s) {
    switch (bt->K) {
        case 1: launch_finish_k<1>(bt, P, X, resid, s); break;
        case 2: launch_finish_k<2>(bt, P, X, resid, s); break;
        case 4: launch_finish_k<4>(bt, P, X, resid, s); break;
        case 8: launch_finish_k<8>(bt, P, X, resid, s); break;
        case 16: launch_finish_k<16>(bt, P, X, resid, s); break;
        case 32: launch_finish_k<32>(bt, P, X, resid, s); break;
        case 64: launch_finish_k<64>(bt, P, X, resid, s); break;
        default: launch_finish_k<128>(bt, P, X, resid, s); break;
    }
}

template <int K>
void launch_admit_k(apxb_batch* bt, const bp& P, const double* B, cudaStream_t s) {
    k_b_admit<K><<<bt->e->vec_grid, kBT, 0, s>>>(P, B, bt->nrhs);
}

void launch_admit(apxb_batch* bt, const bp& P, const double* B, cudaStream_t s) {
    switch (bt->K) {
        case 1: launch_admit_k<1>(bt, P, B, s); break;
        case 2: launch_admit_k<2>(bt, P, B, s); break;
        case 4: launch_admit_k<4>(bt, P, B, s); break;
        case 8: launch_admit_k<8>(bt, P, B, s); break;
        case 16: launch_admit_k<16>(bt, P, B, s); break;
        case 32: launch_admit_k<32>(bt, P, B, s); break;
        case 64: launch_admit_k<64>(bt, P, B, s); break;
        default: launch_admit_k<128>(bt, P, B, s); break;
    }
}

int build_graphs(apxb_batch* bt, int max_iter) {
    if (bt->loop) { cudaGraphExecDestroy(bt->loop); bt->loop = nullptr; }
    if (bt->one) { cudaGraphExecDestroy(bt->one); bt->one = nullptr; }
    cudaStream_t s = bt->e->stream;
    const bp P = bt->params(max_iter);
    // one iteration (host-driven serving loop)
    APXB_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int rc = launch_iteration(bt, P, s, 0, 0);
    cudaGraph_t g1 = nullptr;
    APXB_CK(cudaStreamEndCapture(s, &g1));
    if (rc) { cudaGraphDestroy(g1); return rc; }
    APXB_CK(cudaGraphInstantiate(&bt->one, g1, 0));
    cudaGraphDestroy(g1);
    // WHILE loop until every slot is done
    cudaGraph_t g = nullptr;
    APXB_CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    cudaError_t err = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    if (err == cudaSuccess) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        err = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
        if (err == cudaSuccess) {
            err = cudaStreamBeginCaptureToGraph(s, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                cudaStreamCaptureModeThreadLocal);
            if (err == cudaSuccess) {
                rc = launch_iteration(bt, P, s, static_cast<unsigned long long>(h), 1);
                cudaGraph_t captured = nullptr;
                err = cudaStreamEndCapture(s, &captured);
                if (rc) { cudaGraphDestroy(g); return rc; }
            }
        }
        if (err == cudaSuccess) err = cudaGraphInstantiate(&bt->loop, g, 0);
    }
    cudaGraphDestroy(g);
    bt->loop_cond = err == cudaSuccess;
    if (!bt->loop_cond) { bt->loop = nullptr; cudaGetLastError(); }
    return APXB_OK;
}

// APXB_NO_GRAPH=1: launch every kernel directly (for per-kernel profiling).
bool no_graph() {
    const char* e = std::getenv("APXB_NO_GRAPH");
    return e && *e && *e != '0';
}

template <int K>
void slot_io_k(apxb_batch* bt, const bp& P, unsigned sl, const double* in, double* out, cudaStream_t s) {
    const int g = bt->e->vec_grid;
    if (in) {
        k_b_admit_one<K><<<g, kBT, 0, s>>>(P, sl, in);
    } else {
        k_b_xsum<K><<<g, kBT, 0, s>>>(P);
        k_b_xmean<<<1, kBT, 0, s>>>(P);
        k_b_slot_out<K><<<g, kBT, 0, s>>>(P, sl, out);
    }
}

// in != NULL: load slot sl's right-hand side; else write its solution to out.
void slot_io(apxb_batch* bt, const bp& P, unsigned sl, const double* in, double* out, cudaStream_t s) {
    switch (bt->K) {
        case 1: slot_io_k<1>(bt, P, sl, in, out, s); break;
        case 2: slot_io_k<2>(bt, P, sl, in, out, s); break;
        case 4: slot_io_k<4>(bt, P, sl, in, out, s); break;
        case 8: slot_io_k<8>(bt, P, sl, in, out, s); break;
        case 16: slot_io_k<16>(bt, P, sl, in, out, s); break;
        case 32: slot_io_k<32>(bt, P, sl, in, out, s); break;
        case 64: slot_io_k<64>(bt, P, sl, in, out, s); break;
        default: slot_io_k<128>(bt, P, sl, in, out, s); break;
    }
}

int ensure_graphs(apxb_batch* bt, int max_iter) {
    if (bt->one && bt->graph_max == max_iter) return APXB_OK;
    const int rc = build_graphs(bt, max_iter);
    if (rc) return rc;
    bt->graph_max = max_iter;
    return APXB_OK;
}

}  // namespace

extern "C" {

int apxb_batch_create(apxb_engine* e, int n_inst, apxb_factor* const* factors, apxb_operator* const* ops, int k,
                      apxb_batch** out) {
    return guarded([&]() -> int {
        if (!e || n_inst < 1 || !factors || !ops || !out) return fail(APXB_ERR_INVALID, "bad argument");
        if (k != 1 && k != 2 && k != 4 && k != 8 && k != 16 && k != 32 && k != 64 && k != 128)
            return fail(APXB_ERR_INVALID, "k must be 1, 2, 4, 8, 16, 32, 64 or 128");
        *out = nullptr;
        APXB_CK(cudaSetDevice(e->device));
        std::unique_ptr<apxb_batch> bt(new (std::nothrow) apxb_batch);
        if (!bt) return fail(APXB_ERR_INVALID, "host allocation failed");
        bt->e = e; bt->S = n_inst; bt->K = k;
        std::vector<const apxb_factor*> fs;
        uint64_t nnz_a = 0;
        for (int i = 0; i < n_inst; ++i) {
            const apxb_factor* f = factors[i];
            const apxb_operator* a = ops[i];
            if (!f || !a || f->e != e || a->e != e) return fail(APXB_ERR_INVALID, "instance objects missing or on another engine");
            if (a->n != f->h.n) return fail(APXB_ERR_INVALID, "instance operator / factor dimensions differ");
            bt->off.push_back(bt->n_tot);
            bt->n.push_back(f->h.n);
            bt->lap.push_back(f->h.sddm ? 0 : 1);
            bt->n_tot += f->h.n;
            nnz_a += a->nnz;
            fs.push_back(f);
        }
        if (nnz_a >= 0x7fffffffull) return fail(APXB_ERR_INVALID, "combined operator exceeds the int32 range");
        cudaStream_t s = e->stream;
        const size_t nk = static_cast<size_t>(bt->n_tot) * k, ns = bt->slots();
        int rc;
        // ---- sweep plans (batch plans for this k) ----
        const uint32_t col_lanes = k >= 8 ? static_cast<uint32_t>(k / 4) : 1u;
        // fp16 storage when every instance's factor has it (otherwise every
        // instance sweeps over its fp32 values)
        bt->fp16 = true;
        for (const apxb_factor* f : fs) bt->fp16 = bt->fp16 && f->precision == APXB_PREC_FP16 && f->h.fp16;
        if (n_inst == 1 && fs[0]->dev.on && !bt->fp16) {
            // a device-prepared factor: the plans are built on the device from its canonical arrays
            auto alloc_bytes = [&](void** q, size_t bytes) -> std::string {
                char* c = nullptr;
                const int r = bt->dalloc(&c, bytes);
                *q = c;
                return r ? std::string(apxb_last_error()) : std::string();
            };
            for (int dir = 0; dir < 2; ++dir) {
                apxb::dev_plan_out o;
                const std::string why = apxb::batch_plan_device(fs[0], dir, col_lanes, alloc_bytes, o, s);
                if (!why.empty()) return fail(APXB_ERR_CUDA, why);
                bt->n_items[dir] = o.n_items;
                bt->info[dir] = o.info; bt->ord[dir] = o.ord; bt->ptr[dir] = o.ptr; bt->idx[dir] = o.idx;
                bt->val[dir] = o.val; bt->chunk[dir] = o.chunk; bt->n_chunks[dir] = o.n_chunks;
            }
        } else {
            for (const apxb_factor* f : fs)   // host plans read the canonical arrays on the host
                if (!f->host_arrays) {
                    const std::string why = apxb::factor_host_arrays(const_cast<apxb_factor*>(f));
                    if (!why.empty()) return fail(APXB_ERR_CUDA, why);
                }
            apxb::sweep_plan plans[2];
            std::string bad[2];
            {
                apxb::run_threads(2, [&](unsigned dir) {
                    batch_plan(fs, bt->off, static_cast<int>(dir), col_lanes, plans[dir]);
                    if (n_inst == 1)
                        bad[dir] = apxb::check_batch_plan(fs[0]->h.m, dir == 0 ? fs[0]->h.fwd_level : fs[0]->h.bck_level,
                                                          plans[dir], col_lanes);
                });
            }
            for (int dir = 0; dir < 2; ++dir) {
                const apxb::sweep_plan& pl = plans[dir];
                if (!bad[dir].empty()) return fail(APXB_ERR_INVALID, "internal batch plan error: " + bad[dir]);
                if (bt->fp16 && pl.val16.size() != pl.idx.size())
                    return fail(APXB_ERR_INVALID, "internal batch plan error: fp16 values missing");
                uint32_t *info, *ord, *ptr, *idx, *chunk;
                float* val = nullptr;
                uint16_t* v16 = nullptr;
                if ((rc = bt->dalloc(&info, pl.info.size())) || (rc = bt->dalloc(&ord, pl.ord.size())) ||
                    (rc = bt->dalloc(&ptr, pl.ptr.size())) || (rc = bt->dalloc(&idx, pl.idx.size())) ||
                    (rc = bt->fp16 ? bt->dalloc(&v16, pl.val16.size()) : bt->dalloc(&val, pl.val.size())) ||
                    (rc = bt->dalloc(&chunk, pl.chunk.size())))
                    return rc;
                APXB_CK(cudaMemcpyAsync(info, pl.info.data(), 4 * pl.info.size(), cudaMemcpyHostToDevice, s));
                APXB_CK(cudaMemcpyAsync(ord, pl.ord.data(), 4 * pl.ord.size(), cudaMemcpyHostToDevice, s));
                APXB_CK(cudaMemcpyAsync(ptr, pl.ptr.data(), 4 * pl.ptr.size(), cudaMemcpyHostToDevice, s));
                APXB_CK(cudaMemcpyAsync(idx, pl.idx.data(), 4 * pl.idx.size(), cudaMemcpyHostToDevice, s));
                if (bt->fp16)
                    APXB_CK(cudaMemcpyAsync(v16, pl.val16.data(), 2 * pl.val16.size(), cudaMemcpyHostToDevice, s));
                else
                    APXB_CK(cudaMemcpyAsync(val, pl.val.data(), 4 * pl.val.size(), cudaMemcpyHostToDevice, s));
                APXB_CK(cudaMemcpyAsync(chunk, pl.chunk.data(), 4 * pl.chunk.size(), cudaMemcpyHostToDevice, s));
                APXB_CK(cudaStreamSynchronize(s));
                bt->n_items[dir] = pl.n_items;
                bt->info[dir] = info; bt->ord[dir] = ord; bt->ptr[dir] = ptr; bt->idx[dir] = idx; bt->val[dir] = val;
                bt->val16[dir] = v16;
                bt->chunk[dir] = chunk; bt->n_chunks[dir] = static_cast<uint32_t>(pl.chunk.size() - 1);
            }
        }
        if (bt->fp16) {   // per-row diagonal and inverse scale squared of every instance, at its row offset
            if (n_inst == 1) {
                bt->diag16 = fs[0]->diag16;
                bt->inv_scale2 = fs[0]->inv_scale2;
            } else {
                float* dg;
                double* is2;
                if ((rc = bt->dalloc(&dg, bt->n_tot)) || (rc = bt->dalloc(&is2, bt->n_tot))) return rc;
                APXB_CK(cudaMemsetAsync(dg, 0, 4 * static_cast<size_t>(bt->n_tot), s));
                APXB_CK(cudaMemsetAsync(is2, 0, 8 * static_cast<size_t>(bt->n_tot), s));
                for (int i = 0; i < n_inst; ++i) {
                    const size_t m = fs[i]->h.m;
                    APXB_CK(cudaMemcpyAsync(dg + bt->off[i], fs[i]->diag16, 4 * m, cudaMemcpyDeviceToDevice, s));
                    APXB_CK(cudaMemcpyAsync(is2 + bt->off[i], fs[i]->inv_scale2, 8 * m, cudaMemcpyDeviceToDevice, s));
                }
                APXB_CK(cudaStreamSynchronize(s));
                bt->diag16 = dg;
                bt->inv_scale2 = is2;
            }
        }
        if ((rc = bt->dalloc(&bt->ctl, 2))) return rc;
        APXB_CK(cudaMemsetAsync(bt->ctl, 0, sizeof(apxb::sweep_ctl) * 2, s));
        bt->grid32 = e->sweep_grid > 0 ? e->sweep_grid : apxb::sweep_grid32_batch(k, e->num_sms);
        // ---- operator ----
        if (n_inst == 1) {
            bt->a_ptr = ops[0]->ptr; bt->a_idx = ops[0]->idx; bt->a_val = ops[0]->val; bt->a_valf = ops[0]->valf;
        } else {
            // the combined values are fp32 when every instance stores fp32, else fp64
            // (fp32-stored instances widened: the same values)
            bool all32 = true;
            for (int i = 0; i < n_inst; ++i) all32 = all32 && ops[i]->valf != nullptr;
            int32_t *ap, *ai;
            double* av = nullptr;
            float* avf = nullptr;
            if ((rc = bt->dalloc(&ap, bt->n_tot + 1)) || (rc = bt->dalloc(&ai, nnz_a)) ||
                (rc = all32 ? bt->dalloc(&avf, nnz_a) : bt->dalloc(&av, nnz_a)))
                return rc;
            std::vector<int32_t> hp(bt->n_tot + 1, 0);
            uint64_t base = 0;
            for (int i = 0; i < n_inst; ++i) {
                const apxb_operator* a = ops[i];
                std::vector<int32_t> p(a->n + 1), ix(a->nnz);
                APXB_CK(cudaMemcpy(p.data(), a->ptr, 4 * (static_cast<size_t>(a->n) + 1), cudaMemcpyDeviceToHost));
                APXB_CK(cudaMemcpy(ix.data(), a->idx, 4 * a->nnz, cudaMemcpyDeviceToHost));
                for (uint32_t r = 0; r <= a->n; ++r) hp[bt->off[i] + r] = static_cast<int32_t>(base + p[r]);
                for (auto& c : ix) c += static_cast<int32_t>(bt->off[i]);
                APXB_CK(cudaMemcpy(ai + base, ix.data(), 4 * a->nnz, cudaMemcpyHostToDevice));
                if (all32) {
                    APXB_CK(cudaMemcpy(avf + base, a->valf, 4 * a->nnz, cudaMemcpyDeviceToDevice));
                } else if (a->valf) {
                    k_b_widen<<<e->vec_grid, kBT, 0, s>>>(a->valf, av + base, a->nnz);
                    APXB_CK(cudaGetLastError());
                    APXB_CK(cudaStreamSynchronize(s));
                } else {
                    APXB_CK(cudaMemcpy(av + base, a->val, 8 * a->nnz, cudaMemcpyDeviceToDevice));
                }
                base += a->nnz;
            }
            APXB_CK(cudaMemcpy(ap, hp.data(), 4 * hp.size(), cudaMemcpyHostToDevice));
            bt->a_ptr = ap; bt->a_idx = ai; bt->a_val = av; bt->a_valf = avf;
        }
        // ---- long SpMV rows ----
        {
            std::vector<int32_t> hp(bt->n_tot + 1);
            APXB_CK(cudaMemcpy(hp.data(), bt->a_ptr, 4 * hp.size(), cudaMemcpyDeviceToHost));
            std::vector<uint32_t> lrow, lfirst, clo, chi;
            for (uint32_t r = 0; r < bt->n_tot; ++r) {
                const uint32_t b0 = static_cast<uint32_t>(hp[r]), e0 = static_cast<uint32_t>(hp[r + 1]);
                if (e0 - b0 <= kLongRow) continue;
                lrow.push_back(r);
                lfirst.push_back(static_cast<uint32_t>(clo.size()));
                for (uint32_t q = b0; q < e0; q += kChunkNnz) { clo.push_back(q); chi.push_back(std::min(e0, q + kChunkNnz)); }
            }
            if (!lrow.empty()) {
                lfirst.push_back(static_cast<uint32_t>(clo.size()));
                bt->n_long = static_cast<uint32_t>(lrow.size());
                bt->n_sp_chunks = static_cast<uint32_t>(clo.size());
                if ((rc = bt->dalloc(&bt->lr_row, lrow.size())) || (rc = bt->dalloc(&bt->lr_first, lfirst.size())) ||
                    (rc = bt->dalloc(&bt->ch_lo, clo.size())) || (rc = bt->dalloc(&bt->ch_hi, chi.size())) ||
                    (rc = bt->dalloc(&bt->ch_part, static_cast<size_t>(clo.size()) * k)))
                    return rc;
                APXB_CK(cudaMemcpy(bt->lr_row, lrow.data(), 4 * lrow.size(), cudaMemcpyHostToDevice));
                APXB_CK(cudaMemcpy(bt->lr_first, lfirst.data(), 4 * lfirst.size(), cudaMemcpyHostToDevice));
                APXB_CK(cudaMemcpy(bt->ch_lo, clo.data(), 4 * clo.size(), cudaMemcpyHostToDevice));
                APXB_CK(cudaMemcpy(bt->ch_hi, chi.data(), 4 * chi.size(), cudaMemcpyHostToDevice));
            }
        }
        // ---- permutation (permuted position -> original global index), tiles ----
        {
            std::vector<uint32_t> gp(bt->n_tot), io(bt->n_tot);
            std::vector<uint32_t> ti, tl, th, t0(n_inst), t1(n_inst);
            for (int i = 0; i < n_inst; ++i) {
                const auto& perm = fs[i]->h.perm;
                for (uint32_t v = 0; v < bt->n[i]; ++v) { gp[bt->off[i] + v] = bt->off[i] + perm[v]; io[bt->off[i] + v] = i; }
                t0[i] = static_cast<uint32_t>(ti.size());
                for (uint32_t lo = 0; lo < bt->n[i]; lo += kTile) {
                    ti.push_back(static_cast<uint32_t>(i));
                    tl.push_back(bt->off[i] + lo);
                    th.push_back(bt->off[i] + std::min(bt->n[i], lo + kTile));
                }
                t1[i] = static_cast<uint32_t>(ti.size());
            }
            bt->n_tiles = static_cast<uint32_t>(ti.size());
            if ((rc = bt->dalloc(&bt->gperm, bt->n_tot)) || (rc = bt->dalloc(&bt->inst_of, bt->n_tot)) ||
                (rc = bt->dalloc(&bt->tile_inst, ti.size())) ||
                (rc = bt->dalloc(&bt->tile_lo, ti.size())) || (rc = bt->dalloc(&bt->tile_hi, ti.size())) ||
                (rc = bt->dalloc(&bt->inst_t0, n_inst)) || (rc = bt->dalloc(&bt->inst_t1, n_inst)) ||
                (rc = bt->dalloc(&bt->inst_off, n_inst)) || (rc = bt->dalloc(&bt->inst_n, n_inst)) ||
                (rc = bt->dalloc(&bt->inst_lap, n_inst)) || (rc = bt->dalloc(&bt->nrhs, n_inst)))
                return rc;
            APXB_CK(cudaMemcpy(bt->gperm, gp.data(), 4 * gp.size(), cudaMemcpyHostToDevice));
            APXB_CK(cudaMemcpy(bt->inst_of, io.data(), 4 * io.size(), cudaMemcpyHostToDevice));
            APXB_CK(cudaMemcpy(bt->tile_inst, ti.data(), 4 * ti.size(), cudaMemcpyHostToDevice));
            APXB_CK(cudaMemcpy(bt->tile_lo, tl.data(), 4 * tl.size(), cudaMemcpyHostToDevice));
            APXB_CK(cudaMemcpy(bt->tile_hi, th.data(), 4 * th.size(), cudaMemcpyHostToDevice));
            APXB_CK(cudaMemcpy(bt->inst_t0, t0.data(), 4 * t0.size(), cudaMemcpyHostToDevice));
            APXB_CK(cudaMemcpy(bt->inst_t1, t1.data(), 4 * t1.size(), cudaMemcpyHostToDevice));
            APXB_CK(cudaMemcpy(bt->inst_off, bt->off.data(), 4 * bt->off.size(), cudaMemcpyHostToDevice));
            APXB_CK(cudaMemcpy(bt->inst_n, bt->n.data(), 4 * bt->n.size(), cudaMemcpyHostToDevice));
            APXB_CK(cudaMemcpy(bt->inst_lap, bt->lap.data(), 4 * bt->lap.size(), cudaMemcpyHostToDevice));
        }
        // ---- vectors, state ----
        if ((rc = bt->dalloc(&bt->x, nk)) || (rc = bt->dalloc(&bt->r, nk)) || (rc = bt->dalloc(&bt->p, nk)) ||
            (rc = bt->dalloc(&bt->Ap, nk)) || (rc = bt->dalloc(&bt->b, nk)) || (rc = bt->dalloc(&bt->rhs32, nk)) ||
            (rc = bt->dalloc(&bt->Yf, nk)) || (rc = bt->dalloc(&bt->Zf, nk)) || (rc = bt->dalloc(&bt->sd, kSd * ns)) ||
            (rc = bt->dalloc(&bt->si, 6 * ns + 3)) || (rc = bt->dalloc(&bt->applies, ns)) ||
            (rc = bt->dalloc(&bt->xa, ns)) || (rc = bt->dalloc(&bt->verify, ns)) ||
            (rc = bt->dalloc(&bt->partials, static_cast<size_t>(bt->n_tiles) * k * 2)) || (rc = bt->dalloc(&bt->d_B, nk)) ||
            (rc = bt->dalloc(&bt->sub_partials, static_cast<size_t>(bt->n_tiles) * std::max(1, k / 2) * k)) ||
            (rc = bt->dalloc(&bt->sub_count, bt->n_tiles)))
            return rc;
        APXB_CK(cudaMemsetAsync(bt->sub_count, 0, sizeof(unsigned) * bt->n_tiles, s));
        APXB_CK(cudaMallocHost(&bt->h_sd, sizeof(double) * kSd * ns));
        APXB_CK(cudaMallocHost(&bt->h_si, sizeof(int) * (6 * ns + 1)));
        std::fill(bt->h_sd, bt->h_sd + kSd * ns, 0.0);
        std::fill(bt->h_si, bt->h_si + 6 * ns + 1, 0);
        std::fill(bt->h_si + ns, bt->h_si + 2 * ns, 1);   // host mirror of the idle state below
        APXB_CK(cudaMemsetAsync(bt->sd, 0, sizeof(double) * kSd * ns, s));
        APXB_CK(cudaMemsetAsync(bt->si, 0, sizeof(int) * (6 * ns + 3), s));
        {   // every slot starts idle: done, and the batch all done
            std::vector<int> idle(ns + 1, 1);
            APXB_CK(cudaMemcpyAsync(bt->si + ns, idle.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, s));
            APXB_CK(cudaMemcpyAsync(bt->si + 6 * ns, idle.data(), sizeof(int), cudaMemcpyHostToDevice, s));
        }
        APXB_CK(cudaMemsetAsync(bt->applies, 0, sizeof(unsigned long long) * ns, s));
        APXB_CK(cudaMemsetAsync(bt->xa, 0, sizeof(double) * ns, s));
        APXB_CK(cudaMemsetAsync(bt->verify, 0, sizeof(int) * ns, s));
        APXB_CK(cudaMemsetAsync(bt->p, 0, sizeof(double) * nk, s));
        // Zf: markers on factor rows, 0 on each Laplacian instance's grounded row
        apxb::launch_fill_sent32(bt->Yf, nk, s);
        apxb::launch_fill_sent32(bt->Zf, nk, s);
        {
            std::vector<uint32_t> grounded;
            for (int i = 0; i < n_inst; ++i)
                if (bt->lap[i]) grounded.push_back(bt->off[i] + bt->n[i] - 1);
            if (!grounded.empty()) {
                uint32_t* gr;
                if ((rc = bt->dalloc(&gr, grounded.size()))) return rc;
                APXB_CK(cudaMemcpy(gr, grounded.data(), 4 * grounded.size(), cudaMemcpyHostToDevice));
                k_b_zero_rows<<<1, 256, 0, s>>>(bt->Zf, gr, static_cast<unsigned>(grounded.size()), k);
            }
        }
        bt->y_armed = true;
        APXB_CK(cudaGetLastError());
        APXB_CK(cudaStreamSynchronize(s));
        e->children++;
        *out = bt.release();
        return APXB_OK;
    });
}

int apxb_batch_destroy(apxb_batch* bt) {
    if (!bt) return APXB_OK;
    apxb_engine* e = bt->e;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    delete bt;
    apxb_detail::release_child(e);
    return APXB_OK;
}

int apxb_batch_size(const apxb_batch* bt, int* n_inst, int* k, uint32_t* n_total) {
    if (!bt) return fail(APXB_ERR_INVALID, "batch is NULL");
    if (n_inst) *n_inst = bt->S;
    if (k) *k = bt->K;
    if (n_total) *n_total = bt->n_tot;
    return APXB_OK;
}

int apxb_batch_solve(apxb_batch* bt, const double* B, double* X, const int* nrhs, double tol, int max_iter,
                     int flags, apxb_pcg_result* res) {
    return guarded([&]() -> int {
        if (!bt || !B || !X || !res) return fail(APXB_ERR_INVALID, "bad argument");
        if (!(tol >= 0.0) || max_iter < 0) return fail(APXB_ERR_INVALID, "bad tol / max_iter");
        for (char busy : bt->slot_busy)
            if (busy) return fail(APXB_ERR_BUSY, "slots are admitted for continuous batching");
        apxb_engine* e = bt->e;
        APXB_CK(cudaSetDevice(e->device));
        cudaStream_t s = e->stream;
        const size_t nk = static_cast<size_t>(bt->n_tot) * bt->K, ns = bt->slots();
        const bool dev = flags & APXB_DEVICE_PTRS;
        std::vector<int> nr(bt->S, bt->K);
        if (nrhs)
            for (int i = 0; i < bt->S; ++i) {
                if (nrhs[i] < 0 || nrhs[i] > bt->K) return fail(APXB_ERR_INVALID, "nrhs out of range");
                nr[i] = nrhs[i];
            }
        APXB_CK(cudaMemcpyAsync(bt->nrhs, nr.data(), sizeof(int) * nr.size(), cudaMemcpyHostToDevice, s));
        const double* dB = B;
        if (!dev) {
            APXB_CK(cudaMemcpyAsync(bt->d_B, B, 8 * nk, cudaMemcpyHostToDevice, s));
            dB = bt->d_B;
        }
        {
            const int rc = ensure_graphs(bt, max_iter);
            if (rc) return rc;
        }
        const bp P = bt->params(max_iter);
        // every slot fresh with the call's tolerance, nothing done
        std::vector<int> ones(ns, 1);
        std::vector<double> tols(ns, tol);
        APXB_CK(cudaMemcpyAsync(P.tol, tols.data(), sizeof(double) * ns, cudaMemcpyHostToDevice, s));
        APXB_CK(cudaMemsetAsync(P.done, 0, sizeof(int) * ns, s));
        APXB_CK(cudaMemcpyAsync(P.fresh, ones.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, s));
        APXB_CK(cudaMemsetAsync(P.all_done, 0, sizeof(int), s));
        APXB_CK(cudaMemsetAsync(P.refresh_due, 0, sizeof(int), s));
        if (!bt->y_armed) bt->arm(s);
        APXB_CK(cudaEventRecord(e->ev0, s));
        launch_admit(bt, P, dB, s);
        if (no_graph()) {
            for (int it = 0; it <= max_iter + 1; it += 4) {
                for (int j = 0; j < 4; ++j) {
                    const int rc = launch_iteration(bt, P, s, 0, 0);
                    if (rc) return rc;
                }
                int ad = 0;
                APXB_CK(cudaMemcpyAsync(&ad, P.all_done, sizeof(int), cudaMemcpyDeviceToHost, s));
                APXB_CK(cudaStreamSynchronize(s));
                if (ad) break;
            }
        } else if (bt->loop_cond) {
            APXB_CK(cudaGraphLaunch(bt->loop, s));
        } else {
            for (int it = 0; it <= max_iter + 1; it += 4) {
                for (int j = 0; j < 4; ++j) APXB_CK(cudaGraphLaunch(bt->one, s));
                int ad = 0;
                APXB_CK(cudaMemcpyAsync(&ad, P.all_done, sizeof(int), cudaMemcpyDeviceToHost, s));
                APXB_CK(cudaStreamSynchronize(s));
                if (ad) break;
            }
        }
        double* dX = dev ? X : bt->d_B;
        launch_finish(bt, P, dX, (flags & APXB_TRUE_RESIDUAL) != 0, s);
        APXB_CK(cudaEventRecord(e->ev1, s));
        APXB_CK(cudaGetLastError());
        if (!dev) APXB_CK(cudaMemcpyAsync(X, bt->d_B, 8 * nk, cudaMemcpyDeviceToHost, s));
        APXB_CK(cudaMemcpyAsync(bt->h_sd, bt->sd, sizeof(double) * kSd * ns, cudaMemcpyDeviceToHost, s));
        APXB_CK(cudaMemcpyAsync(bt->h_si, bt->si, sizeof(int) * 6 * ns, cudaMemcpyDeviceToHost, s));
        const int rc = e->take_error();
        if (rc) { bt->y_armed = false; cudaMemsetAsync(bt->ctl, 0, 2 * sizeof(apxb::sweep_ctl), s); return rc; }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e->ev0, e->ev1);
        for (size_t sl = 0; sl < ns; ++sl) {
            res[sl].iterations = bt->h_si[sl];
            res[sl].status = bt->h_si[2 * ns + sl];
            res[sl].residual = bt->h_sd[7 * ns + sl];
            res[sl].true_residual = (flags & APXB_TRUE_RESIDUAL) ? bt->h_sd[12 * ns + sl] : -1.0;
            res[sl].seconds = ms * 1e-3;
        }
        return APXB_OK;
    });
}

// Host-only: the batch plans of one factor for k right-hand sides, built and
// checked as apxb_batch_create does (no GPU).
int apxb_batch_plan_host(uint32_t n, const uint32_t* colptr, const uint32_t* rowidx, const float* vals,
                         const uint32_t* perm, int sddm, const uint64_t* rounds, uint32_t n_rounds, double drop_rel,
                         int k, uint32_t* n_items, uint32_t* n_chunks) {
    return guarded([&]() -> int {
        if (!colptr || !rowidx || !vals || !perm || !n_items || !n_chunks) return fail(APXB_ERR_INVALID, "NULL argument");
        if (k != 1 && k != 2 && k != 4 && k != 8 && k != 16 && k != 32 && k != 64 && k != 128)
            return fail(APXB_ERR_INVALID, "k must be 1, 2, 4, 8, 16, 32, 64 or 128");
        apxb_factor f;
        const std::string why = apxb::prepare_factor(n, colptr, rowidx, vals, perm, sddm != 0, rounds, n_rounds,
                                                     drop_rel < 0.0 ? apxb::kDropRelDefault : drop_rel, f.h);
        if (!why.empty()) return fail(APXB_ERR_BAD_FACTOR, why);
        const uint32_t col_lanes = k >= 8 ? static_cast<uint32_t>(k / 4) : 1u;
        for (int dir = 0; dir < 2; ++dir) {
            apxb::sweep_plan pl;
            batch_plan({&f}, {0u}, dir, col_lanes, pl);
            const std::string bad = apxb::check_batch_plan(f.h.m, dir == 0 ? f.h.fwd_level : f.h.bck_level, pl, col_lanes);
            if (!bad.empty()) return fail(APXB_ERR_INVALID, "batch plan: " + bad);
            n_items[dir] = pl.n_items;
            n_chunks[dir] = static_cast<uint32_t>(pl.chunk.size() - 1);
        }
        return APXB_OK;
    });
}

int apxb_batch_set_refresh(apxb_batch* bt, int every) {
    if (!bt || every < 0) return fail(APXB_ERR_INVALID, "bad argument");
    for (char busy : bt->slot_busy)
        if (busy) return fail(APXB_ERR_BUSY, "slots are admitted");
    if (every == bt->refresh_every) return APXB_OK;
    APXB_CK(cudaSetDevice(bt->e->device));
    APXB_CK(cudaStreamSynchronize(bt->e->stream));
    bt->refresh_every = every;
    // the iteration graphs hold the refresh launches: rebuild them on next use
    if (bt->loop) { cudaGraphExecDestroy(bt->loop); bt->loop = nullptr; }
    if (bt->one) { cudaGraphExecDestroy(bt->one); bt->one = nullptr; }
    bt->graph_max = -1;
    return APXB_OK;
}

// ---- continuous batching ----
// Everything is enqueued on the engine stream in order and nothing waits,
// so the host can keep iterations queued while it admits and retires slots.

namespace {

// Staging of slot sl (instance i, column c) in the caller layout: K*off_i + c*n_i.
double* slot_stage(apxb_batch* bt, unsigned sl) {
    const unsigned i = sl / bt->K, c = sl % bt->K;
    return bt->d_B + static_cast<size_t>(bt->K) * bt->off[i] + static_cast<size_t>(c) * bt->n[i];
}

int serving_init(apxb_batch* bt) {
    if (bt->step_ev[0]) return APXB_OK;
    const size_t ns = bt->slots();
    for (int j = 0; j < 2; ++j) {
        APXB_CK(cudaEventCreateWithFlags(&bt->step_ev[j], cudaEventDisableTiming));
        APXB_CK(cudaMallocHost(&bt->m_sd[j], sizeof(double) * kSd * ns));
        APXB_CK(cudaMallocHost(&bt->m_si[j], sizeof(int) * (6 * ns + 1)));
        APXB_CK(cudaMallocHost(&bt->m_err[j], sizeof(apxb::dev_error)));
    }
    bt->slot_busy.assign(ns, 0);
    bt->slot_ev.assign(ns, nullptr);
    for (auto& ev : bt->slot_ev) APXB_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    return APXB_OK;
}

}  // namespace

int apxb_batch_admit(apxb_batch* bt, int slot, const double* b, double tol, int max_iter, int flags) {
    if (!bt || !b || slot < 0 || static_cast<size_t>(slot) >= bt->slots() || !(tol >= 0.0) || max_iter < 0)
        return fail(APXB_ERR_INVALID, "bad argument");
    apxb_engine* e = bt->e;
    APXB_CK(cudaSetDevice(e->device));
    int rc = serving_init(bt);
    if (rc) return rc;
    if (bt->slot_busy[slot]) return fail(APXB_ERR_BUSY, "slot is admitted and not retired");
    cudaStream_t s = e->stream;
    if (bt->graph_max != max_iter) {
        // the graphs bake max_iter: change it only while no slot is admitted
        for (char busy : bt->slot_busy)
            if (busy) return fail(APXB_ERR_BUSY, "max_iter differs from that of the admitted slots");
        if ((rc = ensure_graphs(bt, max_iter))) return rc;
    }
    const bp P = bt->params(bt->graph_max);
    const unsigned sl = static_cast<unsigned>(slot);
    const double* db = b;
    if (!(flags & APXB_DEVICE_PTRS)) {
        double* st = slot_stage(bt, sl);
        APXB_CK(cudaMemcpyAsync(st, b, 8 * static_cast<size_t>(bt->n[sl / bt->K]), cudaMemcpyHostToDevice, s));
        db = st;
    }
    if (!bt->y_armed) bt->arm(s);
    slot_io(bt, P, sl, db, nullptr, s);
    k_b_mark_admit<<<1, 32, 0, s>>>(P, sl, tol);
    APXB_CK(cudaGetLastError());
    bt->slot_busy[slot] = 1;
    return APXB_OK;
}

int apxb_batch_step(apxb_batch* bt, int iterations, int64_t* step_id) {
    if (!bt || iterations < 1 || !step_id) return fail(APXB_ERR_INVALID, "bad argument");
    if (!bt->one || !bt->step_ev[0]) return fail(APXB_ERR_INVALID, "nothing admitted");
    apxb_engine* e = bt->e;
    APXB_CK(cudaSetDevice(e->device));
    cudaStream_t s = e->stream;
    const int j = static_cast<int>(bt->steps_launched & 1);
    // mirror j was last written by step id - 2, which the caller has consumed
    APXB_CK(cudaEventSynchronize(bt->step_ev[j]));
    for (int k = 0; k < iterations; ++k) APXB_CK(cudaGraphLaunch(bt->one, s));
    const size_t ns = bt->slots();
    APXB_CK(cudaMemcpyAsync(bt->m_si[j], bt->si, sizeof(int) * (6 * ns + 1), cudaMemcpyDeviceToHost, s));
    APXB_CK(cudaMemcpyAsync(bt->m_sd[j], bt->sd, sizeof(double) * kSd * ns, cudaMemcpyDeviceToHost, s));
    APXB_CK(cudaMemcpyAsync(bt->m_err[j], e->d_err, sizeof(apxb::dev_error), cudaMemcpyDeviceToHost, s));
    APXB_CK(cudaEventRecord(bt->step_ev[j], s));
    *step_id = bt->steps_launched++;
    return APXB_OK;
}

namespace {

int step_mirror(const apxb_batch* bt, int64_t step_id, int* j) {
    if (step_id < 0 || step_id >= bt->steps_launched || step_id < bt->steps_launched - 2)
        return fail(APXB_ERR_INVALID, "step id is not one of the last two steps");
    *j = static_cast<int>(step_id & 1);
    return APXB_OK;
}

}  // namespace

int apxb_batch_query(apxb_batch* bt, int64_t step_id, int* ready) {
    if (!bt || !ready) return fail(APXB_ERR_INVALID, "bad argument");
    int j = 0;
    int rc = step_mirror(bt, step_id, &j);
    if (rc) return rc;
    const cudaError_t q = cudaEventQuery(bt->step_ev[j]);
    if (q == cudaErrorNotReady) { *ready = 0; return APXB_OK; }
    if (q != cudaSuccess) return fail(APXB_ERR_CUDA, cudaGetErrorString(q));
    *ready = 1;
    if (bt->m_err[j]->code != 0) {   // a device error recorded during the step
        bt->m_err[j]->code = 0;
        rc = bt->e->take_error();
        bt->y_armed = false;
        cudaMemsetAsync(bt->ctl, 0, 2 * sizeof(apxb::sweep_ctl), bt->e->stream);
        return rc ? rc : fail(APXB_ERR_CUDA, "device error during a step");
    }
    return APXB_OK;
}

int apxb_batch_slots(const apxb_batch* bt, int64_t step_id, int* done, int* iterations, int* status,
                     double* residual) {
    if (!bt) return fail(APXB_ERR_INVALID, "batch is NULL");
    int j = 0;
    const int rc = step_mirror(bt, step_id, &j);
    if (rc) return rc;
    APXB_CK(cudaEventSynchronize(bt->step_ev[j]));
    const size_t ns = bt->slots();
    const int* si = bt->m_si[j];
    for (size_t sl = 0; sl < ns; ++sl) {
        if (done) done[sl] = si[ns + sl] && !si[5 * ns + sl];
        if (iterations) iterations[sl] = si[sl];
        if (status) status[sl] = si[2 * ns + sl];
        if (residual) residual[sl] = bt->m_sd[j][7 * ns + sl];
    }
    return APXB_OK;
}

int apxb_batch_retire(apxb_batch* bt, int slot, double* x, int flags) {
    if (!bt || !x || slot < 0 || static_cast<size_t>(slot) >= bt->slots()) return fail(APXB_ERR_INVALID, "bad argument");
    apxb_engine* e = bt->e;
    APXB_CK(cudaSetDevice(e->device));
    if (bt->slot_busy.empty() || !bt->slot_busy[slot]) return fail(APXB_ERR_INVALID, "slot was not admitted");
    cudaStream_t s = e->stream;
    const bp P = bt->params(bt->graph_max);
    const unsigned sl = static_cast<unsigned>(slot);
    double* dx = (flags & APXB_DEVICE_PTRS) ? x : slot_stage(bt, sl);
    slot_io(bt, P, sl, nullptr, dx, s);
    APXB_CK(cudaGetLastError());
    if (!(flags & APXB_DEVICE_PTRS))
        APXB_CK(cudaMemcpyAsync(x, dx, 8 * static_cast<size_t>(bt->n[sl / bt->K]), cudaMemcpyDeviceToHost, s));
    APXB_CK(cudaEventRecord(bt->slot_ev[slot], s));
    bt->slot_busy[slot] = 0;
    return APXB_OK;
}

int apxb_batch_retired(apxb_batch* bt, int slot, int* ready) {
    if (!bt || !ready || slot < 0 || static_cast<size_t>(slot) >= bt->slots() || bt->slot_ev.empty())
        return fail(APXB_ERR_INVALID, "bad argument");
    const cudaError_t q = cudaEventQuery(bt->slot_ev[slot]);
    if (q == cudaErrorNotReady) { *ready = 0; return APXB_OK; }
    if (q != cudaSuccess) return fail(APXB_ERR_CUDA, cudaGetErrorString(q));
    *ready = 1;
    return APXB_OK;
}

// Times the batch's own forward and backward fp32 sweeps (k columns) on the
// right-hand sides of its last iteration; seconds per sweep of each direction.
int apxb_batch_sweep_timed(apxb_batch* bt, int reps, double* fwd_seconds, double* bck_seconds) {
    if (!bt || reps < 1 || !fwd_seconds || !bck_seconds) return fail(APXB_ERR_INVALID, "bad argument");
    apxb_engine* e = bt->e;
    APXB_CK(cudaSetDevice(e->device));
    cudaStream_t s = e->stream;
    cudaEvent_t ev[3];
    for (auto& v : ev) APXB_CK(cudaEventCreate(&v));
    if (!bt->y_armed) bt->arm(s);
    apxb::sweep_args<float> a{};
    a.k = bt->K; a.err = e->d_err; a.budget_ns = e->budget_ns; a.skip = nullptr; a.m = bt->n_tot;
    double tf = 0.0, tb = 0.0;
    int rc = APXB_OK;
    for (int r = 0; r < reps && rc == APXB_OK; ++r) {
        APXB_CK(cudaEventRecord(ev[0], s));
        for (int dir = 0; dir < 2; ++dir) {
            bt->sweep_dir(dir, a);
            apxb::launch_sweep32_batch(dir, a, bt->grid32, s);
            APXB_CK(cudaEventRecord(ev[dir + 1], s));
        }
        APXB_CK(cudaEventSynchronize(ev[2]));
        float m0 = 0.0f, m1 = 0.0f;
        cudaEventElapsedTime(&m0, ev[0], ev[1]);
        cudaEventElapsedTime(&m1, ev[1], ev[2]);
        tf += m0 * 1e-3; tb += m1 * 1e-3;
        rc = e->take_error();
    }
    for (auto& v : ev) cudaEventDestroy(v);
    if (rc) { bt->y_armed = false; cudaMemsetAsync(bt->ctl, 0, 2 * sizeof(apxb::sweep_ctl), s); return rc; }
    *fwd_seconds = tf / reps;
    *bck_seconds = tb / reps;
    return APXB_OK;
}

}  // extern "C"
