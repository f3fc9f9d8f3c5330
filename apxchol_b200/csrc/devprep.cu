// Factor preparation on the device: the admission path of a factor.
//
// The same arrays as the host preparation (host_prep.cpp: prepare_factor,
// build_plan, build_batch_plan, permute_operator), byte for byte, built by
// kernels from the factor as the reference's setup phase hands it over (CSC,
// diagonal first, rows ascending; perm; per-round independent-set sizes) --
// the work the reference does on the host before its upload (cuda.h:280-420,
// cuda_host.h:66-558, pcg_cuda.h:304-404).
//
// Stages (stream-ordered on the engine stream; the host waits only for sizes):
//   validate         every column: diagonal first, rows ascending and < n,
//                    positive finite diagonal; perm a bijection
//   L11 + drop       one thread per column: the column scale, the keep count,
//                    then (after a scan) the compacted column with the
//                    dropped mass spread over the kept off-diagonals -- the
//                    host's per-column arithmetic in the host's order, every
//                    product and sum rounded on its own (factor_drop.h:131-211)
//   transpose        CSC(L11) -> CSR(L11): row counts, scan, scatter, then
//                    each row sorted by column (rows of <= 32 entries by one
//                    thread, longer ones by a block-wide bitonic network)
//   levels           round-as-level: rounds are contiguous ranges of the
//                    elimination order, so a row's level is a search in the
//                    round bounds and every level is a contiguous row range
//   plans            rows grouped by (level, lane class) with per-class prefix
//                    counts (a stable counting sort without atomics), items of
//                    up to 32 rows, entry offsets by a scan, entries re-laid
//                    by one thread per row; the per-item tables (info, chunk)
//                    come from per-group counts on the host
// Factors without round sizes (topological levels), with fp16 storage or with
// the optional serial segment keep the host path.
#include <algorithm>
#include <cstdlib>
#include <functional>
#include <numeric>

#include "objects.hpp"

namespace apxb {
namespace {

constexpr int kPT = 256;                  // threads of the per-element kernels
constexpr uint32_t kScanPerBlock = 2048;  // elements per block of the scan (kPT x 8)

int grid_for(size_t n, int per_block = kPT) {
    const size_t b = (n + per_block - 1) / per_block;
    return static_cast<int>(std::max<size_t>(1, std::min<size_t>(b, 1u << 20)));
}

// ---------------------------------------------------------------- scan

// Exclusive scan of in[0, n) into out[0, n) (out may alias in), u32 sums.
__global__ void __launch_bounds__(kPT) k_scan_block(const uint32_t* in, uint32_t* out, size_t n, uint32_t* block_sum) {
    __shared__ uint32_t warp_tot[kPT / 32];
    const size_t base = static_cast<size_t>(blockIdx.x) * kScanPerBlock + threadIdx.x * 8u;
    uint32_t v[8];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        v[i] = base + i < n ? in[base + i] : 0u;
        sum += v[i];
    }
    // block-wide exclusive scan of the thread sums
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= static_cast<unsigned>(o)) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kPT / 32 ? warp_tot[lane] : 0u, wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(kFull, wi, o);
            if (lane >= static_cast<unsigned>(o)) wi += t;
        }
        if (lane < kPT / 32) warp_tot[lane] = wi - w;
        if (lane == kPT / 32 - 1) block_sum[blockIdx.x] = wi;
    }
    __syncthreads();
    uint32_t run = warp_tot[warp] + incl - sum;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

__global__ void __launch_bounds__(kPT) k_scan_add(uint32_t* out, size_t n, const uint32_t* block_off) {
    const size_t base = static_cast<size_t>(blockIdx.x) * kScanPerBlock;
    const uint32_t add = block_off[blockIdx.x];
    for (uint32_t i = threadIdx.x; i < kScanPerBlock; i += kPT)
        if (base + i < n) out[base + i] += add;
}

// Device workspace that frees itself (stream-ordered allocator).
struct dbuf {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    dbuf() = default;
    dbuf(const dbuf&) = delete;
    dbuf& operator=(const dbuf&) = delete;
    ~dbuf() { if (p) cudaFreeAsync(p, s); }
    template <class T>
    T* get() const { return static_cast<T*>(p); }
    cudaError_t alloc(size_t bytes, cudaStream_t st) {
        s = st;
        int dev = 0;
        const cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        cudaMemPool_t pool = device_pool(dev);   // the library's pool, else the device's default one
        return pool ? cudaMallocFromPoolAsync(&p, bytes ? bytes : 16, pool, st) : cudaMallocAsync(&p, bytes ? bytes : 16, st);
    }
};

// out[i] = sum of in[0, i) for i < n (in and out may alias).
cudaError_t exclusive_scan(const uint32_t* in, uint32_t* out, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const size_t nb = (n + kScanPerBlock - 1) / kScanPerBlock;
    dbuf sums;
    cudaError_t e = sums.alloc(nb * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    k_scan_block<<<static_cast<unsigned>(nb), kPT, 0, s>>>(in, out, n, sums.get<uint32_t>());
    if (nb > 1) {
        e = exclusive_scan(sums.get<uint32_t>(), sums.get<uint32_t>(), nb, s);
        if (e != cudaSuccess) return e;
        k_scan_add<<<static_cast<unsigned>(nb), kPT, 0, s>>>(out, n, sums.get<uint32_t>());
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------- segmented sort

// Each segment [ptr[i], ptr[i+1]) of (key, val) sorted by key ascending (keys
// of a segment are distinct). Segments of <= 32 entries: one thread each,
// insertion sort; longer ones are listed in `longs` for k_sort_long.
template <class V>
__global__ void __launch_bounds__(kPT) k_sort_short(const uint32_t* ptr, uint32_t nseg, uint32_t* key, V* val,
                                                    uint32_t* longs, uint32_t* n_longs) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nseg; i += gridDim.x * blockDim.x) {
        const uint32_t b = ptr[i], e = ptr[i + 1];
        if (e - b > 32u) {
            longs[atomicAdd(n_longs, 1u)] = i;
            continue;
        }
        for (uint32_t p = b + 1; p < e; ++p) {
            const uint32_t k = key[p];
            const V v = val[p];
            uint32_t q = p;
            while (q > b && key[q - 1] > k) {
                key[q] = key[q - 1];
                val[q] = val[q - 1];
                --q;
            }
            key[q] = k;
            val[q] = v;
        }
    }
}

// One block per long segment: a bitonic network in the "flip" form (every
// comparator ascending), so the segment is padded virtually with +infinity
// to the next power of two and a comparator whose upper end lies past the
// segment does nothing.
template <class V>
__global__ void __launch_bounds__(1024) k_sort_long(const uint32_t* ptr, const uint32_t* longs, const uint32_t* n_longs,
                                                    uint32_t* key, V* val) {
    for (uint32_t li = blockIdx.x; li < *n_longs; li += gridDim.x) {
        const uint32_t s = longs[li];
        const uint32_t b = ptr[s], len = ptr[s + 1] - b;
        uint32_t P = 1;
        while (P < len) P <<= 1;
        uint32_t* k = key + b;
        V* v = val + b;
        auto cmpswap = [&](uint32_t i, uint32_t j) {
            if (j < len && k[i] > k[j]) {
                const uint32_t tk = k[i]; k[i] = k[j]; k[j] = tk;
                const V tv = v[i]; v[i] = v[j]; v[j] = tv;
            }
        };
        for (uint32_t w = 2; w <= P; w <<= 1) {
            for (uint32_t t = threadIdx.x; t < P / 2; t += blockDim.x) {
                const uint32_t half = w >> 1, blk = (t / half) * w, off = t % half;
                cmpswap(blk + off, blk + w - 1 - off);
            }
            __syncthreads();
            for (uint32_t h = w >> 2; h >= 1; h >>= 1) {
                for (uint32_t t = threadIdx.x; t < P / 2; t += blockDim.x) {
                    const uint32_t blk = (t / h) * 2 * h, i = blk + t % h;
                    cmpswap(i, i + h);
                }
                __syncthreads();
            }
        }
        __syncthreads();
    }
}

template <class V>
cudaError_t segmented_sort(const uint32_t* ptr, uint32_t nseg, uint32_t* key, V* val, cudaStream_t s) {
    if (nseg == 0) return cudaSuccess;
    dbuf longs, cnt;
    cudaError_t e = longs.alloc(sizeof(uint32_t) * nseg, s);
    if (e == cudaSuccess) e = cnt.alloc(sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    cudaMemsetAsync(cnt.p, 0, sizeof(uint32_t), s);
    k_sort_short<V><<<grid_for(nseg), kPT, 0, s>>>(ptr, nseg, key, val, longs.get<uint32_t>(), cnt.get<uint32_t>());
    k_sort_long<V><<<296, 1024, 0, s>>>(ptr, longs.get<uint32_t>(), cnt.get<uint32_t>(), key, val);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- validation

// First failing column (smallest j) and its failed check, as (j << 3 | code):
// 1 empty column, 2 diagonal not first, 3 rows not ascending / out of range,
// 4 non-positive or non-finite diagonal.
__global__ void __launch_bounds__(kPT) k_validate(uint32_t n, const uint32_t* colptr, const uint32_t* rowidx,
                                                  const float* vals, unsigned long long* first_bad) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t b = colptr[j], e = colptr[j + 1];
        unsigned code = 0;
        if (e <= b) code = 1;
        else if (rowidx[b] != j) code = 2;
        else {
            for (uint32_t p = b + 1; p < e && !code; ++p)
                if (rowidx[p] <= rowidx[p - 1] || rowidx[p] >= n) code = 3;
            if (!code && !(vals[b] > 0.0f && isfinite(vals[b]))) code = 4;
        }
        if (code) atomicMin(first_bad, (static_cast<unsigned long long>(j) << 3) | code);
    }
}

// perm must be a bijection of [0, n): seen[] counts the hits of every position.
__global__ void __launch_bounds__(kPT) k_perm_check(uint32_t n, const uint32_t* perm, uint32_t* seen, uint32_t* bad) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t p = perm[v];
        if (p >= n || atomicAdd(&seen[p], 1u) != 0u) *bad = 1u;
    }
}

// ---------------------------------------------------------------- L11 + drop

struct col_view {
    uint32_t n, m;
    bool sddm;
    const uint32_t* colptr;
    const uint32_t* rowidx;
    const float* vals;
    __device__ __forceinline__ uint32_t end(uint32_t j) const {
        uint32_t e = colptr[j + 1];
        if (!sddm && e > colptr[j] + 1 && rowidx[e - 1] == n - 1) --e;   // L11: without row n-1
        return e;
    }
};

// |v| >= rel * s (in double) and v != 0: the fp32 storage keep rule.
__device__ __forceinline__ bool keep_dev(float v, float s, double rel) {
    return fabs(static_cast<double>(v)) >= __dmul_rn(rel, static_cast<double>(s)) && v != 0.0f;
}

// The column scale (max |off-diagonal| in double, stored fp32; 1 without
// off-diagonals) and the kept count; nnz of L11 summed into *nf.
__global__ void __launch_bounds__(kPT) k_drop_count(col_view c, double rel, float* col_s, uint32_t* cnt,
                                                    unsigned long long* nf) {
    unsigned long long local = 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < c.m; j += gridDim.x * blockDim.x) {
        const uint32_t b = c.colptr[j], e = c.end(j);
        local += e - b;
        float s = 1.0f;
        uint32_t k = e - b;
        if (rel > 0.0) {
            double mx = 0.0;
            for (uint32_t p = b + 1; p < e; ++p) mx = fmax(mx, fabs(static_cast<double>(c.vals[p])));
            s = mx > 0.0 ? static_cast<float>(mx) : 1.0f;
            k = 1;
            for (uint32_t p = b + 1; p < e; ++p) k += keep_dev(c.vals[p], s, rel) ? 1u : 0u;
        }
        col_s[j] = s;
        cnt[j] = k;
    }
    if (local) atomicAdd(nf, local);
}

// The compacted column at csc_ptr[j], the dropped mass spread over the kept
// off-diagonals: v += (dropped_sum / kept_abs) * |v| (double, each operation
// rounded on its own, in the column's order).
__global__ void __launch_bounds__(kPT) k_drop_write(col_view c, double rel, const float* col_s, const uint32_t* cp,
                                                    uint32_t* ci, float* cv, unsigned long long* dropped) {
    unsigned long long local = 0, flush = 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < c.m; j += gridDim.x * blockDim.x) {
        const uint32_t b = c.colptr[j], e = c.end(j), first = cp[j];
        uint32_t o = first;
        if (rel > 0.0) {
            const float s = col_s[j];
            double dropped_sum = 0.0, kept_abs = 0.0;
            for (uint32_t p = b; p < e; ++p) {
                const float v = c.vals[p];
                if (p != b) {
                    if (!keep_dev(v, s, rel)) {
                        if (fabs(static_cast<double>(v)) >= __dmul_rn(rel, static_cast<double>(s))) ++flush;
                        dropped_sum = __dadd_rn(dropped_sum, static_cast<double>(v));
                        ++local;
                        continue;
                    }
                    kept_abs = __dadd_rn(kept_abs, fabs(static_cast<double>(v)));
                }
                ci[o] = c.rowidx[p];
                cv[o] = v;
                ++o;
            }
            if (dropped_sum != 0.0 && kept_abs > 0.0) {
                const double per_abs = __ddiv_rn(dropped_sum, kept_abs);
                for (uint32_t q = first + 1; q < o; ++q) {
                    const double v = static_cast<double>(cv[q]);
                    cv[q] = __double2float_rn(__dadd_rn(v, __dmul_rn(per_abs, fabs(v))));
                }
            }
        } else {
            for (uint32_t p = b; p < e; ++p) { ci[o] = c.rowidx[p]; cv[o] = c.vals[p]; ++o; }
        }
    }
    if (local) atomicAdd(dropped, local);
    if (flush) atomicAdd(dropped + 1, flush);
}

// ---------------------------------------------------------------- transpose

__global__ void __launch_bounds__(kPT) k_row_count(const uint32_t* ci, size_t nnz, uint32_t* len) {
    for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < nnz;
         p += static_cast<size_t>(gridDim.x) * blockDim.x)
        atomicAdd(&len[ci[p]], 1u);
}

// Each column's entries into their rows (any order inside a row; sorted after).
__global__ void __launch_bounds__(kPT) k_row_scatter(uint32_t m, const uint32_t* cp, const uint32_t* ci, const float* cv,
                                                     uint32_t* cursor, uint32_t* ri, float* rv) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
        for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) {
            const uint32_t slot = atomicAdd(&cursor[ci[p]], 1u);
            ri[slot] = j;
            rv[slot] = cv[p];
        }
}

// ---------------------------------------------------------------- levels

// Forward level of row c: the round holding it (last round bound <= c), or
// n_rounds + (c - last) for the trailing columns past the last round.
__global__ void __launch_bounds__(kPT) k_levels(uint32_t m, const uint64_t* bounds, uint32_t n_rounds, int32_t* fl) {
    const uint64_t last = bounds[n_rounds];
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < m; c += gridDim.x * blockDim.x) {
        if (c >= last) { fl[c] = static_cast<int32_t>(n_rounds + (c - last)); continue; }
        uint32_t lo = 0, hi = n_rounds;   // largest r < n_rounds with bounds[r] <= c
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (bounds[mid] <= c) lo = mid; else hi = mid - 1;
        }
        fl[c] = static_cast<int32_t>(lo < n_rounds ? lo : n_rounds - 1);
    }
}

// ---------------------------------------------------------------- plans

// Lane class of row r in a plan: factor plans (G = 32, 16, 8, 4, 1 -> 0..4) or
// batch plans (G = 32 >> c, G >= col_lanes).
__device__ __forceinline__ uint32_t class_of(uint32_t len, uint32_t col_lanes) {
    if (col_lanes == 0) {
        if (len <= 8) return 4;
        uint32_t g = 4;
        while (g < 32 && g * 8 < len) g *= 2;
        return 5 - __ffs(g) + 1;   // 5 - log2(g)
    }
    uint32_t ge = 1;
    while (ge * col_lanes < 32 && ge * 8 < len) ge *= 2;
    return 5 - (__ffs(ge * col_lanes) - 1);
}

// Class flags of every row for the per-class prefix counts: flag[c * (m+1) + r].
__global__ void __launch_bounds__(kPT) k_class_flags(uint32_t m, const uint32_t* ptr, uint32_t col_lanes, uint32_t n_cls,
                                                     uint8_t* cls, uint32_t* flag) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= m; r += gridDim.x * blockDim.x) {
        const uint32_t c = r < m ? class_of(ptr[r + 1] - ptr[r] - 1, col_lanes) : n_cls;
        if (r < m) cls[r] = static_cast<uint8_t>(c);
        for (uint32_t k = 0; k < n_cls; ++k) flag[static_cast<size_t>(k) * (m + 1) + r] = c == k ? 1u : 0u;
    }
}

// Prefix counts at the forward level bounds: out[l * n_cls + c] = pre_c[B_l].
__global__ void k_gather_bounds(const uint32_t* pre, uint32_t m, uint32_t n_cls, const uint32_t* lb, uint32_t n_lb,
                                uint32_t* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_lb * n_cls; i += gridDim.x * blockDim.x) {
        const uint32_t l = i / n_cls, c = i % n_cls;
        out[i] = pre[static_cast<size_t>(c) * (m + 1) + lb[l]];
    }
}

struct plan_geo {
    uint32_t m, n_cls;
    int32_t maxd;
    int forward;
    const int32_t* fl;          // forward level of every row
    const uint32_t* lb;         // forward level bounds B_l (rows [B_l, B_{l+1}))
    const uint32_t* pre;        // per-class prefix counts, [n_cls][m+1]
    const uint8_t* cls;
    const uint32_t* base;       // first item of group (direction level l', class c): [l' * n_cls + c]
};

__device__ __forceinline__ uint32_t cap_of(uint32_t c, bool factor_plan) {
    const uint32_t lg = factor_plan ? (c == 4 ? 0u : 5u - c) : 5u - c;
    return 32u >> lg;
}

// Row r's position (item * 32 + slot) and its entry count.
__global__ void __launch_bounds__(kPT) k_plan_rows(plan_geo g, bool factor_plan, const uint32_t* ptr, uint32_t* ord,
                                                   uint32_t* poslen, uint32_t* rowpos) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < g.m; r += gridDim.x * blockDim.x) {
        const int32_t l = g.fl[r];
        const uint32_t ld = static_cast<uint32_t>(g.forward ? l : g.maxd - l);
        const uint32_t c = g.cls[r];
        const uint32_t rank = g.pre[static_cast<size_t>(c) * (g.m + 1) + r] - g.pre[static_cast<size_t>(c) * (g.m + 1) + g.lb[l]];
        const uint32_t cap = cap_of(c, factor_plan);
        const size_t pos = static_cast<size_t>(g.base[static_cast<size_t>(ld) * g.n_cls + c] + rank / cap) * 32 + rank % cap;
        ord[pos] = r;
        poslen[pos] = ptr[r + 1] - ptr[r];
        rowpos[r] = static_cast<uint32_t>(pos);
    }
}

// Entries of row r at its plan offset, the diagonal last. Forward rows
// (CSR(L11), diagonal last) keep their order. Backward rows (CSC(L11),
// diagonal first): factor plans take the off-diagonals in order; batch plans
// take them oldest dependency first -- by backward level, then index -- which
// is the runs of equal forward level in reverse run order (forward levels grow
// with the index), each run kept ascending.
__global__ void __launch_bounds__(kPT) k_plan_fill(uint32_t m, int forward, bool batch_order, const int32_t* fl,
                                                   const uint32_t* ptr, const uint32_t* idx, const float* val,
                                                   const uint32_t* rowpos, const uint32_t* pptr, uint32_t* pidx,
                                                   float* pval) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x) {
        const uint32_t b = ptr[r], en = ptr[r + 1];
        uint32_t e = pptr[rowpos[r]];
        if (forward) {
            for (uint32_t p = b; p < en; ++p) { pidx[e] = idx[p]; pval[e] = val[p]; ++e; }
            continue;
        }
        if (!batch_order) {
            for (uint32_t p = b + 1; p < en; ++p) { pidx[e] = idx[p]; pval[e] = val[p]; ++e; }
        } else {
            uint32_t hi = en;   // runs [lo, hi) of equal forward level, from the end
            while (hi > b + 1) {
                uint32_t lo = hi - 1;
                const int32_t lv = fl[idx[lo]];
                while (lo > b + 1 && fl[idx[lo - 1]] == lv) --lo;
                for (uint32_t p = lo; p < hi; ++p) { pidx[e] = idx[p]; pval[e] = val[p]; ++e; }
                hi = lo;
            }
        }
        pidx[e] = idx[b];
        pval[e] = val[b];
    }
}

// ---------------------------------------------------------------- operator

__global__ void __launch_bounds__(kPT) k_op_lengths(uint32_t n, const int32_t* colptr, const uint32_t* perm, uint32_t* len,
                                                    uint32_t* bad) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        if (colptr[j + 1] < colptr[j]) { *bad = 2u; continue; }
        len[perm[j]] = static_cast<uint32_t>(colptr[j + 1] - colptr[j]);
    }
}

// Row perm[j] of P A P^T: column j's entries (A symmetric), columns mapped through perm.
__global__ void __launch_bounds__(kPT) k_op_scatter(uint32_t n, const int32_t* colptr, const int32_t* rowidx,
                                                    const double* vals, const uint32_t* perm, const uint32_t* ptr,
                                                    uint32_t* idx, double* val, uint32_t* bad) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        uint32_t o = ptr[perm[j]];
        for (int32_t p = colptr[j]; p < colptr[j + 1]; ++p) {
            const int32_t r = rowidx[p];
            if (r < 0 || static_cast<uint32_t>(r) >= n) { *bad = 3u; idx[o] = 0; val[o] = 0.0; ++o; continue; }
            idx[o] = perm[r];
            val[o] = vals[p];
            ++o;
        }
    }
}

// Clears *exact unless every value round-trips fp32: v == double(float(v))
// (the reference's fp32_exact test, pcg_cuda.h:298-380).
__global__ void __launch_bounds__(kPT) k_fp32_exact(const double* v, size_t n, uint32_t* inexact) {
    bool bad = false;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const double x = v[i];
        if (static_cast<double>(__double2float_rn(x)) != x) bad = true;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31u) == 0) atomicOr(inexact, 1u);
}

__global__ void __launch_bounds__(kPT) k_narrow(const double* v, float* f, size_t n) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        f[i] = __double2float_rn(v[i]);
}

}  // namespace

// ================================================================ host side

namespace {

#define DP_CK(call)                                                                              \
    do {                                                                                         \
        const cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                                   \
            return std::string("device preparation: ") + #call + ": " + cudaGetErrorString(e_); \
    } while (0)

template <class T>
std::string upload(dbuf& d, const T* h, size_t count, cudaStream_t s) {
    DP_CK(d.alloc(sizeof(T) * count, s));
    DP_CK(cudaMemcpyAsync(d.p, h, sizeof(T) * count, cudaMemcpyHostToDevice, s));
    return {};
}

// Host tables of one plan from the per-(level, class) row counts: the first
// item of every group, the item words, the chunk table (chunk_plan's rule:
// per level, chunks of max(1, min(8, items / 4096)) items).
struct plan_tables {
    uint32_t n_items = 0;
    std::vector<uint32_t> base, info, chunk;
};

void make_tables(const std::vector<uint32_t>& counts /* [fwd level][cls] */, int32_t n_levels, uint32_t n_cls,
                 bool forward, bool factor_plan, const std::vector<uint8_t>& thin_level, plan_tables& t) {
    t.base.assign(static_cast<size_t>(n_levels) * n_cls, 0);
    t.info.clear();
    t.chunk.clear();
    uint32_t items = 0;
    for (int32_t ld = 0; ld < n_levels; ++ld) {
        const int32_t l = forward ? ld : n_levels - 1 - ld;
        const uint32_t level_first = items;
        for (uint32_t c = 0; c < n_cls; ++c) {
            const uint32_t g = counts[static_cast<size_t>(l) * n_cls + c];
            const uint32_t lg = factor_plan ? (c == 4 ? 0u : 5u - c) : 5u - c, cap = 32u >> lg;
            t.base[static_cast<size_t>(ld) * n_cls + c] = items;
            for (uint32_t q = 0; q < g; q += cap) {
                uint32_t w = std::min(cap, g - q) | (lg << 8);
                if (factor_plan) w |= static_cast<uint32_t>(thin_level[l]) << 16;
                t.info.push_back(w);
                ++items;
            }
        }
        const uint32_t in_level = items - level_first;
        const uint32_t per = std::max(1u, std::min(8u, in_level / 4096u));
        for (uint32_t s = level_first; s < items; s += per) t.chunk.push_back(s);
    }
    t.chunk.push_back(items);
    t.n_items = items;
}

}  // namespace

// One direction's plan (factor plan: col_lanes == 0; else a batch plan) from
// the canonical device arrays of the direction. Writes the device arrays into
// the caller's buffers, allocated through `alloc`.

template <class Alloc>
std::string build_plan_dev(uint32_t m, int dir, uint32_t col_lanes, int32_t n_levels, const int32_t* d_fl,
                           const uint32_t* d_lb, const uint32_t* d_ptr, const uint32_t* d_idx, const float* d_val,
                           const std::vector<uint8_t>& thin_level, Alloc&& alloc, dev_plan_out& out, cudaStream_t s) {
    const bool factor_plan = col_lanes == 0;
    uint32_t n_cls = 5;
    if (!factor_plan) {
        n_cls = 1;
        while ((32u >> (n_cls - 1)) > col_lanes) ++n_cls;
    }
    dbuf cls, pre, cnt;
    DP_CK(cls.alloc(m, s));
    DP_CK(pre.alloc(sizeof(uint32_t) * n_cls * (static_cast<size_t>(m) + 1), s));
    k_class_flags<<<grid_for(static_cast<size_t>(m) + 1), kPT, 0, s>>>(m, d_ptr, col_lanes, n_cls, cls.get<uint8_t>(),
                                                                       pre.get<uint32_t>());
    for (uint32_t c = 0; c < n_cls; ++c)
        DP_CK(exclusive_scan(pre.get<uint32_t>() + static_cast<size_t>(c) * (m + 1),
                             pre.get<uint32_t>() + static_cast<size_t>(c) * (m + 1), static_cast<size_t>(m) + 1, s));
    // per-(level, class) counts
    const uint32_t n_lb = static_cast<uint32_t>(n_levels) + 1;
    DP_CK(cnt.alloc(sizeof(uint32_t) * n_lb * n_cls, s));
    k_gather_bounds<<<grid_for(static_cast<size_t>(n_lb) * n_cls), kPT, 0, s>>>(pre.get<uint32_t>(), m, n_cls, d_lb, n_lb,
                                                                               cnt.get<uint32_t>());
    std::vector<uint32_t> at(static_cast<size_t>(n_lb) * n_cls);
    DP_CK(cudaMemcpyAsync(at.data(), cnt.p, 4 * at.size(), cudaMemcpyDeviceToHost, s));
    DP_CK(cudaStreamSynchronize(s));
    std::vector<uint32_t> counts(static_cast<size_t>(n_levels) * n_cls);
    for (int32_t l = 0; l < n_levels; ++l)
        for (uint32_t c = 0; c < n_cls; ++c)
            counts[static_cast<size_t>(l) * n_cls + c] = at[static_cast<size_t>(l + 1) * n_cls + c] - at[static_cast<size_t>(l) * n_cls + c];
    plan_tables t;
    make_tables(counts, n_levels, n_cls, dir == 0, factor_plan, thin_level, t);
    const size_t npos = static_cast<size_t>(t.n_items) * 32;
    dbuf base, poslen, rowpos;
    std::string err;
    if (!(err = upload(base, t.base.data(), t.base.size(), s)).empty()) return err;
    DP_CK(poslen.alloc(sizeof(uint32_t) * (npos + 1), s));
    DP_CK(rowpos.alloc(sizeof(uint32_t) * std::max<size_t>(m, 1), s));
    out = dev_plan_out{};
    out.n_items = t.n_items;
    out.n_chunks = static_cast<uint32_t>(t.chunk.size() - 1);
    if (!(err = alloc(&out.info, t.info.size())).empty() || !(err = alloc(&out.ord, npos)).empty() ||
        !(err = alloc(&out.ptr, npos + 1)).empty() || !(err = alloc(&out.chunk, t.chunk.size())).empty())
        return err;
    DP_CK(cudaMemcpyAsync(out.info, t.info.data(), 4 * t.info.size(), cudaMemcpyHostToDevice, s));
    DP_CK(cudaMemcpyAsync(out.chunk, t.chunk.data(), 4 * t.chunk.size(), cudaMemcpyHostToDevice, s));
    DP_CK(cudaMemsetAsync(out.ord, 0xff, 4 * npos, s));
    DP_CK(cudaMemsetAsync(poslen.p, 0, 4 * (npos + 1), s));
    plan_geo g{m, n_cls, n_levels - 1, dir == 0, d_fl, d_lb, pre.get<uint32_t>(), cls.get<uint8_t>(), base.get<uint32_t>()};
    k_plan_rows<<<grid_for(m), kPT, 0, s>>>(g, factor_plan, d_ptr, out.ord, poslen.get<uint32_t>(), rowpos.get<uint32_t>());
    DP_CK(exclusive_scan(poslen.get<uint32_t>(), out.ptr, npos + 1, s));
    uint32_t total = 0;
    DP_CK(cudaMemcpyAsync(&total, out.ptr + npos, 4, cudaMemcpyDeviceToHost, s));
    DP_CK(cudaStreamSynchronize(s));
    out.n_entries = total;
    if (!(err = alloc(&out.idx, total)).empty() || !(err = alloc(&out.val, total)).empty()) return err;
    k_plan_fill<<<grid_for(m), kPT, 0, s>>>(m, dir == 0, !factor_plan, d_fl, d_ptr, d_idx, d_val, rowpos.get<uint32_t>(),
                                            out.ptr, out.idx, out.val);
    DP_CK(cudaGetLastError());
    return {};
}


// ---------------------------------------------------------------- factor

bool device_prep_applies(bool fp16, uint32_t n_rounds) {
    if (fp16 || n_rounds == 0) return false;
    if (const char* e = std::getenv("APXB_HOST_PREP"))
        if (*e && *e != '0') return false;
    if (const char* e = std::getenv("APXB_SEG_LEVEL_ROWS"))   // the serial segment is built on the host
        if (std::atoi(e) > 0) return false;
    return kSegLevelRows == 0;
}

std::string prepare_factor_device(apxb_factor* f, uint32_t n, const uint32_t* colptr, const uint32_t* rowidx,
                                  const float* vals, const uint32_t* perm, bool sddm, const uint64_t* rounds,
                                  uint32_t n_rounds, double drop_rel, int* alloc_rc) {
    cudaStream_t s = f->e->stream;
    prepared_factor& h = f->h;
    if (n == 0) return "empty factor";
    if (!sddm && n < 2) return "a Laplacian factor needs n >= 2";
    if (colptr[0] != 0) return "colptr[0] != 0";
    const uint32_t m = sddm ? n : n - 1;
    const double rel = drop_rel < 0.0 ? kDropRelDefault : drop_rel;
    h = prepared_factor{};
    h.n = n; h.m = m; h.sddm = sddm; h.fp16 = false;
    auto falloc = [&](auto** q, size_t count) -> std::string {
        const int rc = f->dalloc(q, std::max<size_t>(count, 1));
        if (rc) *alloc_rc = rc;
        return rc ? std::string(apxb_last_error()) : std::string();
    };
    std::string err;
    // ---- upload and validate
    const size_t nnz_in = colptr[n];   // a non-monotone colptr fails the per-column checks below
    {
        for (uint32_t j = 0; j < n; ++j)   // the kernels index entries through colptr: bound it first
            if (colptr[j + 1] < colptr[j]) return "column " + std::to_string(j) + " is empty (no diagonal)";
    }
    dbuf d_cp, d_ri, d_va, d_perm, d_bad, d_seen;
    if (!(err = upload(d_cp, colptr, static_cast<size_t>(n) + 1, s)).empty() ||
        !(err = upload(d_ri, rowidx, nnz_in, s)).empty() || !(err = upload(d_va, vals, nnz_in, s)).empty() ||
        !(err = upload(d_perm, perm, n, s)).empty())
        return err;
    DP_CK(d_bad.alloc(16, s));
    DP_CK(d_seen.alloc(4 * static_cast<size_t>(n), s));
    DP_CK(cudaMemsetAsync(d_bad.p, 0xff, 8, s));
    DP_CK(cudaMemsetAsync(static_cast<char*>(d_bad.p) + 8, 0, 8, s));
    DP_CK(cudaMemsetAsync(d_seen.p, 0, 4 * static_cast<size_t>(n), s));
    k_validate<<<grid_for(n), kPT, 0, s>>>(n, d_cp.get<uint32_t>(), d_ri.get<uint32_t>(), d_va.get<float>(),
                                           d_bad.get<unsigned long long>());
    k_perm_check<<<grid_for(n), kPT, 0, s>>>(n, d_perm.get<uint32_t>(), d_seen.get<uint32_t>(),
                                             reinterpret_cast<uint32_t*>(static_cast<char*>(d_bad.p) + 8));
    unsigned long long bad[2] = {0, 0};
    DP_CK(cudaMemcpyAsync(bad, d_bad.p, 16, cudaMemcpyDeviceToHost, s));
    DP_CK(cudaStreamSynchronize(s));
    if (bad[0] != ~0ull) {
        const std::string col = "column " + std::to_string(bad[0] >> 3);
        switch (bad[0] & 7u) {
            case 1: return col + " is empty (no diagonal)";
            case 2: return col + " does not start with its diagonal";
            case 3: return col + " rows not ascending / out of range";
            default: return col + " has a non-positive or non-finite diagonal";
        }
    }
    // ---- L11 and the compacting drop
    const col_view cv{n, m, sddm, d_cp.get<uint32_t>(), d_ri.get<uint32_t>(), d_va.get<float>()};
    dbuf d_cs, d_cnt, d_stat;
    DP_CK(d_cs.alloc(4 * static_cast<size_t>(m), s));
    DP_CK(d_stat.alloc(24, s));
    DP_CK(cudaMemsetAsync(d_stat.p, 0, 24, s));
    uint32_t* cp = nullptr;
    if (!(err = falloc(&cp, static_cast<size_t>(m) + 1)).empty()) return err;
    DP_CK(cudaMemsetAsync(cp + m, 0, 4, s));
    k_drop_count<<<grid_for(m), kPT, 0, s>>>(cv, rel, d_cs.get<float>(), cp, d_stat.get<unsigned long long>());
    unsigned long long nf = 0;
    DP_CK(cudaMemcpyAsync(&nf, d_stat.p, 8, cudaMemcpyDeviceToHost, s));
    DP_CK(cudaStreamSynchronize(s));
    if (nf >= 0xffffffffull) return "factor nnz exceeds the 32-bit offset range";
    DP_CK(exclusive_scan(cp, cp, static_cast<size_t>(m) + 1, s));
    uint32_t nnz = 0;
    DP_CK(cudaMemcpyAsync(&nnz, cp + m, 4, cudaMemcpyDeviceToHost, s));
    DP_CK(cudaStreamSynchronize(s));
    uint32_t* ci = nullptr;
    float* cval = nullptr;
    if (!(err = falloc(&ci, nnz)).empty() || !(err = falloc(&cval, nnz)).empty()) return err;
    k_drop_write<<<grid_for(m), kPT, 0, s>>>(cv, rel, d_cs.get<float>(), cp, ci, cval,
                                             d_stat.get<unsigned long long>() + 1);
    // ---- CSC -> CSR, columns ascending in every row
    uint32_t* rp = nullptr;
    uint32_t* ri = nullptr;
    float* rval = nullptr;
    if (!(err = falloc(&rp, static_cast<size_t>(m) + 1)).empty() || !(err = falloc(&ri, nnz)).empty() ||
        !(err = falloc(&rval, nnz)).empty())
        return err;
    DP_CK(cudaMemsetAsync(rp, 0, 4 * (static_cast<size_t>(m) + 1), s));
    k_row_count<<<grid_for(nnz), kPT, 0, s>>>(ci, nnz, rp);
    DP_CK(exclusive_scan(rp, rp, static_cast<size_t>(m) + 1, s));
    {
        dbuf cursor;
        DP_CK(cursor.alloc(4 * static_cast<size_t>(m), s));
        DP_CK(cudaMemcpyAsync(cursor.p, rp, 4 * static_cast<size_t>(m), cudaMemcpyDeviceToDevice, s));
        k_row_scatter<<<grid_for(m), kPT, 0, s>>>(m, cp, ci, cval, cursor.get<uint32_t>(), ri, rval);
        DP_CK(segmented_sort<float>(rp, m, ri, rval, s));
    }
    // ---- levels from the round bounds (omp.h:880-932; preconditioner.h:247-258)
    std::vector<uint64_t> b(static_cast<size_t>(n_rounds) + 1, 0);
    {
        uint64_t acc = 0;
        for (uint32_t r = 0; r < n_rounds; ++r) {
            acc += rounds[r];
            if (acc > m) acc = m;
            b[r + 1] = acc;
        }
    }
    const uint64_t last = b[n_rounds];
    int32_t maxd;
    if (last < m) {
        maxd = static_cast<int32_t>(n_rounds + (m - 1 - last));
    } else {
        uint32_t r = 0;   // the level of row m - 1: the largest r < n_rounds with b[r] <= m - 1
        while (r + 1 < n_rounds && b[r + 1] <= m - 1) ++r;
        maxd = static_cast<int32_t>(r);
    }
    const int32_t n_levels = maxd + 1;
    std::vector<uint32_t> lb(static_cast<size_t>(n_levels) + 1);
    for (int32_t l = 0; l <= n_levels; ++l) {
        uint64_t v;
        if (l == n_levels) v = m;
        else if (static_cast<uint32_t>(l) < n_rounds) v = b[l];
        else v = last + (static_cast<uint64_t>(l) - n_rounds);
        lb[l] = static_cast<uint32_t>(std::min<uint64_t>(v, m));
    }
    std::vector<uint8_t> thin_level(static_cast<size_t>(n_levels));
    for (int32_t l = 0; l < n_levels; ++l) thin_level[l] = (lb[l + 1] - lb[l]) <= kThinLevelRows ? 1 : 0;
    int32_t* fl = nullptr;
    uint32_t* dlb = nullptr;
    if (!(err = falloc(&fl, m)).empty() || !(err = falloc(&dlb, lb.size())).empty()) return err;
    DP_CK(cudaMemcpyAsync(dlb, lb.data(), 4 * lb.size(), cudaMemcpyHostToDevice, s));
    {
        dbuf d_b;
        if (!(err = upload(d_b, b.data(), b.size(), s)).empty()) return err;
        k_levels<<<grid_for(m), kPT, 0, s>>>(m, d_b.get<uint64_t>(), n_rounds, fl);
        DP_CK(cudaGetLastError());
        DP_CK(cudaStreamSynchronize(s));   // d_b is freed below; the stream has used it
    }
    // ---- sweep plans of both directions
    for (int dir = 0; dir < 2; ++dir) {
        dev_plan_out o;
        auto alloc = [&](auto** q, size_t count) { return falloc(q, count); };
        err = dir == 0 ? build_plan_dev(m, 0, 0, n_levels, fl, dlb, rp, ri, rval, thin_level, alloc, o, s)
                       : build_plan_dev(m, 1, 0, n_levels, fl, dlb, cp, ci, cval, thin_level, alloc, o, s);
        if (!err.empty()) return err;
        f->info[dir] = o.info; f->ord[dir] = o.ord; f->ptr[dir] = o.ptr; f->idx[dir] = o.idx; f->val[dir] = o.val;
        f->chunk[dir] = o.chunk; f->n_chunks[dir] = o.n_chunks;
        sweep_plan& pl = dir == 0 ? h.fwd_plan : h.bck_plan;
        pl.n_items = o.n_items;
    }
    // ---- what stays: the canonical arrays (batch plans, host copies on demand), sizes, counts
    unsigned long long st[3] = {0, 0, 0};
    DP_CK(cudaMemcpyAsync(st, d_stat.p, 24, cudaMemcpyDeviceToHost, s));
    DP_CK(cudaStreamSynchronize(s));
    h.nnz_factor = st[0];
    h.nnz_stored = nnz;
    h.dropped = st[1];
    h.dropped_flush = st[2];
    h.fwd_levels = h.bck_levels = n_levels;
    h.perm.assign(perm, perm + n);
    if (bad[1]) return "perm is not a permutation of [0, n)";
    auto& d = f->dev;
    d.on = true;
    d.csc_ptr = cp; d.csc_idx = ci; d.csc_val = cval;
    d.csr_ptr = rp; d.csr_idx = ri; d.csr_val = rval;
    d.fl = fl; d.lb = dlb; d.n_levels = n_levels;
    d.thin_level = std::move(thin_level);
    f->host_arrays = false;
    if ((err = falloc(&f->perm, n)).empty())
        DP_CK(cudaMemcpyAsync(f->perm, d_perm.p, 4 * static_cast<size_t>(n), cudaMemcpyDeviceToDevice, s));
    return err;
}

// The host copies of a device-prepared factor's canonical arrays, levels and
// thin bits (what apxb_factor_arrays returns and multi-instance batch plans read).
std::string factor_host_arrays(apxb_factor* f) {
    if (f->host_arrays) return {};
    cudaStream_t s = f->e->stream;
    prepared_factor& h = f->h;
    const auto& d = f->dev;
    const uint32_t m = h.m;
    const size_t nnz = h.nnz_stored;
    h.csr_ptr.resize(static_cast<size_t>(m) + 1);
    h.csc_ptr.resize(static_cast<size_t>(m) + 1);
    h.csr_idx.resize(nnz); h.csr_val.resize(nnz); h.csc_idx.resize(nnz); h.csc_val.resize(nnz);
    h.fwd_level.resize(m);
    DP_CK(cudaMemcpyAsync(h.csr_ptr.data(), d.csr_ptr, 4 * h.csr_ptr.size(), cudaMemcpyDeviceToHost, s));
    DP_CK(cudaMemcpyAsync(h.csc_ptr.data(), d.csc_ptr, 4 * h.csc_ptr.size(), cudaMemcpyDeviceToHost, s));
    DP_CK(cudaMemcpyAsync(h.csr_idx.data(), d.csr_idx, 4 * nnz, cudaMemcpyDeviceToHost, s));
    DP_CK(cudaMemcpyAsync(h.csr_val.data(), d.csr_val, 4 * nnz, cudaMemcpyDeviceToHost, s));
    DP_CK(cudaMemcpyAsync(h.csc_idx.data(), d.csc_idx, 4 * nnz, cudaMemcpyDeviceToHost, s));
    DP_CK(cudaMemcpyAsync(h.csc_val.data(), d.csc_val, 4 * nnz, cudaMemcpyDeviceToHost, s));
    DP_CK(cudaMemcpyAsync(h.fwd_level.data(), d.fl, 4 * static_cast<size_t>(m), cudaMemcpyDeviceToHost, s));
    DP_CK(cudaStreamSynchronize(s));
    h.bck_level.resize(m);
    const int32_t maxd = d.n_levels - 1;
    for (uint32_t r = 0; r < m; ++r) h.bck_level[r] = maxd - h.fwd_level[r];
    h.fwd_thin_bits.assign((static_cast<size_t>(m) + 31) / 32, 0u);
    for (uint32_t r = 0; r < m; ++r)
        if (d.thin_level[h.fwd_level[r]]) h.fwd_thin_bits[r >> 5] |= 1u << (r & 31);
    h.bck_thin_bits = h.fwd_thin_bits;
    f->host_arrays = true;
    return {};
}

// The batch plan of direction dir for col_lanes column lanes, on the device,
// from a device-prepared factor (single-instance batches).
std::string batch_plan_device(const apxb_factor* f, int dir, uint32_t col_lanes,
                              const std::function<std::string(void**, size_t)>& alloc_bytes, dev_plan_out& out,
                              cudaStream_t s) {
    const auto& d = f->dev;
    auto alloc = [&](auto** q, size_t count) {
        return alloc_bytes(reinterpret_cast<void**>(q), sizeof(**q) * std::max<size_t>(count, 1));
    };
    const uint32_t m = f->h.m;
    std::string err = dir == 0
        ? build_plan_dev(m, 0, col_lanes, d.n_levels, d.fl, d.lb, d.csr_ptr, d.csr_idx, d.csr_val, d.thin_level, alloc, out, s)
        : build_plan_dev(m, 1, col_lanes, d.n_levels, d.fl, d.lb, d.csc_ptr, d.csc_idx, d.csc_val, d.thin_level, alloc, out, s);
    if (err.empty()) {
        const cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) err = std::string("device batch plan: ") + cudaGetErrorString(e);
    }
    return err;
}

// ---------------------------------------------------------------- operator

// P A P^T on the device (permute_operator's arrays): ptr on the host for the
// caller's long-row tables.
std::string permute_operator_device(apxb_operator* a, uint32_t n, const int32_t* colptr, const int32_t* rowidx,
                                    const double* vals, const uint32_t* perm, std::vector<int32_t>& hptr, int* alloc_rc) {
    cudaStream_t s = a->e->stream;
    if (colptr[0] != 0) return "operator colptr[0] != 0";
    const int64_t nnz = colptr[n];
    if (nnz < 0 || nnz > INT32_MAX) return "operator nnz out of the int32 range";
    for (uint32_t j = 0; j < n; ++j)
        if (colptr[j + 1] < colptr[j]) return "operator colptr not monotone";
    std::string err;
    dbuf d_cp, d_ri, d_va, d_perm, d_len, d_bad, d_seen;
    if (!(err = upload(d_cp, colptr, static_cast<size_t>(n) + 1, s)).empty() ||
        !(err = upload(d_ri, rowidx, static_cast<size_t>(nnz), s)).empty() ||
        !(err = upload(d_va, vals, static_cast<size_t>(nnz), s)).empty() || !(err = upload(d_perm, perm, n, s)).empty())
        return err;
    DP_CK(d_bad.alloc(4, s));
    DP_CK(d_seen.alloc(4 * static_cast<size_t>(n), s));
    DP_CK(cudaMemsetAsync(d_bad.p, 0, 4, s));
    DP_CK(cudaMemsetAsync(d_seen.p, 0, 4 * static_cast<size_t>(n), s));
    k_perm_check<<<grid_for(n), kPT, 0, s>>>(n, d_perm.get<uint32_t>(), d_seen.get<uint32_t>(), d_bad.get<uint32_t>());
    uint32_t bad = 0;
    DP_CK(cudaMemcpyAsync(&bad, d_bad.p, 4, cudaMemcpyDeviceToHost, s));
    DP_CK(cudaStreamSynchronize(s));
    if (bad) return "perm is not a permutation of [0, n)";
    int rc;
    if ((rc = a->dalloc(&a->ptr, static_cast<size_t>(n) + 1)) || (rc = a->dalloc(&a->idx, std::max<int64_t>(nnz, 1))) ||
        (rc = a->dalloc(&a->val, std::max<int64_t>(nnz, 1)))) {
        *alloc_rc = rc;
        return std::string(apxb_last_error());
    }
    uint32_t* ptr = reinterpret_cast<uint32_t*>(a->ptr);
    DP_CK(cudaMemsetAsync(ptr + n, 0, 4, s));
    k_op_lengths<<<grid_for(n), kPT, 0, s>>>(n, d_cp.get<int32_t>(), d_perm.get<uint32_t>(), ptr, d_bad.get<uint32_t>());
    DP_CK(exclusive_scan(ptr, ptr, static_cast<size_t>(n) + 1, s));
    k_op_scatter<<<grid_for(n), kPT, 0, s>>>(n, d_cp.get<int32_t>(), d_ri.get<int32_t>(), d_va.get<double>(),
                                             d_perm.get<uint32_t>(), ptr, reinterpret_cast<uint32_t*>(a->idx), a->val,
                                             d_bad.get<uint32_t>());
    DP_CK(segmented_sort<double>(ptr, n, reinterpret_cast<uint32_t*>(a->idx), a->val, s));
    hptr.resize(static_cast<size_t>(n) + 1);
    DP_CK(cudaMemcpyAsync(hptr.data(), ptr, 4 * hptr.size(), cudaMemcpyDeviceToHost, s));
    DP_CK(cudaMemcpyAsync(&bad, d_bad.p, 4, cudaMemcpyDeviceToHost, s));
    DP_CK(cudaStreamSynchronize(s));
    if (bad == 3u) return "operator row index out of range";
    a->nnz = static_cast<uint64_t>(nnz);
    return {};
}

std::string operator_precision_device(apxb_operator* a, int want, int* alloc_rc) {
    cudaStream_t s = a->e->stream;
    const size_t nnz = a->nnz;
    bool fp32 = want > 0;
    if (want < 0 && nnz > 0) {
        dbuf flag;
        DP_CK(flag.alloc(4, s));
        DP_CK(cudaMemsetAsync(flag.p, 0, 4, s));
        k_fp32_exact<<<grid_for(nnz), kPT, 0, s>>>(a->val, nnz, flag.get<uint32_t>());
        uint32_t inexact = 1;
        DP_CK(cudaMemcpyAsync(&inexact, flag.p, 4, cudaMemcpyDeviceToHost, s));
        DP_CK(cudaStreamSynchronize(s));
        fp32 = inexact == 0;
    }
    if (!fp32 || nnz == 0) return {};
    const int rc = a->dalloc(&a->valf, nnz);
    if (rc) {
        *alloc_rc = rc;
        return std::string(apxb_last_error());
    }
    k_narrow<<<grid_for(nnz), kPT, 0, s>>>(a->val, a->valf, nnz);
    DP_CK(cudaGetLastError());
    DP_CK(cudaStreamSynchronize(s));
    a->drop(a->val);
    a->val = nullptr;
    return {};
}

namespace {

template <class T, class V>
std::string same(const char* what, const T* dev, const V& host, size_t count, cudaStream_t s) {
    if (host.size() != count) return std::string(what) + ": sizes differ (" + std::to_string(count) + " on the device, " +
                                     std::to_string(host.size()) + " on the host)";
    std::vector<T> d(count);
    if (count) {
        const cudaError_t e = cudaMemcpyAsync(d.data(), dev, sizeof(T) * count, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return std::string(what) + ": copy failed";
    }
    for (size_t i = 0; i < count; ++i)
        if (std::memcmp(&d[i], &host[i], sizeof(T)) != 0) return std::string(what) + ": first difference at " + std::to_string(i);
    return {};
}

std::string same_plan(const char* dir, const dev_plan_out& o, const sweep_plan& pl, cudaStream_t s) {
    std::string e;
    const std::string p = std::string(dir) + " ";
    if (o.n_items != pl.n_items) return p + "item counts differ";
    if (!(e = same((p + "info").c_str(), o.info, pl.info, pl.n_items, s)).empty()) return e;
    if (!(e = same((p + "ord").c_str(), o.ord, pl.ord, static_cast<size_t>(pl.n_items) * 32, s)).empty()) return e;
    if (!(e = same((p + "ptr").c_str(), o.ptr, pl.ptr, static_cast<size_t>(pl.n_items) * 32 + 1, s)).empty()) return e;
    if (!(e = same((p + "idx").c_str(), o.idx, pl.idx, o.n_entries, s)).empty()) return e;
    if (!(e = same((p + "val").c_str(), o.val, pl.val, o.n_entries, s)).empty()) return e;
    if (!(e = same((p + "chunk").c_str(), o.chunk, pl.chunk, static_cast<size_t>(o.n_chunks) + 1, s)).empty()) return e;
    return {};
}

}  // namespace
}  // namespace apxb

extern "C" int apxb_test_prep_compare(apxb_engine* e, uint32_t n, const uint32_t* colptr, const uint32_t* rowidx,
                                      const float* vals, const uint32_t* perm, int sddm, const uint64_t* rounds,
                                      uint32_t n_rounds, double drop_rel, int k, const int32_t* a_colptr,
                                      const int32_t* a_rowidx, const double* a_vals) {
    return guarded([&]() -> int {
        if (!e || !colptr || !rowidx || !vals || !perm || !rounds || n_rounds == 0)
            return fail(APXB_ERR_INVALID, "bad argument (the device path needs round sizes)");
        if (k != 0 && k != 1 && k != 2 && k != 4 && k != 8 && k != 16 && k != 32 && k != 64 && k != 128)
            return fail(APXB_ERR_INVALID, "k must be 0 or 1..128");
        APXB_CK(cudaSetDevice(e->device));
        cudaStream_t s = e->stream;
        apxb::prepared_factor hf;
        const std::string hwhy = apxb::prepare_factor(n, colptr, rowidx, vals, perm, sddm != 0, rounds, n_rounds,
                                                      drop_rel, hf, false);
        apxb_factor f;
        f.e = e;
        int arc = 0;
        const std::string dwhy = apxb::prepare_factor_device(&f, n, colptr, rowidx, vals, perm, sddm != 0, rounds,
                                                             n_rounds, drop_rel, &arc);
        if (arc) return arc;
        if (hwhy != dwhy) return fail(APXB_ERR_INVALID, "preparation outcomes differ: host '" + hwhy + "', device '" + dwhy + "'");
        if (!hwhy.empty()) return APXB_OK;   // both rejected the factor the same way
        std::string why;
        const auto& h = f.h;
        if (h.m != hf.m || h.nnz_factor != hf.nnz_factor || h.nnz_stored != hf.nnz_stored || h.dropped != hf.dropped ||
            h.dropped_flush != hf.dropped_flush || h.fwd_levels != hf.fwd_levels || h.bck_levels != hf.bck_levels)
            return fail(APXB_ERR_INVALID, "sizes or counts differ");
        for (int dir = 0; dir < 2 && why.empty(); ++dir) {
            apxb::dev_plan_out o;
            o.n_items = (dir == 0 ? h.fwd_plan : h.bck_plan).n_items;
            o.info = f.info[dir]; o.ord = f.ord[dir]; o.ptr = f.ptr[dir]; o.idx = f.idx[dir]; o.val = f.val[dir];
            o.chunk = f.chunk[dir]; o.n_chunks = f.n_chunks[dir];
            o.n_entries = (dir == 0 ? hf.fwd_plan : hf.bck_plan).idx.size();
            why = apxb::same_plan(dir == 0 ? "forward plan" : "backward plan", o, dir == 0 ? hf.fwd_plan : hf.bck_plan, s);
        }
        if (why.empty()) why = apxb::factor_host_arrays(&f);
        if (why.empty()) {
            const auto eq = [](const auto& a, const auto& b) {
                return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), sizeof(a[0]) * a.size()) == 0);
            };
            if (!eq(h.csc_ptr, hf.csc_ptr) || !eq(h.csc_idx, hf.csc_idx) || !eq(h.csc_val, hf.csc_val)) why = "CSC(L11) differs";
            else if (!eq(h.csr_ptr, hf.csr_ptr) || !eq(h.csr_idx, hf.csr_idx) || !eq(h.csr_val, hf.csr_val)) why = "CSR(L11) differs";
            else if (!eq(h.fwd_level, hf.fwd_level) || !eq(h.bck_level, hf.bck_level)) why = "levels differ";
            else if (!eq(h.fwd_thin_bits, hf.fwd_thin_bits) || !eq(h.bck_thin_bits, hf.bck_thin_bits)) why = "thin flags differ";
        }
        if (why.empty() && k > 0) {
            const uint32_t col_lanes = k >= 8 ? static_cast<uint32_t>(k / 4) : 1u;
            std::vector<void*> tmp;
            auto alloc_bytes = [&](void** q, size_t bytes) -> std::string {
                const cudaError_t ce = cudaMalloc(q, bytes ? bytes : 16);
                if (ce != cudaSuccess) return cudaGetErrorString(ce);
                tmp.push_back(*q);
                return {};
            };
            for (int dir = 0; dir < 2 && why.empty(); ++dir) {
                apxb::sweep_plan hp;
                apxb::build_batch_plan(hf, dir, col_lanes, hp);
                apxb::dev_plan_out o;
                why = apxb::batch_plan_device(&f, dir, col_lanes, alloc_bytes, o, s);
                if (why.empty()) why = apxb::same_plan(dir == 0 ? "forward batch plan" : "backward batch plan", o, hp, s);
            }
            for (void* q : tmp) cudaFree(q);
        }
        if (why.empty() && a_colptr && a_rowidx && a_vals) {
            std::vector<int32_t> hptr, dptr;
            apxb::plan_vec<int32_t> hidx;
            apxb::plan_vec<double> hval;
            const std::string w1 = apxb::permute_operator(n, a_colptr, a_rowidx, a_vals, perm, hptr, hidx, hval);
            apxb_operator a;
            a.e = e;
            int orc = 0;
            const std::string w2 = apxb::permute_operator_device(&a, n, a_colptr, a_rowidx, a_vals, perm, dptr, &orc);
            if (orc) return orc;
            if (w1 != w2) why = "operator outcomes differ: host '" + w1 + "', device '" + w2 + "'";
            else if (w1.empty()) {
                if (hptr != dptr) why = "operator row offsets differ";
                else if (!(why = apxb::same("operator idx", a.idx, hidx, hidx.size(), s)).empty()) {
                } else why = apxb::same("operator val", a.val, hval, hval.size(), s);
            }
        }
        cudaStreamSynchronize(s);
        if (!why.empty()) return fail(APXB_ERR_INVALID, why);
        return APXB_OK;
    });
}
