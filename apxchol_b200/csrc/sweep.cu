// Sync-free persistent triangular sweeps over the approximate-Cholesky factor
// (the preconditioner's forward and backward solves; the reference's
// dataflow_kernel, src/cuda_dataflow.cu:321-478, and its CPU counterpart
// omp_sptrsv::solve_levelset, include/apxchol/solver/sptrsv/omp.h:1094-1119).
//
// Design (B200):
//  * A sweep is a dataflow launch plus, for factors whose elimination ends in
//    a long run of tiny rounds, a serial-segment launch (one block, shared
//    memory, __syncthreads per level; forward: after the dataflow, backward:
//    before it). The dataflow grid's warps work off the direction's plan
//    (host_prep.hpp, sweep_plan): work items of up to 32 rows
//    of one level and one lane-group width G, G lanes per row, with the rows'
//    entries re-laid in processing order. A warp claims items from an atomic
//    ticket in level order, so a row only waits on rows of earlier items; the
//    lowest unfinished item is always being run by its owner, so progress
//    never depends on scheduling.
//  * Latency pipeline: a warp runs item i while the entries and right-hand
//    sides of item i+1 and the row descriptors of item i+2 are in flight, and
//    the ticket for item i+3 is being claimed. A row's critical path is then
//    its dependency loads, the arithmetic and one store.
//  * No level barriers and no separate ready flags: the output vector starts
//    filled with a signalling-NaN marker and a solved value replaces it, so one
//    relaxed load both tests a dependency and fetches it. The kernel re-arms
//    the buffer the next sweep writes (reset), so no fill pass runs between
//    applications.
//  * Every wait has a time budget (globaltimer): a warp that makes no progress
//    for the budget records APXB_ERR_TIMEOUT in the engine's error word and
//    every warp drains; the host turns it into an error status.
//  * fp64 sweep: products and sums are individually rounded (__dmul_rn /
//    __dadd_rn, no contraction) in the reference's order -- rows of "thin"
//    levels use the 4-way split sum of dot_thin (omp.h:1343-1357), rows of
//    "fat" levels one serial sum (omp.h:1434-1439), finished by one correctly
//    rounded subtract and divide (omp.h:1440). With G lanes per row the
//    products are formed in parallel and the order is replayed through
//    shuffles: the result is the reference CPU sweep's bytes.
//  * fp32 sweep: fp32 values and fp32 fused multiply-add accumulation, each
//    lane adding its entries in order as they arrive, lane partials combined
//    by a fixed butterfly (deterministic); k right-hand sides per row
//    interleaved [row][k]: each factor entry is read once for all k.
//  * Rows are consumed progressively: in the fp64 sweep the reference's sum
//    order is advanced step by step as operands arrive, so most of a row's
//    arithmetic is done before its last dependency lands.
//  * fp16 factor storage (the reference's GPU default, cuda.h:131-163): the
//    fp32 sweep reads binary16 weights of the column-scaled factor, widened
//    exactly to fp32, a per-row fp32 diagonal, and (backward) its right-hand
//    side times the fp64 inv_scale^2 (cuda_dataflow.cu:395), 6 instead of 8
//    bytes per stored entry.
#include <cstdlib>
#include <cuda_fp16.h>

#include "kernels.cuh"

namespace apxb {

namespace {

constexpr int kBatch = 8;               // entries in flight per lane
constexpr uint32_t kNoRowDev = 0xffffffffu;

__device__ __forceinline__ unsigned backoff_ns(int spins) {
    return spins < 4 ? 0u : min(16u << min((spins - 4) >> 1, 3), 128u);
}

// Warp-uniform check of the error word and the time budget. Returns true when
// the warp must drain (budget exhausted -> error raised, or another warp failed).
__device__ __forceinline__ bool wait_must_stop(dev_error* err, unsigned long long t0, unsigned long long budget,
                                               int where, uint32_t row) {
    int stop = 0;
    if ((threadIdx.x & 31) == 0) {
        if (ld_relaxed_int(&err->code) != 0) {
            stop = 1;
        } else if (globaltimer() - t0 > budget) {
            raise_error(err, -4 /* APXB_ERR_TIMEOUT */, where, row);
            stop = 1;
        }
    }
    return __shfl_sync(kFull, stop, 0) != 0;
}

// Idle bookkeeping of a warp-uniform polling loop; returns true to drain.
struct idle_clock {
    int spins = 0;
    unsigned long long t0 = 0;
    __device__ __forceinline__ bool idle(dev_error* err, unsigned long long budget, int where, uint32_t row) {
        if (spins == 0 && (threadIdx.x & 31) == 0) t0 = globaltimer();
        ++spins;
        if ((spins & 15) == 0 && wait_must_stop(err, __shfl_sync(kFull, t0, 0), budget, where, row)) return true;
        const unsigned ns = backoff_ns(spins);
        if (ns) __nanosleep(ns);
        return false;
    }
};

__device__ __forceinline__ void leave(sweep_ctl* ctl) {
    if ((threadIdx.x & 31) == 0) {
        const unsigned total = gridDim.x * (blockDim.x >> 5);
        if (atomicAdd(&ctl->done, 1u) == total - 1) {
            ctl->ticket = 0;
            ctl->done = 0;
        }
    }
}

__device__ __forceinline__ double dadd4(double a, double b, double c, double d) {
    return __dadd_rn(__dadd_rn(a, b), __dadd_rn(c, d));
}

// ---------------------------------------------------------------------------
// Exact-order accumulation for a G-lane group (G = 2^LG = 4..32). Lane u of
// the group holds the product of entry t = t0 + u of the current step.
// thin: chain c (entries t = c mod 4, t < gend) accumulates in lane c in entry
// order; the step holding gend (when the row has a tail, gend < len) then
// combines the chains as (s0 + s1) + (s2 + s3) and adds the <= 3 tail entries
// in order. fat: lane 0 adds every entry in order. Steps are consumed in
// order, each as soon as all of its operands are ready, so most of a row's
// arithmetic is done before its last dependency arrives.
struct exact_state {
    double s = 0.0, sum = 0.0;
    bool combined = false;
};

template <unsigned LG>
__device__ __forceinline__ void exact_step(bool thin, bool consume, unsigned u, uint32_t t0, uint32_t len,
                                           uint32_t gend, double pk, exact_state& e) {
    constexpr unsigned G = 1u << LG;
    if (thin) {
        const unsigned c = u & 3u;
#pragma unroll
        for (unsigned i = 0; i < G / 4; ++i) {
            const double v = __shfl_sync(kFull, pk, static_cast<int>(c + 4u * i), static_cast<int>(G));
            if (consume && u < 4 && t0 + c + 4u * i < gend) e.s = __dadd_rn(e.s, v);
        }
        const bool tail = consume && !e.combined && gend < len && (gend >> LG) == (t0 >> LG);
        if (__any_sync(kFull, tail)) {
            const double s1 = __shfl_sync(kFull, e.s, 1, static_cast<int>(G));
            const double s2 = __shfl_sync(kFull, e.s, 2, static_cast<int>(G));
            const double s3 = __shfl_sync(kFull, e.s, 3, static_cast<int>(G));
            if (tail && u == 0) e.sum = dadd4(e.s, s1, s2, s3);
#pragma unroll
            for (unsigned i = 0; i < 3; ++i) {
                const double v = __shfl_sync(kFull, pk, static_cast<int>((gend + i) & (G - 1u)), static_cast<int>(G));
                if (tail && u == 0 && gend + i < len) e.sum = __dadd_rn(e.sum, v);
            }
            if (tail) e.combined = true;
        }
    } else {
#pragma unroll
        for (unsigned i = 0; i < G; ++i) {
            const double v = __shfl_sync(kFull, pk, static_cast<int>(i), static_cast<int>(G));
            if (consume && u == 0 && t0 + i < len) e.s = __dadd_rn(e.s, v);
        }
    }
}

// ---------------------------------------------------------------------------
// Pipeline stages shared by both precisions.

// Stage D: the item's descriptor words, loaded by every lane for its own slot.
struct stage_desc {
    unsigned c;          // item (>= n_items: none)
    uint32_t info, row, q, e;
};

template <class T>
__device__ __forceinline__ void load_desc(const sweep_args<T>& a, unsigned c, stage_desc& d) {
    const unsigned lane = threadIdx.x & 31u;
    d.c = c;
    d.info = 0; d.row = kNoRowDev; d.q = 0; d.e = 0;
    if (c < a.n_items) {
        const size_t pos = static_cast<size_t>(c) * 32 + lane;
        d.info = __ldg(a.info + c);
        d.row = __ldg(a.ord + pos);
        d.q = __ldg(a.ptr + pos);
        d.e = __ldg(a.ptr + pos + 1);
    }
}

// Lane view of an item after stage D: the lane's group, its row, and its range.
struct lane_view {
    unsigned c, lg, G, u, gid;
    bool valid, thin;
    uint32_t row, q, len;   // off-diagonals at [q, q + len); diagonal at q + len
};

__device__ __forceinline__ lane_view view_of(const stage_desc& d) {
    const unsigned lane = threadIdx.x & 31u;
    lane_view v;
    v.c = d.c;
    v.lg = (d.info >> 8) & 0xffu;
    v.G = 1u << v.lg;
    v.u = lane & (v.G - 1u);
    v.gid = lane >> v.lg;
    v.thin = (d.info >> 16) & 1u;
    // slot gid's descriptor lives in lane gid
    v.row = __shfl_sync(kFull, d.row, static_cast<int>(v.gid));
    v.q = __shfl_sync(kFull, d.q, static_cast<int>(v.gid));
    const uint32_t e = __shfl_sync(kFull, d.e, static_cast<int>(v.gid));
    v.valid = v.row != kNoRowDev;
    v.len = v.valid ? e - v.q - 1u : 0u;
    return v;
}

// Warp-uniform chunked claim: the items of the current chunk, then those of
// the pending chunk, whose ticket was taken when the current one began and
// whose bounds are loaded when the current chunk hands out its last item.
// A contended same-address atomic takes about (claimers x 0.7 ns), so the
// ticket is only read a chunk later.
struct chunk_claim {
    template <class T>
    __device__ __forceinline__ void start(const sweep_args<T>& a) {
        unsigned t = 0;
        if ((threadIdx.x & 31u) == 0) t = atomicAdd(&a.ctl->ticket, 1u);
        pend = __shfl_sync(kFull, t, 0);
    }
    unsigned cur = 0, end = 0;
    unsigned pend = 0;            // ticket of the next chunk
    unsigned plo = 0, phi = 0;    // its bounds (valid when loaded)
    bool loaded = false;
    template <class T>
    __device__ __forceinline__ void load_pending(const sweep_args<T>& a) {
        if (!loaded && pend < a.n_chunks) {
            plo = __ldg(a.chunk + pend);
            phi = __ldg(a.chunk + pend + 1);
            loaded = true;
        }
    }
    template <class T>
    __device__ __forceinline__ unsigned next(const sweep_args<T>& a) {
        if (cur >= end) {
            if (pend >= a.n_chunks) return a.n_items;
            load_pending(a);
            cur = plo;
            end = phi;
            loaded = false;
            unsigned t = 0;
            if ((threadIdx.x & 31u) == 0) t = atomicAdd(&a.ctl->ticket, 1u);
            pend = __shfl_sync(kFull, t, 0);
            return cur++;
        }
        const unsigned c = cur++;
        if (cur >= end) load_pending(a);
        return c;
    }
};

// ---------------------------------------------------------------------------
// fp64 dataflow sweep.

// Stage L data of one item (fp64).
struct stage_data64 {
    lane_view v;
    double rhs, d;
    uint32_t jj[kBatch];
    float ww[kBatch];
};

__device__ __forceinline__ void load_data64(const sweep_args<double>& a, const stage_desc& ds, stage_data64& s) {
    s.v = view_of(ds);
    const lane_view& v = s.v;
    s.rhs = 0.0; s.d = 1.0;
    if (v.c >= a.n_items) return;
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
        const uint32_t t = (static_cast<uint32_t>(k) << v.lg) + v.u;
        if (t < v.len) { s.jj[k] = __ldg(a.idx + v.q + t); s.ww[k] = __ldg(a.val + v.q + t); }
    }
    if (v.valid && v.u == 0) {
        s.rhs = a.in[v.row];
        s.d = static_cast<double>(__ldg(a.val + v.q + v.len));
    }
}

// Group rows (G = 2^LG lanes per row): batches of kBatch steps; inside a
// batch the steps are consumed in order as their operands arrive.
template <unsigned LG>
__device__ __forceinline__ bool run_group64(const sweep_args<double>& a, stage_data64& s, int where,
                                            double& total) {
    constexpr unsigned G = 1u << LG;
    const lane_view& v = s.v;
    const unsigned gmask = G == 32 ? kFull : (((1u << G) - 1u) << (v.gid * G));
    const uint32_t J = (v.len + G - 1u) >> LG;
    const uint32_t Jmax = __reduce_max_sync(kFull, J);
    const uint32_t gend = v.thin ? (v.len & ~3u) : 0u;
    exact_state e;
    idle_clock clk;
    for (uint32_t jb = 0; jb < Jmax; jb += kBatch) {
        if (jb > 0) {
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                const uint32_t t = ((jb + k) << LG) + v.u;
                if (t < v.len) { s.jj[k] = __ldg(a.idx + v.q + t); s.ww[k] = __ldg(a.val + v.q + t); }
            }
        }
        const uint32_t nsteps = J > jb ? min(static_cast<uint32_t>(kBatch), J - jb) : 0u;
        double p[kBatch];
        unsigned rdy = 0;   // bit k: entry of step k absent or its product is in p[k]
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t t = ((jb + k) << LG) + v.u;
            p[k] = 0.0;
            if (t < v.len) p[k] = ld_relaxed(a.out + s.jj[k]);
        }
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const uint32_t t = ((jb + k) << LG) + v.u;
            if (t >= v.len) rdy |= 1u << k;
            else if (!is_sent(p[k])) { p[k] = __dmul_rn(static_cast<double>(s.ww[k]), p[k]); rdy |= 1u << k; }
        }
        uint32_t kpos = 0;
        for (;;) {
            bool progressed = false;
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                const unsigned bal = __ballot_sync(kFull, (rdy >> k) & 1u);
                const bool consume = kpos == static_cast<uint32_t>(k) && static_cast<uint32_t>(k) < nsteps &&
                                     (bal & gmask) == gmask;
                if (__any_sync(kFull, consume)) {
                    exact_step<LG>(v.thin, consume, v.u, (jb + k) << LG, v.len, gend, p[k], e);
                    progressed = true;
                }
                if (consume) ++kpos;
            }
            if (__all_sync(kFull, kpos >= nsteps)) break;
            if (progressed) clk.spins = 0;
            else if (clk.idle(a.err, a.budget_ns, where, v.row)) return false;
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                if (!((rdy >> k) & 1u)) {
                    const double y = ld_relaxed(a.out + s.jj[k]);
                    if (!is_sent(y)) { p[k] = __dmul_rn(static_cast<double>(s.ww[k]), y); rdy |= 1u << k; }
                }
            }
        }
    }
    const double s1 = __shfl_sync(kFull, e.s, 1, static_cast<int>(G));
    const double s2 = __shfl_sync(kFull, e.s, 2, static_cast<int>(G));
    const double s3 = __shfl_sync(kFull, e.s, 3, static_cast<int>(G));
    total = !v.thin ? e.s : (e.combined ? e.sum : dadd4(e.s, s1, s2, s3));
    return true;
}

// One lane per row (<= kBatch off-diagonals): each lane consumes its entries
// in order as they arrive, 4-way rotating chains then the serial tail.
__device__ __forceinline__ bool run_lane64(const sweep_args<double>& a, stage_data64& s, int where, double& total) {
    const lane_view& v = s.v;
    const uint32_t n = v.len;   // <= kBatch for these rows
    const uint32_t gend = v.thin ? (n & ~3u) : 0u;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, sum = 0.0;
    bool combined = false;
    double yv[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; ++k)
        if (static_cast<uint32_t>(k) < n) yv[k] = ld_relaxed(a.out + s.jj[k]);
    uint32_t kpos = 0;
    idle_clock clk;
    for (;;) {
        const uint32_t before = kpos;
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            if (kpos == static_cast<uint32_t>(k) && kpos < n && !is_sent(yv[k])) {
                const double pr = __dmul_rn(static_cast<double>(s.ww[k]), yv[k]);
                if (kpos < gend) {
                    const double w = __dadd_rn(s0, pr);
                    s0 = s1; s1 = s2; s2 = s3; s3 = w;
                } else {
                    if (!combined) { sum = dadd4(s0, s1, s2, s3); combined = true; }
                    sum = __dadd_rn(sum, pr);
                }
                ++kpos;
            }
        }
        if (__all_sync(kFull, kpos >= n)) break;
        if (__any_sync(kFull, kpos != before)) clk.spins = 0;
        else if (clk.idle(a.err, a.budget_ns, where, v.row)) return false;
#pragma unroll
        for (int k = 0; k < kBatch; ++k)
            if (static_cast<uint32_t>(k) >= kpos && static_cast<uint32_t>(k) < n && is_sent(yv[k]))
                yv[k] = ld_relaxed(a.out + s.jj[k]);
    }
    total = combined ? sum : dadd4(s0, s1, s2, s3);
    return true;
}

// Run one item: wait for its operands, replay the reference's sum order, store.
// Returns false when the warp must drain.
template <int DIR>
__device__ __forceinline__ bool run64(const sweep_args<double>& a, stage_data64& s) {
    const lane_view& v = s.v;
    const int where = DIR == 0 ? kFwdSweep : kBckSweep;
    double total = 0.0;
    bool ok;
    switch (v.lg) {
        case 0: ok = run_lane64(a, s, where, total); break;
        case 2: ok = run_group64<2>(a, s, where, total); break;
        case 3: ok = run_group64<3>(a, s, where, total); break;
        case 4: ok = run_group64<4>(a, s, where, total); break;
        default: ok = run_group64<5>(a, s, where, total); break;
    }
    if (!ok) return false;
    if (v.valid && v.u == 0) {
        double rhs = s.rhs;
        if (a.rhs_sub) rhs = __dsub_rn(rhs, *a.rhs_sub);
        const double y = __ddiv_rn(__dsub_rn(rhs, total), s.d);
        st_relaxed(a.out + v.row, y);
        if (a.copy_out) a.copy_out[v.row] = y;
        // re-arm after the right-hand side was consumed: the backward sweep
        // reads it from the buffer it re-arms (a store issued right behind the
        // load of the same address would wait for that load)
        if (a.reset) a.reset[v.row] = sent_of(0.0);
    }
    return true;
}

template <int DIR>
__global__ void __launch_bounds__(kSweepThreads, 2) k_df64(const sweep_args<double> a) {
    if (a.skip && *a.skip) return;
    const unsigned lane = threadIdx.x & 31u;
    chunk_claim cc;
    cc.start(a);
    stage_desc dD;
    load_desc(a, cc.next(a), dD);
    stage_data64 sL;
    load_data64(a, dD, sL);
    load_desc(a, cc.next(a), dD);
    int bad = 0;   // the error word, read one item late so the load is never waited on
    while (sL.v.c < a.n_items) {
        // rotate: run L, data for D, descriptor of the next claimed item
        stage_data64 sR = sL;
        load_data64(a, dD, sL);
        load_desc(a, cc.next(a), dD);
        if (__shfl_sync(kFull, bad, 0)) break;
        if (lane == 0) bad = ld_relaxed_int(&a.err->code);
        if (!run64<DIR>(a, sR)) break;
    }
    leave(a.ctl);
}

// ---------------------------------------------------------------------------
// fp32, K right-hand sides per row.

template <int K>
__device__ __forceinline__ void ld_row(const float* p, float (&y)[K]) {
    if constexpr (K == 1) {
        y[0] = ld_relaxed(p);
    } else if constexpr (K == 2) {
        unsigned a0, a1;
        asm volatile("ld.relaxed.gpu.global.v2.b32 {%0,%1}, [%2];" : "=r"(a0), "=r"(a1) : "l"(p) : "memory");
        y[0] = __uint_as_float(a0); y[1] = __uint_as_float(a1);
    } else {
#pragma unroll
        for (int h = 0; h < K; h += 4) {
            unsigned a0, a1, a2, a3;
            asm volatile("ld.relaxed.gpu.global.v4.b32 {%0,%1,%2,%3}, [%4];"
                         : "=r"(a0), "=r"(a1), "=r"(a2), "=r"(a3) : "l"(p + h) : "memory");
            y[h] = __uint_as_float(a0); y[h + 1] = __uint_as_float(a1);
            y[h + 2] = __uint_as_float(a2); y[h + 3] = __uint_as_float(a3);
        }
    }
}

template <int K>
__device__ __forceinline__ void st_row(float* p, const float (&y)[K]) {
    if constexpr (K == 1) {
        st_relaxed(p, y[0]);
    } else if constexpr (K == 2) {
        asm volatile("st.relaxed.gpu.global.v2.b32 [%0], {%1,%2};"
                     :: "l"(p), "r"(__float_as_uint(y[0])), "r"(__float_as_uint(y[1])) : "memory");
    } else {
#pragma unroll
        for (int h = 0; h < K; h += 4)
            asm volatile("st.relaxed.gpu.global.v4.b32 [%0], {%1,%2,%3,%4};"
                         :: "l"(p + h), "r"(__float_as_uint(y[h])), "r"(__float_as_uint(y[h + 1])),
                            "r"(__float_as_uint(y[h + 2])), "r"(__float_as_uint(y[h + 3])) : "memory");
    }
}

template <int K>
__device__ __forceinline__ bool row_ready(const float (&y)[K]) {
    bool ok = true;
#pragma unroll
    for (int s = 0; s < K; ++s) ok &= !is_sent(y[s]);
    return ok;
}

template <int K>
struct batch_of { static constexpr int value = K >= 16 ? 2 : (K >= 8 ? 4 : 8); };

template <int K>
struct stage_data32 {
    lane_view v;
    float rhs[K];
    float d;
    uint32_t jj[batch_of<K>::value];
    float ww[batch_of<K>::value];
};

// Weight of plan entry e: fp32, or the binary16 value widened (exact).
template <bool H>
__device__ __forceinline__ float weight32(const sweep_args<float>& a, uint32_t e) {
    if constexpr (H) return __half2float(__ushort_as_half(__ldg(a.val16 + e)));
    else return __ldg(a.val + e);
}

template <int K, bool H>
__device__ __forceinline__ void load_data32(const sweep_args<float>& a, const double* in64, const stage_desc& ds,
                                            stage_data32<K>& s) {
    constexpr int B = batch_of<K>::value;
    s.v = view_of(ds);
    const lane_view& v = s.v;
    s.d = 1.0f;
#pragma unroll
    for (int r = 0; r < K; ++r) s.rhs[r] = 0.0f;
    if (v.c >= a.n_items) return;
#pragma unroll
    for (int k = 0; k < B; ++k) {
        const uint32_t t = (static_cast<uint32_t>(k) << v.lg) + v.u;
        if (t < v.len) { s.jj[k] = __ldg(a.idx + v.q + t); s.ww[k] = weight32<H>(a, v.q + t); }
    }
    if (v.valid && v.u == 0) {
        const size_t base = static_cast<size_t>(v.row) * K;
        if (in64) {
#pragma unroll
            for (int r = 0; r < K; ++r) {
                double x = in64[base + r];
                if (a.rhs_sub) x -= a.rhs_sub[r];
                s.rhs[r] = static_cast<float>(x);
            }
        } else if (H && a.in_scale2) {
            const double sc = a.in_scale2[v.row];
#pragma unroll
            for (int r = 0; r < K; ++r) s.rhs[r] = static_cast<float>(static_cast<double>(a.in[base + r]) * sc);
        } else {
#pragma unroll
            for (int r = 0; r < K; ++r) s.rhs[r] = a.in[base + r];
        }
        s.d = H ? __ldg(a.diag16 + v.row) : __ldg(a.val + v.q + v.len);
    }
}

template <int DIR, int K, bool H>
__device__ __forceinline__ bool run32(const sweep_args<float>& a, stage_data32<K>& s) {
    constexpr int B = batch_of<K>::value;
    const lane_view& v = s.v;
    const int where = DIR == 0 ? kFwdSweep32 : kBckSweep32;
    const uint32_t J = (v.len + v.G - 1u) >> v.lg;
    const uint32_t Jmax = __reduce_max_sync(kFull, J);
    float acc[K];
#pragma unroll
    for (int r = 0; r < K; ++r) acc[r] = 0.0f;
    idle_clock clk;
    for (uint32_t jb = 0; jb < Jmax; jb += B) {
        if (jb > 0) {
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const uint32_t t = ((jb + k) << v.lg) + v.u;
                if (t < v.len) { s.jj[k] = __ldg(a.idx + v.q + t); s.ww[k] = weight32<H>(a, v.q + t); }
            }
        }
        // this lane's entries in the batch: steps 0 .. nk-1
        const uint32_t t0 = (jb << v.lg) + v.u;
        const uint32_t nk = t0 < v.len ? min(static_cast<uint32_t>(B), ((v.len - t0 - 1u) >> v.lg) + 1u) : 0u;
        float yv[B][K];
#pragma unroll
        for (int k = 0; k < B; ++k)
            if (static_cast<uint32_t>(k) < nk) ld_row<K>(a.out + static_cast<size_t>(s.jj[k]) * K, yv[k]);
        // each lane consumes its own entries in order as they arrive
        uint32_t kpos = 0;
        for (;;) {
            const uint32_t before = kpos;
#pragma unroll
            for (int k = 0; k < B; ++k) {
                if (kpos == static_cast<uint32_t>(k) && kpos < nk && row_ready<K>(yv[k])) {
#pragma unroll
                    for (int r = 0; r < K; ++r) acc[r] = __fmaf_rn(s.ww[k], yv[k][r], acc[r]);
                    ++kpos;
                }
            }
            if (__all_sync(kFull, kpos >= nk)) break;
            if (__any_sync(kFull, kpos != before)) clk.spins = 0;
            else if (clk.idle(a.err, a.budget_ns, where, v.row)) return false;
#pragma unroll
            for (int k = 0; k < B; ++k)
                if (static_cast<uint32_t>(k) >= kpos && static_cast<uint32_t>(k) < nk && !row_ready<K>(yv[k]))
                    ld_row<K>(a.out + static_cast<size_t>(s.jj[k]) * K, yv[k]);
        }
    }
    // fixed butterfly over the group's lanes
    for (unsigned o = v.G >> 1; o > 0; o >>= 1)
#pragma unroll
        for (int r = 0; r < K; ++r) acc[r] += __shfl_xor_sync(kFull, acc[r], static_cast<int>(o), static_cast<int>(v.G));
    if (v.valid && v.u == 0) {
        float y[K];
#pragma unroll
        for (int r = 0; r < K; ++r) y[r] = __fdiv_rn(s.rhs[r] - acc[r], s.d);
        st_row<K>(a.out + static_cast<size_t>(v.row) * K, y);
        if (a.copy_out) {
#pragma unroll
            for (int r = 0; r < K; ++r) a.copy_out[static_cast<size_t>(v.row) * K + r] = y[r];
        }
        if (a.reset) {   // re-arm after the right-hand side was consumed (see run64)
            float sent[K];
#pragma unroll
            for (int r = 0; r < K; ++r) sent[r] = sent_of(0.0f);
            st_row<K>(a.reset + static_cast<size_t>(v.row) * K, sent);
        }
    }
    return true;
}

template <int DIR, int K, bool H>
__global__ void __launch_bounds__(kSweepThreads, 2) k_df32(const sweep_args<float> a, const double* in64) {
    if (a.skip && *a.skip) return;
    const unsigned lane = threadIdx.x & 31u;
    chunk_claim cc;
    cc.start(a);
    stage_desc dD;
    load_desc(a, cc.next(a), dD);
    stage_data32<K> sL;
    load_data32<K, H>(a, in64, dD, sL);
    load_desc(a, cc.next(a), dD);
    int bad = 0;   // the error word, read one item late
    while (sL.v.c < a.n_items) {
        stage_data32<K> sR = sL;
        load_data32<K, H>(a, in64, dD, sL);
        load_desc(a, cc.next(a), dD);
        if (__shfl_sync(kFull, bad, 0)) break;
        if (lane == 0) bad = ld_relaxed_int(&a.err->code);
        if (!run32<DIR, K, H>(a, sR)) break;
    }
    leave(a.ctl);
}


// ---------------------------------------------------------------------------
// Batched fp32 sweep over a batch plan (host_prep.hpp, build_batch_plan).
// A row's G lanes are C column lanes x ge entry lanes: lane u of the group
// handles columns [KC * (u % C), KC * (u % C) + KC) and entries t = u / C,
// u / C + ge, ... of the row (oldest dependency first), 8 at a time, so each
// gather is one 16-byte load (k >= 4) and a lane keeps 8 of them in flight.
// Partial sums are combined by a fixed butterfly over the entry lanes. Work is
// claimed in chunks (consecutive items of one level) from the ticket counter;
// the next chunk is claimed when the current one starts, so the atomic's
// latency is hidden behind a chunk of work.

template <int K>
struct wide_cfg {
    static constexpr int KC = K < 4 ? K : 4;   // columns per lane
    static constexpr int C = K / KC;           // column lanes per row
    static constexpr int LC = C == 32 ? 5 : (C == 16 ? 4 : (C == 8 ? 3 : (C == 4 ? 2 : (C == 2 ? 1 : 0))));
    static constexpr int B = 8;                // entries in flight per lane
};

template <int K>
struct stage_wide {
    lane_view v;
    unsigned cl, ue, glg;        // column lane, entry lane, log2(entry lanes)
    float rhs[wide_cfg<K>::KC];
    float d;
    uint32_t jj[wide_cfg<K>::B];
    float ww[wide_cfg<K>::B];
};

template <int K, bool H>
__device__ __forceinline__ void load_wide(const sweep_args<float>& a, const stage_desc& ds, stage_wide<K>& s) {
    using W = wide_cfg<K>;
    s.v = view_of(ds);
    const lane_view& v = s.v;
    s.cl = v.u & static_cast<unsigned>(W::C - 1);
    s.ue = v.u >> W::LC;
    s.glg = v.lg - W::LC;
    s.d = 1.0f;
#pragma unroll
    for (int r = 0; r < W::KC; ++r) s.rhs[r] = 0.0f;
    if (v.c >= a.n_items) return;
#pragma unroll
    for (int k = 0; k < W::B; ++k) {
        const uint32_t t = (static_cast<uint32_t>(k) << s.glg) + s.ue;
        if (t < v.len) { s.jj[k] = __ldg(a.idx + v.q + t); s.ww[k] = weight32<H>(a, v.q + t); }
    }
    if (v.valid && s.ue == 0) {
        const size_t base = static_cast<size_t>(v.row) * K + s.cl * W::KC;
        if (H && a.in_scale2) {   // fp16 storage, backward: the input times inv_scale^2, in fp64, rounded once
            const double sc = a.in_scale2[v.row];
#pragma unroll
            for (int r = 0; r < W::KC; ++r) s.rhs[r] = static_cast<float>(static_cast<double>(a.in[base + r]) * sc);
        } else {
#pragma unroll
            for (int r = 0; r < W::KC; ++r) s.rhs[r] = a.in[base + r];
        }
        s.d = H ? __ldg(a.diag16 + v.row) : __ldg(a.val + v.q + v.len);
    }
}

// L2 prefetch of the dependency rows the lane will gather for its next item
// (whose indices arrived while the current item ran). A prefetch holds no
// register and L2 is the point of coherence, so the later relaxed load still
// sees whatever the row holds then, solved or not.
template <int K>
__device__ __forceinline__ void prefetch_wide(const sweep_args<float>& a, const stage_wide<K>& s) {
    using W = wide_cfg<K>;
    const lane_view& v = s.v;
    if (v.c >= a.n_items) return;
    const size_t col = static_cast<size_t>(s.cl) * W::KC;
#pragma unroll
    for (int k = 0; k < W::B; ++k) {
        const uint32_t t = (static_cast<uint32_t>(k) << s.glg) + s.ue;
        if (t < v.len) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.out + static_cast<size_t>(s.jj[k]) * K + col));
    }
}

template <int DIR, int K, bool H>
__device__ __forceinline__ bool run_wide(const sweep_args<float>& a, stage_wide<K>& s, const stage_wide<K>& next) {
    using W = wide_cfg<K>;
    constexpr int B = W::B, KC = W::KC;
    const lane_view& v = s.v;
    const int where = DIR == 0 ? kFwdSweep32 : kBckSweep32;
    const uint32_t ge = 1u << s.glg;
    const uint32_t J = (v.len + ge - 1u) >> s.glg;
    const uint32_t Jmax = __reduce_max_sync(kFull, J);
    const size_t col = static_cast<size_t>(s.cl) * KC;
    float acc[KC];
#pragma unroll
    for (int r = 0; r < KC; ++r) acc[r] = 0.0f;
    idle_clock clk;
    for (uint32_t jb = 0; jb < Jmax; jb += B) {
        if (jb > 0) {
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const uint32_t t = ((jb + k) << s.glg) + s.ue;
                if (t < v.len) { s.jj[k] = __ldg(a.idx + v.q + t); s.ww[k] = weight32<H>(a, v.q + t); }
            }
        }
        const uint32_t t0 = (jb << s.glg) + s.ue;
        const uint32_t nk = t0 < v.len ? min(static_cast<uint32_t>(B), ((v.len - t0 - 1u) >> s.glg) + 1u) : 0u;
        float yv[B][KC];
#pragma unroll
        for (int k = 0; k < B; ++k)
            if (static_cast<uint32_t>(k) < nk) ld_row<KC>(a.out + static_cast<size_t>(s.jj[k]) * K + col, yv[k]);
        if (jb == 0) prefetch_wide<K>(a, next);   // the next item's gathers start while these are in flight
        uint32_t kpos = 0;
        for (;;) {
            const uint32_t before = kpos;
#pragma unroll
            for (int k = 0; k < B; ++k) {
                if (kpos == static_cast<uint32_t>(k) && kpos < nk && row_ready<KC>(yv[k])) {
#pragma unroll
                    for (int r = 0; r < KC; ++r) acc[r] = __fmaf_rn(s.ww[k], yv[k][r], acc[r]);
                    ++kpos;
                }
            }
            if (__all_sync(kFull, kpos >= nk)) break;
            if (__any_sync(kFull, kpos != before)) clk.spins = 0;
            else if (clk.idle(a.err, a.budget_ns, where, v.row)) return false;
            // re-poll only the entry this lane is blocked on and the ones after it
#pragma unroll
            for (int k = 0; k < B; ++k)
                if (static_cast<uint32_t>(k) >= kpos && static_cast<uint32_t>(k) < nk && !row_ready<KC>(yv[k]))
                    ld_row<KC>(a.out + static_cast<size_t>(s.jj[k]) * K + col, yv[k]);
        }
    }
    // fixed butterfly over the entry lanes (same column lane)
    for (unsigned o = v.G >> 1; o >= static_cast<unsigned>(W::C); o >>= 1)
#pragma unroll
        for (int r = 0; r < KC; ++r) acc[r] += __shfl_xor_sync(kFull, acc[r], static_cast<int>(o), static_cast<int>(v.G));
    if (v.valid && s.ue == 0) {
        float y[KC];
#pragma unroll
        for (int r = 0; r < KC; ++r) y[r] = __fdiv_rn(s.rhs[r] - acc[r], s.d);
        st_row<KC>(a.out + static_cast<size_t>(v.row) * K + col, y);
        // re-arm the row in the buffer the other direction writes next; done
        // here, after the row's right-hand side has been consumed, since the
        // backward sweep reads its right-hand side from that same buffer
        if (a.reset) {
            float sent[KC];
#pragma unroll
            for (int r = 0; r < KC; ++r) sent[r] = sent_of(0.0f);
            st_row<KC>(a.reset + static_cast<size_t>(v.row) * K + col, sent);
        }
    }
    return true;
}

template <int DIR, int K, bool H>
__global__ void __launch_bounds__(kSweepThreads, 2) k_dw32(const sweep_args<float> a) {
    if (a.skip && *a.skip) return;
    const unsigned lane = threadIdx.x & 31u;
    chunk_claim cc;
    cc.start(a);
    stage_desc dD;
    load_desc(a, cc.next(a), dD);
    stage_wide<K> sL;
    load_wide<K, H>(a, dD, sL);
    load_desc(a, cc.next(a), dD);
    int bad = 0;   // the error word, read one item late so the load is never waited on
    while (sL.v.c < a.n_items) {
        stage_wide<K> sR = sL;
        load_wide<K, H>(a, dD, sL);
        load_desc(a, cc.next(a), dD);
        if (__shfl_sync(kFull, bad, 0)) break;
        if (lane == 0) bad = ld_relaxed_int(&a.err->code);
        if (!run_wide<DIR, K, H>(a, sR, sL)) break;
    }
    leave(a.ctl);
}

// ---------------------------------------------------------------------------
// Serial segment: one block solves the run of small trailing levels (forward:
// after the dataflow launch; backward: before it) level by level, values in
// shared memory, __syncthreads between levels. Each warp solves its rows (the
// segment rows round-robin over the warps, in processing order) with all 32
// lanes, and prefetches its next row while working on the current one.

constexpr int kSegThreads = 512;
constexpr uint64_t kBox = 0xFFF6000000000000ull;   // NaN box carrying a segment-local index

__device__ __forceinline__ double box_index(uint32_t i) { return __longlong_as_double(static_cast<long long>(kBox | i)); }
__device__ __forceinline__ bool is_box(double v) {
    return (static_cast<unsigned long long>(__double_as_longlong(v)) & 0xFFFF000000000000ull) == kBox;
}
__device__ __forceinline__ uint32_t unbox(double v) {
    return static_cast<uint32_t>(static_cast<unsigned long long>(__double_as_longlong(v)) & 0xffffffffull);
}

struct seg_slot {
    uint32_t i, r, q, len;
    double rhs, d;
    double pv[kBatch];   // product (operand outside the segment, final) or the boxed segment index
    float ww[kBatch];
};

__device__ __forceinline__ void seg_batch64(const sweep_args<double>& a, const seg_slot& s, uint32_t jb,
                                            double (&pv)[kBatch], float (&ww)[kBatch]) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t s0 = a.seg_first, s1 = a.seg_first + a.seg_rows;
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
        const uint32_t t = ((jb + k) << 5) + lane;
        pv[k] = 0.0;
        ww[k] = 0.0f;
        if (t < s.len) {
            const uint32_t j = __ldg(a.seg_idx + s.q + t);
            const float w = __ldg(a.seg_val + s.q + t);
            ww[k] = w;
            pv[k] = (j >= s0 && j < s1) ? box_index(j - s0) : __dmul_rn(static_cast<double>(w), a.out[j]);
        }
    }
}

__device__ __forceinline__ void seg_fetch64(const sweep_args<double>& a, uint32_t i, seg_slot& s) {
    s.i = i;
    s.len = 0;
    if (i >= a.seg_rows) return;
    s.r = __ldg(a.seg_row + i);
    s.q = __ldg(a.seg_ptr + i);
    s.len = __ldg(a.seg_ptr + i + 1) - s.q - 1u;
    seg_batch64(a, s, 0, s.pv, s.ww);
    if ((threadIdx.x & 31u) == 0) {
        s.rhs = a.in[s.r];
        s.d = static_cast<double>(__ldg(a.seg_val + s.q + s.len));
    }
}

__device__ __forceinline__ void seg_solve64(const sweep_args<double>& a, seg_slot& s, bool thin, double* segv) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t J = (s.len + 31u) >> 5;
    const uint32_t gend = thin ? (s.len & ~3u) : 0u;
    exact_state e;
    for (uint32_t jb = 0; jb < J; jb += kBatch) {
        if (jb > 0) seg_batch64(a, s, jb, s.pv, s.ww);
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            double p = s.pv[k];
            if (is_box(p)) p = __dmul_rn(static_cast<double>(s.ww[k]), segv[unbox(p)]);
            exact_step<5>(thin, jb + k < J, lane, (jb + k) << 5, s.len, gend, p, e);
        }
    }
    const double s1 = __shfl_sync(kFull, e.s, 1), s2 = __shfl_sync(kFull, e.s, 2), s3 = __shfl_sync(kFull, e.s, 3);
    const double total = !thin ? e.s : (e.combined ? e.sum : dadd4(e.s, s1, s2, s3));
    if (lane == 0) {
        double rhs = s.rhs;
        if (a.rhs_sub) rhs = __dsub_rn(rhs, *a.rhs_sub);
        const double y = __ddiv_rn(__dsub_rn(rhs, total), s.d);
        segv[s.r - a.seg_first] = y;
        a.out[s.r] = y;
        if (a.copy_out) a.copy_out[s.r] = y;
        if (a.reset) a.reset[s.r] = sent_of(0.0);
    }
}

__global__ void __launch_bounds__(kSegThreads, 1) k_seg64(const sweep_args<double> a) {
    if (a.skip && *a.skip) return;
    if (a.err->code != 0) return;
    extern __shared__ double segv[];
    const unsigned warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    seg_slot cur, nxt;
    seg_fetch64(a, warp, cur);
    for (uint32_t l = 0; l < a.seg_levels; ++l) {
        const uint32_t w0 = __ldg(a.seg_lvl + l), hi = __ldg(a.seg_lvl + l + 1) & 0x7fffffffu;
        const bool thin = (w0 >> 31) != 0;
        while (cur.i < hi) {
            seg_fetch64(a, cur.i + nw, nxt);
            seg_solve64(a, cur, thin, segv);
            cur = nxt;
        }
        __syncthreads();
    }
}

// fp32, K right-hand sides: lanes stride the row's entries, operands from
// shared memory (inside the segment) or the output vector (final), fixed
// butterfly.
template <int K>
__global__ void __launch_bounds__(kSegThreads, 1) k_seg32(const sweep_args<float> a, const double* in64) {
    if (a.skip && *a.skip) return;
    if (a.err->code != 0) return;
    extern __shared__ float segf[];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t s0 = a.seg_first, s1 = a.seg_first + a.seg_rows;
    uint32_t i = warp;
    for (uint32_t l = 0; l < a.seg_levels; ++l) {
        const uint32_t hi = __ldg(a.seg_lvl + l + 1) & 0x7fffffffu;
        for (; i < hi; i += nw) {
            const uint32_t r = __ldg(a.seg_row + i), q = __ldg(a.seg_ptr + i);
            const uint32_t len = __ldg(a.seg_ptr + i + 1) - q - 1u;
            float acc[K];
#pragma unroll
            for (int c = 0; c < K; ++c) acc[c] = 0.0f;
            for (uint32_t t = lane; t < len; t += 32u) {
                const uint32_t j = __ldg(a.seg_idx + q + t);
                const float w = __ldg(a.seg_val + q + t);
                const float* src = (j >= s0 && j < s1) ? segf + static_cast<size_t>(j - s0) * K
                                                       : a.out + static_cast<size_t>(j) * K;
#pragma unroll
                for (int c = 0; c < K; ++c) acc[c] = __fmaf_rn(w, src[c], acc[c]);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int c = 0; c < K; ++c) acc[c] += __shfl_xor_sync(kFull, acc[c], o);
            if (lane == 0) {
                const size_t base = static_cast<size_t>(r) * K;
                const float d = __ldg(a.seg_val + q + len);
#pragma unroll
                for (int c = 0; c < K; ++c) {
                    float rhs;
                    if (in64) {
                        double x = in64[base + c];
                        if (a.rhs_sub) x -= a.rhs_sub[c];
                        rhs = static_cast<float>(x);
                    } else {
                        rhs = a.in[base + c];
                    }
                    const float y = __fdiv_rn(rhs - acc[c], d);
                    segf[static_cast<size_t>(r - s0) * K + c] = y;
                    a.out[base + c] = y;
                    if (a.copy_out) a.copy_out[base + c] = y;
                    if (a.reset) a.reset[base + c] = sent_of(0.0f);
                }
            }
        }
        __syncthreads();
    }
}

__global__ void k_fill64(double* p, size_t n, double v) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        p[i] = v;
}
__global__ void k_fill32(float* p, size_t n, float v) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        p[i] = v;
}

int fill_grid(size_t n) {
    const size_t b = (n + 255) / 256;
    return static_cast<int>(b < 4096 ? (b ? b : 1) : 4096);
}

template <int K>
int occ32() {
    int b0 = 0, b1 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_df32<0, K, false>, kSweepThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_df32<1, K, false>, kSweepThreads, 0);
    return b0 < b1 ? b0 : b1;
}

template <class F>
void set_smem(F* kernel, size_t bytes) {
    if (bytes > 48 * 1024)
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

template <int K>
void seg32(const sweep_args<float>& a, const double* in64, cudaStream_t s) {
    const size_t smem = static_cast<size_t>(a.seg_rows) * K * sizeof(float);
    set_smem(k_seg32<K>, smem);
    k_seg32<K><<<1, kSegThreads, smem, s>>>(a, in64);
}

template <int K>
void sweep32_dir(int dir, const sweep_args<float>& a, const double* in64, int grid, cudaStream_t s) {
    if (dir == 1 && a.seg_rows) seg32<K>(a, in64, s);
    if (a.n_items) {
        if (a.val16) {
            if (dir == 0) k_df32<0, K, true><<<grid, kSweepThreads, 0, s>>>(a, in64);
            else          k_df32<1, K, true><<<grid, kSweepThreads, 0, s>>>(a, in64);
        } else {
            if (dir == 0) k_df32<0, K, false><<<grid, kSweepThreads, 0, s>>>(a, in64);
            else          k_df32<1, K, false><<<grid, kSweepThreads, 0, s>>>(a, in64);
        }
    }
    if (dir == 0 && a.seg_rows) seg32<K>(a, in64, s);
}

}  // namespace

void launch_sweep64(int dir, const sweep_args<double>& a, int grid, cudaStream_t s) {
    const size_t smem = static_cast<size_t>(a.seg_rows) * sizeof(double);
    if (dir == 1 && a.seg_rows) { set_smem(k_seg64, smem); k_seg64<<<1, kSegThreads, smem, s>>>(a); }
    if (a.n_items) {
        if (dir == 0) k_df64<0><<<grid, kSweepThreads, 0, s>>>(a);
        else          k_df64<1><<<grid, kSweepThreads, 0, s>>>(a);
    }
    if (dir == 0 && a.seg_rows) { set_smem(k_seg64, smem); k_seg64<<<1, kSegThreads, smem, s>>>(a); }
}

void launch_sweep32(int dir, const sweep_args<float>& a, int grid, cudaStream_t s) {
    launch_sweep32_from64(dir, a, nullptr, grid, s);
}

void launch_sweep32_from64(int dir, const sweep_args<float>& a, const double* in64, int grid, cudaStream_t s) {
    switch (a.k) {
        case 1:  sweep32_dir<1>(dir, a, in64, grid, s); break;
        case 2:  sweep32_dir<2>(dir, a, in64, grid, s); break;
        case 4:  sweep32_dir<4>(dir, a, in64, grid, s); break;
        case 8:  sweep32_dir<8>(dir, a, in64, grid, s); break;
        default: sweep32_dir<16>(dir, a, in64, grid, s); break;
    }
}

int sweep_grid64(int num_sms) {
    int b0 = 0, b1 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_df64<0>, kSweepThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_df64<1>, kSweepThreads, 0);
    const int b = b0 < b1 ? b0 : b1;
    return (b > 0 ? b : 1) * num_sms;
}

template <int K>
void sweep32_batch_dir(int dir, const sweep_args<float>& a, int grid, cudaStream_t s) {
    if (!a.n_items) return;
    if (a.val16) {
        if (dir == 0) k_dw32<0, K, true><<<grid, kSweepThreads, 0, s>>>(a);
        else          k_dw32<1, K, true><<<grid, kSweepThreads, 0, s>>>(a);
    } else {
        if (dir == 0) k_dw32<0, K, false><<<grid, kSweepThreads, 0, s>>>(a);
        else          k_dw32<1, K, false><<<grid, kSweepThreads, 0, s>>>(a);
    }
}

void launch_sweep32_batch(int dir, const sweep_args<float>& a, int grid, cudaStream_t s) {
    switch (a.k) {
        case 1:  sweep32_batch_dir<1>(dir, a, grid, s); break;
        case 2:  sweep32_batch_dir<2>(dir, a, grid, s); break;
        case 4:  sweep32_batch_dir<4>(dir, a, grid, s); break;
        case 8:  sweep32_batch_dir<8>(dir, a, grid, s); break;
        case 16: sweep32_batch_dir<16>(dir, a, grid, s); break;
        case 32: sweep32_batch_dir<32>(dir, a, grid, s); break;
        case 64: sweep32_batch_dir<64>(dir, a, grid, s); break;
        default: sweep32_batch_dir<128>(dir, a, grid, s); break;
    }
}

template <int K>
int occ32_batch() {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_dw32<1, K, false>, kSweepThreads, 0);
    return b;
}

int sweep_grid32_batch(int k, int num_sms) {
    int b = 1;
    switch (k) {
        case 1: b = occ32_batch<1>(); break;
        case 2: b = occ32_batch<2>(); break;
        case 4: b = occ32_batch<4>(); break;
        case 8: b = occ32_batch<8>(); break;
        case 16: b = occ32_batch<16>(); break;
        case 32: b = occ32_batch<32>(); break;
        case 64: b = occ32_batch<64>(); break;
        default: b = occ32_batch<128>(); break;
    }
    return (b > 0 ? b : 1) * num_sms;
}

int sweep_grid32(int k, int num_sms) {
    int b = 1;
    switch (k) {
        case 1: b = occ32<1>(); break;
        case 2: b = occ32<2>(); break;
        case 4: b = occ32<4>(); break;
        case 8: b = occ32<8>(); break;
        default: b = occ32<16>(); break;
    }
    return (b > 0 ? b : 1) * num_sms;
}

void launch_fill64(double* p, size_t n, double v, cudaStream_t s) {
    if (n) k_fill64<<<fill_grid(n), 256, 0, s>>>(p, n, v);
}
void launch_fill32(float* p, size_t n, float v, cudaStream_t s) {
    if (n) k_fill32<<<fill_grid(n), 256, 0, s>>>(p, n, v);
}
void launch_fill_sent64(double* p, size_t n, cudaStream_t s) {
    double v;
    const uint64_t bits = kSent64;
    __builtin_memcpy(&v, &bits, sizeof(v));
    launch_fill64(p, n, v, s);
}
void launch_fill_sent32(float* p, size_t n, cudaStream_t s) {
    float v;
    const uint32_t bits = kSent32;
    __builtin_memcpy(&v, &bits, sizeof(v));
    launch_fill32(p, n, v, s);
}

}  // namespace apxb
