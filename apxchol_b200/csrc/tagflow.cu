// The reference's raw dataflow sweep entry points, apxchol::dataflow_solve /
// dataflow_solve_fp16 / dataflow_grid_size / dataflow_prefetch_depth
// (include/apxchol/solver/sptrsv/cuda_dataflow.h:160-208), on sm_100a, for
// callers that drive the sweep with the reference's own plan tables
// (cuda_host.h: dataflow_build_plan) -- the reference's GPU tests do.
//
// The contract is the reference's (cuda_dataflow.h:20-120), restated here:
//  * T out = rhs, T triangular in CSR with the diagonal inside every row;
//    sweep order is the row order (forward) or its reverse (back);
//  * every row i owns a 64-bit tagged word tag[i] = {value, epoch}; a sweep
//    publishes row i by storing {out[i], epoch} in one relaxed 64-bit store,
//    and a consumer reads value and flag in one load (no fence on the data
//    path); words of another epoch are "not yet";
//  * warps claim batches b = 0, 1, ... in order from ctrl[0]; batch_spec[b]
//    < 0 is a plain batch: the rows at sweep positions [batch_start[b],
//    batch_start[b+1]) packed into 32 lanes, a row of `len` entries
//    (diagonal included) taking the smallest power-of-two group G <= 32 with
//    G * kPre >= len, aligned to G (dataflow_lane_group); lane `sub` of the
//    group takes entries sub, sub + G, ... in order. batch_spec[b] >= 0 names
//    a special item spec[..]: a SEGMENT {row, lo, hi, slot} sums the row's CSR
//    slice [lo, hi) (diagonal skipped) with 32 lanes and publishes the partial
//    in tag[m + slot]; a FINALIZER {~row, s0, S, dpos} adds slots [s0, s0 + S)
//    in slot order, divides by the diagonal and publishes the row;
//  * ctrl = {ticket, finished warps} is zero at entry and reset to zero by
//    the last warp out.
// Values: fp32 (vals), or binary16 (vals16, widened exactly) with the row's
// fp32 diagonal diag[i] instead of its diagonal slot and, when in_scale is
// given, rhs[i] * in_scale[i] formed in fp64 and rounded once.
//
// The kernel is this library's own: a lane keeps up to kPre entries of its
// row in flight and consumes them in entry order as their words arrive; a row
// that needs more than kPre entries per lane (G = 32, alone in its batch)
// walks its chunks lane by lane, each lane loading its next chunk as soon as
// it has consumed the current one. A group's lanes are combined by a fixed
// xor butterfly, so the result depends only on the row lengths and the plan:
// bit-identical across launches and grid sizes. Every wait is bounded (one
// second without progress): a plan that breaks the contract ends the launch
// with an error recorded for apxb_dataflow_status instead of hanging.
#include <cstdlib>
#include <cstring>
#include <string>

#include <cuda_fp16.h>

#include "device.cuh"
#include "objects.hpp"

namespace apxb {
namespace {

constexpr int kPre = 8;                       // entries of a row in flight per lane
constexpr int kDfThreads = 256;               // kDataflowBlock of the contract
constexpr unsigned long long kDfBudgetNs = 1000000000ull;
constexpr int kWhereDf = 10;                  // dev_error::where of this kernel

__device__ dev_error g_df_err;                // first failure of any launch since the last status read

struct df_args {
    int m;
    int reverse;
    const int* rowptr;
    const int* colidx;
    const float* vals;                        // fp32 storage (vals16 == nullptr)
    const uint16_t* vals16;                   // binary16 storage
    const float* diag;                        // binary16 storage: per-row fp32 diagonal
    const double* in_scale;                   // nullable: per-row rhs scale (fp64)
    const int* batch_start;
    const int* batch_spec;
    const int4* spec;
    int n_batches;
    unsigned long long* tag;
    unsigned epoch;
    int* ctrl;
    const float* rhs;
    float* out;
};

__device__ __forceinline__ unsigned long long ld_tag(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_tag(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long pack_tag(float v, unsigned e) {
    return (static_cast<unsigned long long>(e) << 32) | __float_as_uint(v);
}
__device__ __forceinline__ bool tag_is(unsigned long long t, unsigned e) { return static_cast<unsigned>(t >> 32) == e; }
__device__ __forceinline__ float tag_val(unsigned long long t) { return __uint_as_float(static_cast<unsigned>(t)); }

__device__ __forceinline__ int lane_group(int entries) {
    int G = 1;
    while (G < 32 && G * kPre < entries) G <<= 1;
    return G;
}

template <bool H>
__device__ __forceinline__ float weight(const df_args& a, int t) {
    if constexpr (H) return __half2float(__ushort_as_half(__ldg(a.vals16 + t)));
    else return __ldg(a.vals + t);
}

__device__ __forceinline__ float row_rhs(const df_args& a, int row) {
    const float r = a.rhs[row];
    return a.in_scale ? static_cast<float>(static_cast<double>(r) * a.in_scale[row]) : r;
}

// The idle bookkeeping of a warp's wait: true when the warp must stop waiting
// (another warp failed, or lane 0 saw no progress for the budget: a timeout is
// recorded). Every lane of the warp calls idle() together, and progress() only
// with a warp-uniform condition; lane 0's count alone decides, and the
// decision reaches the lanes through one shuffle that every call executes.
struct df_clock {
    int spins = 0;
    unsigned long long t0 = 0;
    __device__ __forceinline__ void progress() { spins = 0; }
    __device__ __forceinline__ bool idle(int row) {
        if (spins == 0) t0 = globaltimer();
        ++spins;
        int stop = 0;
        if ((threadIdx.x & 31) == 0 && (spins & 15) == 0) {
            if (ld_relaxed_int(&g_df_err.code) != 0) stop = 1;
            else if (globaltimer() - t0 > kDfBudgetNs) {
                raise_error(&g_df_err, APXB_ERR_TIMEOUT, kWhereDf, static_cast<unsigned long long>(row));
                stop = 1;
            }
        }
        if (__shfl_sync(kFull, stop, 0)) return true;
        if (spins > 4) __nanosleep(spins > 64 ? 256u : 32u);
        return false;
    }
};

// One lane's walk over its share of a CSR range: entries first, first + step,
// ... below end, kPre at a time; `skip` (a column) is not accumulated.
struct lane_walk {
    int t, end, step, skip;
    int cnt;                                  // entries of the current chunk
    int kpos;                                 // consumed entries of the current chunk
    int jj[kPre];
    float w[kPre];
    unsigned long long v[kPre];
    float acc, dsum;                          // running sum; diagonal weight seen (fp32 storage)

    template <bool H>
    __device__ __forceinline__ void load(const df_args& a, const unsigned long long* words) {
        cnt = 0;
        kpos = 0;
#pragma unroll
        for (int k = 0; k < kPre; ++k) {
            const int q = t + k * step;
            if (q < end) {
                jj[k] = __ldg(a.colidx + q);
                w[k] = jj[k] == skip ? 0.0f : weight<H>(a, q);
                if (!H && jj[k] == skip) dsum += __ldg(a.vals + q);
                cnt = k + 1;
            }
        }
#pragma unroll
        for (int k = 0; k < kPre; ++k)
            if (k < cnt && jj[k] != skip) v[k] = ld_tag(words + jj[k]);
        t += kPre * step;
    }
    // Consumes the arrived entries in order; true when it moved.
    __device__ __forceinline__ bool consume(unsigned e, int skip_col) {
        const int before = kpos;
#pragma unroll
        for (int k = 0; k < kPre; ++k)
            if (k == kpos && k < cnt) {
                if (jj[k] == skip_col) ++kpos;
                else if (tag_is(v[k], e)) { acc = __fmaf_rn(w[k], tag_val(v[k]), acc); ++kpos; }
            }
        return kpos != before;
    }
    __device__ __forceinline__ void repoll(const unsigned long long* words, int skip_col) {
#pragma unroll
        for (int k = 0; k < kPre; ++k)
            if (k >= kpos && k < cnt && jj[k] != skip_col) v[k] = ld_tag(words + jj[k]);
    }
    __device__ __forceinline__ bool chunk_done() const { return kpos >= cnt; }
    __device__ __forceinline__ bool more() const { return t < end; }
};

// Sum over the aligned group of G lanes (fixed butterfly; every lane runs all
// five steps so the shuffles stay warp-uniform).
__device__ __forceinline__ float group_sum(float x, int G) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float y = __shfl_xor_sync(kFull, x, o);
        if (o < G) x += y;
    }
    return x;
}

// A plain batch: up to 32 rows, each in its lane group; rows that wait on rows
// of the same batch are served by the loop (ready groups publish, the others
// re-poll). Returns false when the warp must stop.
template <bool H>
__device__ bool plain_batch(const df_args& a, int q0, int q1, unsigned lane) {
    const int n = q1 - q0;
    int my_len = 0, my_row_pos = 0;
    if (static_cast<int>(lane) < n) {
        const int q = q0 + static_cast<int>(lane);
        const int row = a.reverse ? a.m - 1 - q : q;
        my_len = __ldg(a.rowptr + row + 1) - __ldg(a.rowptr + row);
        my_row_pos = row;
    }
    int row = -1, sub = 0, G = 1, pos = 0;
    bool bad = false;
    for (int i = 0; i < n; ++i) {
        const int li = __shfl_sync(kFull, my_len, i);
        const int ri = __shfl_sync(kFull, my_row_pos, i);
        const int g = lane_group(li);
        const int aligned = (pos + g - 1) & ~(g - 1);
        if (aligned + g > 32) { bad = true; break; }
        if (static_cast<int>(lane) >= aligned && static_cast<int>(lane) < aligned + g) {
            row = ri; sub = static_cast<int>(lane) - aligned; G = g;
        }
        pos = aligned + g;
    }
    if (bad) {   // the batch does not fit one warp: not a plan of this contract
        if (lane == 0) raise_error(&g_df_err, APXB_ERR_INVALID, kWhereDf, static_cast<unsigned long long>(q0));
        return false;
    }
    lane_walk wk;
    wk.acc = 0.0f;
    wk.dsum = 0.0f;
    float r = 0.0f, d = 1.0f;
    bool published = row < 0;   // idle lanes count as published
    if (row >= 0) {
        wk.t = __ldg(a.rowptr + row) + sub;
        wk.end = __ldg(a.rowptr + row + 1);
        wk.step = G;
        wk.skip = row;
        wk.template load<H>(a, a.tag);
        if (sub == 0) {
            r = row_rhs(a, row);
            if (H) d = __ldg(a.diag + row);
        }
    } else {
        wk.cnt = 0; wk.kpos = 0; wk.t = 0; wk.end = 0; wk.step = 1; wk.skip = -1;
    }
    df_clock clk;
    for (;;) {
        bool moved = false;
        if (row >= 0 && !published) {
            moved = wk.consume(a.epoch, row);
            while (wk.chunk_done() && wk.more()) {   // next chunk of a long row (G = 32)
                wk.template load<H>(a, a.tag);
                moved = wk.consume(a.epoch, row) || true;
            }
        }
        const bool lane_ready = published || (wk.chunk_done() && !wk.more());
        const unsigned ready = __ballot_sync(kFull, lane_ready);
        const unsigned gmask = G == 32 ? kFull : (((1u << G) - 1u) << (static_cast<int>(lane) & ~(G - 1)));
        const bool group_ready = row >= 0 && !published && (ready & gmask) == gmask;
        const float s = group_sum(wk.acc, G);
        const float dd = H ? 0.0f : group_sum(wk.dsum, G);
        bool pub = false;
        if (group_ready) {
            if (sub == 0) {
                const float y = __fdiv_rn(r - s, H ? d : dd);
                a.out[row] = y;
                st_tag(a.tag + row, pack_tag(y, a.epoch));
            }
            published = true;
            pub = true;
        }
        if (__all_sync(kFull, published)) return true;
        if (__any_sync(kFull, moved || pub)) clk.progress();
        else if (clk.idle(row)) return false;
        if (row >= 0 && !published) wk.repoll(a.tag, row);
    }
}

// A segment: 32 lanes over the CSR slice [lo, hi) of `row` (diagonal
// skipped); the partial goes to tag[m + slot].
template <bool H>
__device__ bool segment(const df_args& a, int row, int lo, int hi, int slot, unsigned lane) {
    lane_walk wk;
    wk.acc = 0.0f;
    wk.dsum = 0.0f;
    wk.t = lo + static_cast<int>(lane);
    wk.end = hi;
    wk.step = 32;
    wk.skip = row;
    wk.template load<H>(a, a.tag);
    df_clock clk;
    for (;;) {
        bool moved = wk.consume(a.epoch, row);
        while (wk.chunk_done() && wk.more()) {
            wk.template load<H>(a, a.tag);
            wk.consume(a.epoch, row);
            moved = true;
        }
        if (__all_sync(kFull, wk.chunk_done() && !wk.more())) break;
        if (__any_sync(kFull, moved)) clk.progress();
        else if (clk.idle(row)) return false;
        wk.repoll(a.tag, row);
    }
    const float s = group_sum(wk.acc, 32);
    if (lane == 0) st_tag(a.tag + a.m + slot, pack_tag(s, a.epoch));
    return true;
}

// A finalizer: slots [s0, s0 + S) added in slot order (lane-strided, then the
// butterfly), divided by the diagonal (vals[dpos], or diag[row] for binary16).
template <bool H>
__device__ bool finalize(const df_args& a, int row, int s0, int S, int dpos, unsigned lane) {
    const unsigned long long* slots = a.tag + a.m + s0;
    float acc = 0.0f;
    df_clock clk;
    for (int base = 0; base < S; base += 32) {
        const int s = base + static_cast<int>(lane);
        bool have = s >= S;
        unsigned long long v = have ? 0ull : ld_tag(slots + s);
        for (;;) {
            bool got = false;
            if (!have && tag_is(v, a.epoch)) { acc += tag_val(v); have = true; got = true; }
            if (__all_sync(kFull, have)) break;
            if (__any_sync(kFull, got)) clk.progress();
            else if (clk.idle(row)) return false;
            if (!have) v = ld_tag(slots + s);
        }
    }
    const float s = group_sum(acc, 32);
    if (lane == 0) {
        const float d = H ? __ldg(a.diag + row) : __ldg(a.vals + dpos);
        const float y = __fdiv_rn(row_rhs(a, row) - s, d);
        a.out[row] = y;
        st_tag(a.tag + row, pack_tag(y, a.epoch));
    }
    return true;
}

template <bool H>
__global__ void __launch_bounds__(kDfThreads) k_tagflow(const df_args a) {
    const unsigned lane = threadIdx.x & 31u;
    for (;;) {
        int b = 0;
        if (lane == 0) b = atomicAdd(a.ctrl, 1);
        b = __shfl_sync(kFull, b, 0);
        if (b >= a.n_batches) break;
        const int sel = __ldg(a.batch_spec + b);
        bool ok;
        if (sel < 0) {
            ok = plain_batch<H>(a, __ldg(a.batch_start + b), __ldg(a.batch_start + b + 1), lane);
        } else {
            const int4 sp = __ldg(a.spec + sel);
            ok = sp.x >= 0 ? segment<H>(a, sp.x, sp.y, sp.z, sp.w, lane) : finalize<H>(a, ~sp.x, sp.y, sp.z, sp.w, lane);
        }
        if (!ok) break;
    }
    if (lane == 0) {   // the last warp out resets the claim counters for the next launch
        __threadfence();
        const int total = static_cast<int>(gridDim.x * (blockDim.x >> 5));
        if (atomicAdd(a.ctrl + 1, 1) == total - 1) {
            a.ctrl[0] = 0;
            a.ctrl[1] = 0;
            __threadfence();
        }
    }
}

int env_blocks() {
    const char* e = std::getenv("APXCHOL_GPU_DATAFLOW_BLOCKS");
    if (!e || !*e) return 0;
    const long v = std::strtol(e, nullptr, 10);
    return v > 0 && v < (1 << 24) ? static_cast<int>(v) : 0;
}

void launch(const df_args& a, int grid, cudaStream_t s, bool fp16) {
    if (a.m <= 0 || a.n_batches <= 0 || grid <= 0) return;
    if (fp16) k_tagflow<true><<<grid, kDfThreads, 0, s>>>(a);
    else k_tagflow<false><<<grid, kDfThreads, 0, s>>>(a);
}

}  // namespace
}  // namespace apxb

namespace apxchol {

int dataflow_prefetch_depth() { return apxb::kPre; }

int dataflow_grid_size(bool fp16) {
    const int forced = apxb::env_blocks();
    if (forced) return forced;
    int dev = 0, sms = 1, b = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 1;
    if (fp16) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, apxb::k_tagflow<true>, apxb::kDfThreads, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, apxb::k_tagflow<false>, apxb::kDfThreads, 0);
    return (b > 0 ? b : 1) * sms;
}

void dataflow_solve(cudaStream_t stream, int m, bool reverse, const int* rowptr, const int* colidx, const float* vals,
                    const int* batch_start, const int* batch_spec, const int4* spec, int n_batches,
                    unsigned long long* tag, unsigned epoch, int* ctrl, int grid, const float* rhs, float* out) {
    const apxb::df_args a{m, reverse ? 1 : 0, rowptr, colidx, vals, nullptr, nullptr, nullptr, batch_start, batch_spec,
                          spec, n_batches, tag, epoch, ctrl, rhs, out};
    apxb::launch(a, grid, stream, false);
}

void dataflow_solve_fp16(cudaStream_t stream, int m, bool reverse, const int* rowptr, const int* colidx,
                         const unsigned short* vals16, const float* diag, const double* in_scale,
                         const int* batch_start, const int* batch_spec, const int4* spec, int n_batches,
                         unsigned long long* tag, unsigned epoch, int* ctrl, int grid, const float* rhs, float* out) {
    const apxb::df_args a{m, reverse ? 1 : 0, rowptr, colidx, nullptr, vals16, diag, in_scale, batch_start, batch_spec,
                          spec, n_batches, tag, epoch, ctrl, rhs, out};
    apxb::launch(a, grid, stream, true);
}

}  // namespace apxchol

extern "C" int apxb_dataflow_status(void) {
    apxb::dev_error e{};
    cudaError_t rc = cudaMemcpyFromSymbol(&e, apxb::g_df_err, sizeof(e));
    if (rc != cudaSuccess) return apxb_detail::fail(APXB_ERR_CUDA, std::string("apxb_dataflow_status: ") + cudaGetErrorString(rc));
    if (e.code == 0) return APXB_OK;
    const apxb::dev_error zero{};
    rc = cudaMemcpyToSymbol(apxb::g_df_err, &zero, sizeof(zero));
    if (rc != cudaSuccess) return apxb_detail::fail(APXB_ERR_CUDA, std::string("apxb_dataflow_status: ") + cudaGetErrorString(rc));
    return apxb_detail::fail(e.code, e.code == APXB_ERR_TIMEOUT
                                         ? "dataflow sweep: a wait made no progress for 1 s at row " + std::to_string(e.info) +
                                               " (the plan or the tag epoch breaks the contract)"
                                         : "dataflow sweep: a plain batch does not fit one warp (position " +
                                               std::to_string(e.info) + ")");
}
