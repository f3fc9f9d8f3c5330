// Sync-free persistent triangular sweeps over the approximate-Cholesky factor
// (the preconditioner's forward and backward solves, the reference's
// dataflow_kernel, src/cuda_dataflow.cu:321-478, and its CPU counterpart
// omp_sptrsv::solve_levelset, include/apxchol/solver/sptrsv/omp.h:1094-1119).
//
// Design (B200):
//  * One launch per sweep, a resident grid of 256-thread blocks. Each warp
//    claims 32 consecutive rows in sweep order from an atomic ticket, one
//    thread per row. A row only waits on rows earlier in sweep order, which
//    were claimed earlier by warps that are running, so progress never
//    depends on scheduling.
//  * No level barriers and no separate ready flags: the output vector starts
//    filled with a signalling-NaN marker and a solved value replaces it, so one
//    relaxed 64-bit load both tests a dependency and fetches it. The kernel
//    re-arms the buffer the next sweep writes (reset), so no extra fill pass
//    runs between applications.
//  * Each thread streams its row's column indices and values through the
//    read-only path and keeps up to 8 dependency loads in flight. A thread
//    whose operands are ready consumes them and moves on; the others re-poll
//    only the missing ones on the warp's next pass (with a nanosleep backoff
//    when no lane of the warp progressed). Threads never wait for each other,
//    so a row may depend on a row of the same warp.
//  * Every wait has a time budget (globaltimer): a warp that makes no progress
//    for the budget records APXB_ERR_TIMEOUT in the engine's error word, and
//    every warp drains; the host turns it into an error status. Nothing spins
//    unbounded.
//  * fp64 sweep: products and sums are individually rounded (__dmul_rn /
//    __dadd_rn, no contraction) in the reference's order -- rows of "thin"
//    levels use the 4-way split sum of dot_thin (omp.h:1343-1357), rows of
//    "fat" levels one serial sum (omp.h:1434-1439) -- and the row is finished
//    with one correctly rounded subtract and divide (omp.h:1440). The result is
//    the reference CPU sweep's bytes.
//  * fp32 sweep: fp32 values, fp32 fused multiply-add accumulation in entry
//    order, k right-hand sides per row interleaved [row][k]: each factor entry
//    is read once for all k.
#include "kernels.cuh"

namespace apxb {

namespace {

constexpr int kBatch = 8;   // dependency loads in flight per thread (fp64)

__device__ __forceinline__ unsigned backoff_ns(int spins) {
    return spins < 2 ? 0u : min(32u << min(spins >> 1, 4), 512u);
}

// Warp-uniform check of the error word and the time budget. Returns true when
// the warp must drain (budget exhausted -> error raised, or another warp failed).
__device__ __forceinline__ bool wait_must_stop(dev_error* err, unsigned long long t0,
                                               unsigned long long budget, int where, uint32_t row) {
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

__device__ __forceinline__ void leave(sweep_ctl* ctl) {
    if ((threadIdx.x & 31) == 0) {
        const unsigned total = gridDim.x * (blockDim.x >> 5);
        if (atomicAdd(&ctl->done, 1u) == total - 1) {
            ctl->ticket = 0;
            ctl->done = 0;
        }
    }
}

template <int DIR>
__global__ void __launch_bounds__(kSweepThreads) k_sweep64(const sweep_args<double> a) {
    if (a.skip && *a.skip) return;
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned c = 0;
        int bad = 0;
        if (lane == 0) {
            c = atomicAdd(&a.ctl->ticket, 1u);
            bad = ld_relaxed_int(&a.err->code);
        }
        c = __shfl_sync(kFull, c, 0);
        bad = __shfl_sync(kFull, bad, 0);
        if (c >= a.nchunks || bad) break;

        const uint32_t pos = c * 32u + lane;
        const bool valid = pos < a.m;
        const uint32_t r = DIR == 0 ? pos : a.m - 1u - pos;
        uint32_t q = 0, qend = 0, gend = 0;
        double rhs = 0.0, d = 1.0;
        if (valid) {
            const uint32_t p0 = __ldg(a.ptr + r), p1 = __ldg(a.ptr + r + 1);
            q = DIR == 0 ? p0 : p0 + 1;
            qend = DIR == 0 ? p1 - 1 : p1;
            const uint32_t dslot = DIR == 0 ? p1 - 1 : p0;
            const bool thin = (__ldg(a.thin + (r >> 5)) >> (r & 31)) & 1u;
            gend = thin ? q + ((qend - q) & ~3u) : q;
            rhs = a.in[r];
            if (a.rhs_sub) rhs = __dsub_rn(rhs, *a.rhs_sub);
            if (a.reset) a.reset[r] = sent_of(0.0);
            d = static_cast<double>(__ldg(a.val + dslot));
        }
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, sum = 0.0;
        bool combined = false;
        bool active = valid;
        // Each lane keeps one batch of up to kBatch entries in flight. A lane
        // whose operands are ready consumes them and moves on; the others
        // re-poll only their missing ones on the next pass. Lanes never wait
        // for each other, so a row may depend on a row of the same warp.
        bool loaded = false, stop = false;
        uint32_t cnt = 0;
        unsigned need = 0;
        uint32_t jj[kBatch];
        float ww[kBatch];
        double yv[kBatch];
        int spins = 0;
        unsigned long long t_idle = 0;
        while (__any_sync(kFull, active)) {
            bool progress = false;
            if (active) {
                if (!loaded) {
                    cnt = min(static_cast<uint32_t>(kBatch), qend - q);
#pragma unroll
                    for (int k = 0; k < kBatch; ++k)
                        if (k < cnt) { jj[k] = __ldg(a.idx + q + k); ww[k] = __ldg(a.val + q + k); }
#pragma unroll
                    for (int k = 0; k < kBatch; ++k)
                        if (k < cnt) yv[k] = ld_relaxed(a.out + jj[k]);
                    need = 0;
#pragma unroll
                    for (int k = 0; k < kBatch; ++k)
                        if (k < cnt && is_sent(yv[k])) need |= 1u << k;
                    loaded = true;
                } else {
#pragma unroll
                    for (int k = 0; k < kBatch; ++k)
                        if ((need >> k) & 1u) yv[k] = ld_relaxed(a.out + jj[k]);
#pragma unroll
                    for (int k = 0; k < kBatch; ++k)
                        if (((need >> k) & 1u) && !is_sent(yv[k])) need &= ~(1u << k);
                }
                if (need == 0) {
#pragma unroll
                    for (int k = 0; k < kBatch; ++k) {
                        if (k < cnt) {
                            const double pr = __dmul_rn(static_cast<double>(ww[k]), yv[k]);
                            if (q + k < gend) {
                                const double t = __dadd_rn(s0, pr);
                                s0 = s1; s1 = s2; s2 = s3; s3 = t;
                            } else {
                                if (!combined) {
                                    sum = __dadd_rn(__dadd_rn(s0, s1), __dadd_rn(s2, s3));
                                    combined = true;
                                }
                                sum = __dadd_rn(sum, pr);
                            }
                        }
                    }
                    q += cnt;
                    loaded = false;
                    progress = true;
                    if (q == qend) {
                        if (!combined) sum = __dadd_rn(__dadd_rn(s0, s1), __dadd_rn(s2, s3));
                        const double v = __ddiv_rn(__dsub_rn(rhs, sum), d);
                        st_relaxed(a.out + r, v);
                        if (a.copy_out) a.copy_out[r] = v;
                        active = false;
                    }
                }
            }
            if (__any_sync(kFull, progress)) {
                spins = 0;
            } else {
                if (spins == 0 && lane == 0) t_idle = globaltimer();
                ++spins;
                if ((spins & 15) == 0 &&
                    wait_must_stop(a.err, __shfl_sync(kFull, t_idle, 0), a.budget_ns,
                                   DIR == 0 ? kFwdSweep : kBckSweep, r)) {
                    stop = true;
                    break;
                }
                const unsigned ns = backoff_ns(spins);
                if (ns) __nanosleep(ns);
            }
        }
        if (stop) break;
    }
    leave(a.ctl);
}

// ---- fp32, K right-hand sides per row ----

template <int K> struct vecf;
template <> struct vecf<1> { float v[1]; };
template <> struct vecf<2> { float v[2]; };
template <> struct vecf<4> { float v[4]; };
template <> struct vecf<8> { float v[8]; };
template <> struct vecf<16> { float v[16]; };

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

template <int DIR, int K>
__global__ void __launch_bounds__(kSweepThreads) k_sweep32(const sweep_args<float> a,
                                                           const double* in64) {
    constexpr int B = K >= 16 ? 2 : (K >= 8 ? 4 : 8);   // entries in flight per thread
    if (a.skip && *a.skip) return;
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned c = 0;
        int bad = 0;
        if (lane == 0) {
            c = atomicAdd(&a.ctl->ticket, 1u);
            bad = ld_relaxed_int(&a.err->code);
        }
        c = __shfl_sync(kFull, c, 0);
        bad = __shfl_sync(kFull, bad, 0);
        if (c >= a.nchunks || bad) break;

        const uint32_t pos = c * 32u + lane;
        const bool valid = pos < a.m;
        const uint32_t r = DIR == 0 ? pos : a.m - 1u - pos;
        uint32_t q = 0, qend = 0;
        float rhs[K], acc[K];
        float dinv = 1.0f, d = 1.0f;
#pragma unroll
        for (int s = 0; s < K; ++s) { rhs[s] = 0.0f; acc[s] = 0.0f; }
        if (valid) {
            const uint32_t p0 = __ldg(a.ptr + r), p1 = __ldg(a.ptr + r + 1);
            q = DIR == 0 ? p0 : p0 + 1;
            qend = DIR == 0 ? p1 - 1 : p1;
            d = __ldg(a.val + (DIR == 0 ? p1 - 1 : p0));
            (void)dinv;
            if (in64) {
#pragma unroll
                for (int s = 0; s < K; ++s) {
                    double v = in64[static_cast<size_t>(r) * K + s];
                    if (a.rhs_sub) v -= a.rhs_sub[s];
                    rhs[s] = static_cast<float>(v);
                }
            } else {
#pragma unroll
                for (int s = 0; s < K; ++s) rhs[s] = a.in[static_cast<size_t>(r) * K + s];
            }
            if (a.reset) {
                float sent[K];
#pragma unroll
                for (int s = 0; s < K; ++s) sent[s] = sent_of(0.0f);
                st_row<K>(a.reset + static_cast<size_t>(r) * K, sent);
            }
        }
        bool active = valid;
        bool loaded = false, stop = false;
        uint32_t cnt = 0;
        unsigned need = 0;
        uint32_t jj[B];
        float ww[B];
        float yv[B][K];
        int spins = 0;
        unsigned long long t_idle = 0;
        while (__any_sync(kFull, active)) {
            bool progress = false;
            if (active) {
                if (!loaded) {
                    cnt = min(static_cast<uint32_t>(B), qend - q);
#pragma unroll
                    for (int e = 0; e < B; ++e)
                        if (e < cnt) { jj[e] = __ldg(a.idx + q + e); ww[e] = __ldg(a.val + q + e); }
#pragma unroll
                    for (int e = 0; e < B; ++e)
                        if (e < cnt) ld_row<K>(a.out + static_cast<size_t>(jj[e]) * K, yv[e]);
                    need = 0;
#pragma unroll
                    for (int e = 0; e < B; ++e)
                        if (e < cnt && !row_ready<K>(yv[e])) need |= 1u << e;
                    loaded = true;
                } else {
#pragma unroll
                    for (int e = 0; e < B; ++e)
                        if ((need >> e) & 1u) ld_row<K>(a.out + static_cast<size_t>(jj[e]) * K, yv[e]);
#pragma unroll
                    for (int e = 0; e < B; ++e)
                        if (((need >> e) & 1u) && row_ready<K>(yv[e])) need &= ~(1u << e);
                }
                if (need == 0) {
#pragma unroll
                    for (int e = 0; e < B; ++e)
                        if (e < cnt)
#pragma unroll
                            for (int s = 0; s < K; ++s) acc[s] = __fmaf_rn(ww[e], yv[e][s], acc[s]);
                    q += cnt;
                    loaded = false;
                    progress = true;
                    if (q == qend) {
                        float v[K];
#pragma unroll
                        for (int s = 0; s < K; ++s) v[s] = __fdiv_rn(rhs[s] - acc[s], d);
                        st_row<K>(a.out + static_cast<size_t>(r) * K, v);
                        if (a.copy_out) {
#pragma unroll
                            for (int s = 0; s < K; ++s) a.copy_out[static_cast<size_t>(r) * K + s] = v[s];
                        }
                        active = false;
                    }
                }
            }
            if (__any_sync(kFull, progress)) {
                spins = 0;
            } else {
                if (spins == 0 && lane == 0) t_idle = globaltimer();
                ++spins;
                if ((spins & 15) == 0 &&
                    wait_must_stop(a.err, __shfl_sync(kFull, t_idle, 0), a.budget_ns,
                                   DIR == 0 ? kFwdSweep32 : kBckSweep32, r)) {
                    stop = true;
                    break;
                }
                const unsigned ns = backoff_ns(spins);
                if (ns) __nanosleep(ns);
            }
        }
        if (stop) break;
    }
    leave(a.ctl);
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

template <int DIR, int K>
void sweep32_k(const sweep_args<float>& a, const double* in64, int grid, cudaStream_t s) {
    k_sweep32<DIR, K><<<grid, kSweepThreads, 0, s>>>(a, in64);
}

template <int K>
int occ32() {
    int b0 = 0, b1 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_sweep32<0, K>, kSweepThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_sweep32<1, K>, kSweepThreads, 0);
    return b0 < b1 ? b0 : b1;
}

}  // namespace

void launch_sweep64(int dir, const sweep_args<double>& a, int grid, cudaStream_t s) {
    if (dir == 0) k_sweep64<0><<<grid, kSweepThreads, 0, s>>>(a);
    else          k_sweep64<1><<<grid, kSweepThreads, 0, s>>>(a);
}

void launch_sweep32(int dir, const sweep_args<float>& a, int grid, cudaStream_t s) {
    // The fp32 sweep reads its rhs from `in` (fp32) -- the fp64 variant used by
    // the PCG passes it as a double pointer through rhs-widening in pcg.cu.
    const double* in64 = nullptr;
    switch (a.k) {
        case 1:  dir == 0 ? sweep32_k<0, 1>(a, in64, grid, s) : sweep32_k<1, 1>(a, in64, grid, s); break;
        case 2:  dir == 0 ? sweep32_k<0, 2>(a, in64, grid, s) : sweep32_k<1, 2>(a, in64, grid, s); break;
        case 4:  dir == 0 ? sweep32_k<0, 4>(a, in64, grid, s) : sweep32_k<1, 4>(a, in64, grid, s); break;
        case 8:  dir == 0 ? sweep32_k<0, 8>(a, in64, grid, s) : sweep32_k<1, 8>(a, in64, grid, s); break;
        default: dir == 0 ? sweep32_k<0, 16>(a, in64, grid, s) : sweep32_k<1, 16>(a, in64, grid, s); break;
    }
}

void launch_sweep32_from64(const sweep_args<float>& a, const double* in64, int grid, cudaStream_t s) {
    switch (a.k) {
        case 1:  sweep32_k<0, 1>(a, in64, grid, s); break;
        case 2:  sweep32_k<0, 2>(a, in64, grid, s); break;
        case 4:  sweep32_k<0, 4>(a, in64, grid, s); break;
        case 8:  sweep32_k<0, 8>(a, in64, grid, s); break;
        default: sweep32_k<0, 16>(a, in64, grid, s); break;
    }
}

int sweep_grid64(int num_sms) {
    int b0 = 0, b1 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_sweep64<0>, kSweepThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_sweep64<1>, kSweepThreads, 0);
    const int b = b0 < b1 ? b0 : b1;
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
    static_assert(sizeof(v) == sizeof(bits), "");
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
