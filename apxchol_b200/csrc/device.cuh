// Device primitives shared by the solve-phase kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace apxb {

constexpr unsigned kFull = 0xffffffffu;

// "Not yet solved" markers of the sweep outputs. They are signalling NaNs:
// IEEE arithmetic never produces one (every NaN result is quiet), so a solved
// value can never be mistaken for the marker. A solved row's value is itself
// its ready flag: one 64-bit (or 32-bit) load both tests readiness and
// delivers the operand.
constexpr uint64_t kSent64 = 0xFFF5A5A5A5A5A5A5ull;
constexpr uint32_t kSent32 = 0xFFA5A5A5u;

// Error word shared by all kernels of an engine. The first failure wins.
struct dev_error {
    int code;            // 0 = ok, else an APXB_ERR_* value
    int where;           // kernel id
    unsigned long long info;
};

enum kernel_id : int {
    kFwdSweep = 1, kBckSweep = 2, kFwdSweep32 = 3, kBckSweep32 = 4,
};

__device__ __forceinline__ double ld_relaxed(const double* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return __longlong_as_double(static_cast<long long>(v));
}
__device__ __forceinline__ float ld_relaxed(const float* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return __uint_as_float(v);
}
__device__ __forceinline__ void st_relaxed(double* p, double x) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" :: "l"(p), "l"(__double_as_longlong(x)) : "memory");
}
__device__ __forceinline__ void st_relaxed(float* p, float x) {
    asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" :: "l"(p), "r"(__float_as_uint(x)) : "memory");
}
__device__ __forceinline__ int ld_relaxed_int(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool is_sent(double v) {
    return static_cast<unsigned long long>(__double_as_longlong(v)) == kSent64;
}
__device__ __forceinline__ bool is_sent(float v) { return __float_as_uint(v) == kSent32; }
__device__ __forceinline__ double sent_of(double) { return __longlong_as_double(static_cast<long long>(kSent64)); }
__device__ __forceinline__ float sent_of(float) { return __uint_as_float(kSent32); }

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void raise_error(dev_error* e, int code, int where, unsigned long long info) {
    if (atomicCAS(&e->code, 0, code) == 0) {
        e->where = where;
        e->info = info;
    }
}

// Deterministic block sum of NV values: a fixed xor-butterfly inside each warp,
// then warp 0 adds the warp totals in warp order. Result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem /* [NV*32] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(kFull, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) smem[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = lane < nw ? smem[k * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
            v[k] = s;
        }
    }
}

// Grid-level deterministic reduction: every block stores its NV partials, the
// last block to arrive sums them in block order (lanes stride the blocks, then
// a fixed butterfly) and returns true in thread 0 of that block with the totals
// in `tot`; the counter is reset for the next launch. A fixed grid size makes
// the result bit-identical run to run.
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double* partials, unsigned* counter,
                                         double (&tot)[NV]) {
    __shared__ double red[NV * 32];
    __shared__ bool last;
    block_sum<NV>(v, red);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) partials[static_cast<size_t>(blockIdx.x) * NV + k] = v[k];
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = 0.0;
            for (unsigned b = lane; b < gridDim.x; b += 32)
                s += ld_relaxed(partials + static_cast<size_t>(b) * NV + k);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
            tot[k] = s;
        }
        if (lane == 0) *counter = 0;
    }
    return threadIdx.x == 0;
}

}  // namespace apxb
