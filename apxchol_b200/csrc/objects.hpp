// Internal object definitions shared by the C ABI translation units
// (capi.cu, batch.cu). Not part of the public interface.
#pragma once
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <functional>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "apxb200.h"
#include "host_prep.hpp"
#include "kernels.cuh"

struct apxb_engine;
namespace apxb_detail {
int fail(int code, const std::string& msg);
// Runs an entry point's body and turns a host exception (an allocation that
// failed, a thread that could not start) into a status, so none crosses the C ABI.
template <class F>
int guarded(F&& body) noexcept {
    try {
        return body();
    } catch (const std::bad_alloc&) {
        return fail(APXB_ERR_INVALID, "host allocation failed");
    } catch (const std::exception& ex) {
        return fail(APXB_ERR_INVALID, std::string("host error: ") + ex.what());
    } catch (...) {
        return fail(APXB_ERR_INVALID, "host error");
    }
}
int center_k_from_env();
// A factor, operator or batch on engine e was destroyed.
void release_child(apxb_engine* e);
}  // namespace apxb_detail
using apxb_detail::fail;
using apxb_detail::guarded;

#define APXB_CK(call)                                                                            \
    do {                                                                                         \
        const cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                                   \
            return fail(e_ == cudaErrorMemoryAllocation ? APXB_ERR_OOM : APXB_ERR_CUDA,          \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                    \
    } while (0)


namespace apxb {
// The library's stream-ordered memory pool on `device` (created on first use,
// kept for the process): freed buffers stay mapped in it for the next
// allocation instead of going back to the driver, and freeing does not
// synchronize the device. nullptr when pools are off (APXB_NO_POOL=1) or the
// device has none; then plain cudaMalloc / cudaFree are used.
cudaMemPool_t device_pool(int device);
// Engines alive per device; the pool is trimmed when the last one goes.
void pool_engine_added(int device);
void pool_engine_removed(int device);
}  // namespace apxb

struct apxb_engine {
    int device = 0;
    cudaMemPool_t pool = nullptr;         // apxb::device_pool(device) for factor / operator / batch buffers
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    apxb::dev_error* d_err = nullptr;
    apxb::dev_error* h_err = nullptr;     // pinned
    unsigned long long budget_ns = 2000000000ull;
    uint64_t mem_budget = 0, mem_used = 0;
    double* d_partials = nullptr;         // [vec_grid * 4]
    unsigned* d_counters = nullptr;       // [16]
    double* d_scal = nullptr;             // [8]
    double* h_scal = nullptr;             // pinned [8]
    int vec_grid = 592;
    int center_k = 10;
    int sweep_grid = 0;                   // 0 = resident grid
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // staging for host-pointer entry points
    double* d_stage_a = nullptr; double* d_stage_b = nullptr; size_t stage_n = 0;
    double* h_stage_a = nullptr; double* h_stage_b = nullptr; size_t h_stage_n = 0;
    // Factors and operators alive on this engine. apxb_engine_destroy with
    // live children only marks the engine closing; the last child frees it.
    int children = 0;
    bool closing = false;

    int alloc(void** p, size_t bytes) {
        if (mem_budget && mem_used + bytes > mem_budget)
            return fail(APXB_ERR_BUDGET, "device memory budget exhausted: " + std::to_string(mem_used) + " + " +
                                             std::to_string(bytes) + " > " + std::to_string(mem_budget));
        cudaError_t e;
        if (pool) {   // stream-ordered; synchronized so that every stream may use the buffer at once
            e = cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        } else {
            e = cudaMalloc(p, bytes ? bytes : 16);
        }
        if (e != cudaSuccess) {
            *p = nullptr;
            cudaGetLastError();
            return fail(APXB_ERR_OOM, std::string(pool ? "cudaMallocFromPoolAsync: " : "cudaMalloc: ") +
                                          cudaGetErrorString(e));
        }
        mem_used += bytes;
        return APXB_OK;
    }
    // Frees a buffer from alloc(): in stream order on the engine stream (after
    // the work already queued there), without a device-wide synchronization.
    void release(void* p, size_t bytes) {
        if (p) {
            if (pool) cudaFreeAsync(p, stream);
            else cudaFree(p);
            mem_used -= bytes;
        }
    }
    // Reads and clears the device error word; returns its code (0 = none).
    int take_error() {
        if (cudaMemcpyAsync(h_err, d_err, sizeof(apxb::dev_error), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            return fail(APXB_ERR_CUDA, std::string("device fault: ") + cudaGetErrorString(cudaGetLastError()));
        if (h_err->code == 0) return APXB_OK;
        const int code = h_err->code;
        const std::string msg = code == APXB_ERR_TIMEOUT
            ? "a sweep wait exceeded its spin budget (kernel " + std::to_string(h_err->where) + ", row " +
                  std::to_string(h_err->info) + ")"
            : "device error " + std::to_string(code);
        cudaMemsetAsync(d_err, 0, sizeof(apxb::dev_error), stream);
        cudaStreamSynchronize(stream);
        return fail(code, msg);
    }
    int ensure_stage(size_t n) {
        if (stage_n < n) {
            release(d_stage_a, stage_n * 8); release(d_stage_b, stage_n * 8);
            d_stage_a = d_stage_b = nullptr; stage_n = 0;
            int rc = alloc(reinterpret_cast<void**>(&d_stage_a), n * 8);
            if (rc) return rc;
            rc = alloc(reinterpret_cast<void**>(&d_stage_b), n * 8);
            if (rc) return rc;
            stage_n = n;
        }
        if (h_stage_n < n) {
            if (h_stage_a) cudaFreeHost(h_stage_a);
            if (h_stage_b) cudaFreeHost(h_stage_b);
            h_stage_a = h_stage_b = nullptr; h_stage_n = 0;
            APXB_CK(cudaMallocHost(&h_stage_a, n * 8));
            APXB_CK(cudaMallocHost(&h_stage_b, n * 8));
            h_stage_n = n;
        }
        return APXB_OK;
    }
};

struct apxb_factor {
    apxb_engine* e = nullptr;
    apxb::prepared_factor h;
    int precision = APXB_PREC_FP64;
    double drop_rel = 0.0;                             // threshold in effect
    uint64_t apply_count = 0;
    uint64_t dev_bytes = 0;
    std::vector<std::pair<void*, size_t>> owned;
    uint32_t* perm = nullptr;
    double *Y = nullptr, *Z = nullptr, *zp = nullptr;   // fp64 tracked buffers, permuted rhs
    bool y_armed = false, z_armed = false;
    apxb::sweep_ctl* ctl = nullptr;                    // [2]
    int grid64 = 0;
    // sweep plans (the kernels' layout), per direction
    uint32_t* info[2] = {nullptr, nullptr};
    uint32_t* ord[2] = {nullptr, nullptr};
    uint32_t* ptr[2] = {nullptr, nullptr};
    uint32_t* idx[2] = {nullptr, nullptr};
    float* val[2] = {nullptr, nullptr};                // fp32 values (not on fp16 factors)
    uint16_t* val16[2] = {nullptr, nullptr};           // fp16 factors: binary16 values
    float* diag16 = nullptr;                           // fp16 factors: per-row diagonal
    double* inv_scale2 = nullptr;                      // fp16 factors: per-row (1 / s)^2, fp64
    uint32_t* chunk[2] = {nullptr, nullptr};           // claim units (host_prep.hpp, chunk_plan)
    uint32_t n_chunks[2] = {0, 0};
    uint32_t *seg_row[2] = {nullptr, nullptr}, *seg_lvl[2] = {nullptr, nullptr};
    uint32_t *seg_ptr[2] = {nullptr, nullptr}, *seg_idx[2] = {nullptr, nullptr};
    float* seg_val[2] = {nullptr, nullptr};
    // Factors prepared on the device (devprep.cu): the canonical arrays stay
    // there for batch plans; h then holds sizes and counts only, and its
    // arrays are filled on demand (factor_host_arrays).
    struct device_canon {
        bool on = false;
        uint32_t *csc_ptr = nullptr, *csc_idx = nullptr, *csr_ptr = nullptr, *csr_idx = nullptr;
        float *csc_val = nullptr, *csr_val = nullptr;
        int32_t* fl = nullptr;                         // forward level of every row
        uint32_t* lb = nullptr;                        // forward level bounds (levels are row ranges)
        int32_t n_levels = 0;
        std::vector<uint8_t> thin_level;               // per forward level
    } dev;
    bool host_arrays = true;                           // h holds the canonical arrays
    // fp32 sweeps, k right-hand sides
    float *Yf = nullptr, *Zf = nullptr;
    size_t f32_cap = 0;                                // floats per buffer
    bool yf_armed = false, zf_armed = false;
    int f32_k = 0;

    template <class T>
    int dalloc(T** p, size_t count) {
        const size_t bytes = count * sizeof(T);
        const int rc = e->alloc(reinterpret_cast<void**>(p), bytes);
        if (rc) return rc;
        owned.emplace_back(*p, bytes);
        dev_bytes += bytes;
        return APXB_OK;
    }
    ~apxb_factor() {
        for (auto& [p, b] : owned) e->release(p, b);
    }
};

struct apxb_operator {
    apxb_engine* e = nullptr;
    uint32_t n = 0;
    uint64_t nnz = 0;
    std::vector<std::pair<void*, size_t>> owned;
    int32_t *ptr = nullptr, *idx = nullptr;
    double* val = nullptr;    // fp64 values (null once narrowed into valf)
    float* valf = nullptr;    // fp32 values when every value is fp32-exact (or forced)
    uint32_t* perm = nullptr;
    // SpMV rows longer than apxb::kLongRowPlain (see pcg_ptrs)
    uint32_t n_long = 0, n_chunks = 0;
    uint32_t *lr_row = nullptr, *lr_first = nullptr, *ch_lo = nullptr, *ch_hi = nullptr;
    double* ch_part = nullptr;
    // PCG workspace (permuted ordering) + original-ordering staging
    double *x = nullptr, *r = nullptr, *p = nullptr, *Ap = nullptr, *b_orig = nullptr, *x_orig = nullptr;
    apxb::pcg_state* st = nullptr;
    apxb::pcg_state* h_st = nullptr;   // pinned
    // cached loop graph for one factor
    const apxb_factor* graph_factor = nullptr;
    cudaGraphExec_t loop = nullptr;
    bool loop_conditional = false;

    template <class T>
    int dalloc(T** q, size_t count) {
        const size_t bytes = count * sizeof(T);
        const int rc = e->alloc(reinterpret_cast<void**>(q), bytes);
        if (rc) return rc;
        owned.emplace_back(*q, bytes);
        return APXB_OK;
    }
    // Releases one buffer this operator allocated (no-op for any other pointer).
    void drop(void* q) {
        for (size_t i = 0; i < owned.size(); ++i)
            if (owned[i].first == q) {
                e->release(q, owned[i].second);
                owned.erase(owned.begin() + static_cast<std::ptrdiff_t>(i));
                return;
            }
    }
    ~apxb_operator() {
        if (loop) cudaGraphExecDestroy(loop);
        for (auto& [q, b] : owned) e->release(q, b);
        if (h_st) cudaFreeHost(h_st);
    }
};

// The plan pointers of direction dir of factor f (forward: CSR(L11), backward:
// CSC(L11)) in a sweep's launch arguments; every sweep entry point starts from
// this, then sets its vectors, counters and error word.
template <class T>
inline void plan_args(const apxb_factor* f, int dir, apxb::sweep_args<T>& a) {
    const apxb::sweep_plan& pl = dir == 0 ? f->h.fwd_plan : f->h.bck_plan;
    a.m = f->h.m;
    a.n_items = pl.n_items;
    a.info = f->info[dir];
    a.ord = f->ord[dir];
    a.ptr = f->ptr[dir];
    a.idx = f->idx[dir];
    a.val = f->val[dir];
    a.val16 = f->val16[dir];
    a.diag16 = f->diag16;
    a.in_scale2 = nullptr;   // set for the backward of an fp16 factor by its caller
    a.seg_first = pl.seg_first;
    a.seg_rows = pl.seg_rows;
    a.seg_levels = pl.seg_levels;
    a.seg_row = f->seg_row[dir];
    a.seg_lvl = f->seg_lvl[dir];
    a.seg_ptr = f->seg_ptr[dir];
    a.seg_idx = f->seg_idx[dir];
    a.seg_val = f->seg_val[dir];
    a.chunk = f->chunk[dir];
    a.n_chunks = f->n_chunks[dir];
}

namespace apxb {
// Device preparation (devprep.cu): the host preparation's arrays, byte for
// byte, built by kernels. Applies to fp32/fp64 storage with round sizes.
bool device_prep_applies(bool fp16, uint32_t n_rounds);
// Fills f's plans (device), f->dev and f->h's sizes; "" or the reason it
// failed (*alloc_rc set when a device allocation failed).
std::string prepare_factor_device(apxb_factor* f, uint32_t n, const uint32_t* colptr, const uint32_t* rowidx,
                                  const float* vals, const uint32_t* perm, bool sddm, const uint64_t* rounds,
                                  uint32_t n_rounds, double drop_rel, int* alloc_rc);
// Host copies of a device-prepared factor's canonical arrays, levels and thin bits.
std::string factor_host_arrays(apxb_factor* f);
// One plan on the device: factor plan (col_lanes 0) or batch plan.
struct dev_plan_out {
    uint32_t n_items = 0, n_chunks = 0;
    uint64_t n_entries = 0;
    uint32_t *info = nullptr, *ord = nullptr, *ptr = nullptr, *idx = nullptr, *chunk = nullptr;
    float* val = nullptr;
};
std::string batch_plan_device(const apxb_factor* f, int dir, uint32_t col_lanes,
                              const std::function<std::string(void**, size_t)>& alloc_bytes, dev_plan_out& out,
                              cudaStream_t s);
// P A P^T into a->ptr / idx / val on the device; hptr receives the row offsets.
std::string permute_operator_device(apxb_operator* a, uint32_t n, const int32_t* colptr, const int32_t* rowidx,
                                    const double* vals, const uint32_t* perm, std::vector<int32_t>& hptr, int* alloc_rc);
// Storage precision of a's values: want > 0 stores them in fp32, want == 0 keeps
// fp64, want < 0 stores fp32 when every value is fp32-exact. fp32 storage
// narrows a->val into a->valf and releases a->val.
std::string operator_precision_device(apxb_operator* a, int want, int* alloc_rc);
}  // namespace apxb
