// The C ABI (include/apxb200.h): engines, factors, operators and the solve
// phase's entry points. No exception crosses the boundary; every failure is a
// negative status with the message in apxb_last_error().
#include "apxb200.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "objects.hpp"

namespace {

int env_int(const char* name, int dflt) {
    const char* v = std::getenv(name);
    return (v && *v) ? std::atoi(v) : dflt;
}

thread_local std::string g_err;

}  // namespace

namespace apxb_detail {

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

// center-k period as the reference's env knobs resolve it (env_knobs.h:90-103).
int center_k_from_env() {
    int k = env_int("APXCHOL_CENTER_K", 10);
    if (k < 1) k = 10;
    const char* g = std::getenv("APXCHOL_GROUND");
    if (g && std::strcmp(g, "center") == 0) k = 1;
    return k;
}

}  // namespace apxb_detail
using apxb_detail::center_k_from_env;

extern "C" {

const char* apxb_last_error(void) { return g_err.c_str(); }
const char* apxb_version(void) { return "apxb200 0.1 (sm_100a)"; }

int apxb_engine_create(int device, apxb_engine** out) {
    if (!out) return fail(APXB_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    APXB_CK(cudaGetDeviceCount(&ndev));
    if (device == APXB_CURRENT_DEVICE) APXB_CK(cudaGetDevice(&device));
    if (device < 0 || device >= ndev) return fail(APXB_ERR_INVALID, "no such device " + std::to_string(device));
    APXB_CK(cudaSetDevice(device));
    std::unique_ptr<apxb_engine> e(new (std::nothrow) apxb_engine);
    if (!e) return fail(APXB_ERR_INVALID, "host allocation failed");
    e->device = device;
    APXB_CK(cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, device));
    APXB_CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    e->vec_grid = e->num_sms * 4;
    e->center_k = center_k_from_env();
    int rc = e->alloc(reinterpret_cast<void**>(&e->d_err), sizeof(apxb::dev_error));
    if (rc) return rc;
    rc = e->alloc(reinterpret_cast<void**>(&e->d_partials), sizeof(double) * e->vec_grid * 4);
    if (rc) return rc;
    rc = e->alloc(reinterpret_cast<void**>(&e->d_counters), sizeof(unsigned) * 16);
    if (rc) return rc;
    rc = e->alloc(reinterpret_cast<void**>(&e->d_scal), sizeof(double) * 8);
    if (rc) return rc;
    APXB_CK(cudaMallocHost(&e->h_err, sizeof(apxb::dev_error)));
    APXB_CK(cudaMallocHost(&e->h_scal, sizeof(double) * 8));
    APXB_CK(cudaMemsetAsync(e->d_err, 0, sizeof(apxb::dev_error), e->stream));
    APXB_CK(cudaMemsetAsync(e->d_counters, 0, sizeof(unsigned) * 16, e->stream));
    APXB_CK(cudaEventCreate(&e->ev0));
    APXB_CK(cudaEventCreate(&e->ev1));
    APXB_CK(cudaStreamSynchronize(e->stream));
    e->mem_used = 0;   // engine scratch is not charged to the factor/operator budget
    e->pool = apxb::device_pool(device);   // the scratch above stays on cudaMalloc (engine_free frees it)
    apxb::pool_engine_added(device);
    *out = e.release();
    return APXB_OK;
}

}  // extern "C"

namespace {
void engine_free(apxb_engine* e) {
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    cudaFree(e->d_err); cudaFree(e->d_partials); cudaFree(e->d_counters); cudaFree(e->d_scal);
    e->release(e->d_stage_a, e->stage_n * 8);
    e->release(e->d_stage_b, e->stage_n * 8);
    cudaStreamSynchronize(e->stream);
    apxb::pool_engine_removed(e->device);
    if (e->h_err) cudaFreeHost(e->h_err);
    if (e->h_scal) cudaFreeHost(e->h_scal);
    if (e->h_stage_a) cudaFreeHost(e->h_stage_a);
    if (e->h_stage_b) cudaFreeHost(e->h_stage_b);
    cudaEventDestroy(e->ev0); cudaEventDestroy(e->ev1);
    cudaStreamDestroy(e->stream);
    delete e;
}

}  // namespace

void apxb_detail::release_child(apxb_engine* e) {
    if (--e->children == 0 && e->closing) engine_free(e);
}
using apxb_detail::release_child;

namespace apxb {

namespace {
std::mutex g_pool_mu;
std::vector<cudaMemPool_t> g_pools;   // per device
std::vector<int> g_pool_engines;      // engines alive per device
int g_pools_off = -1;
}  // namespace

cudaMemPool_t device_pool(int device) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (g_pools_off < 0) {
        const char* ev = std::getenv("APXB_NO_POOL");
        g_pools_off = ev && *ev && *ev != '0' ? 1 : 0;
    }
    if (g_pools_off || device < 0) return nullptr;
    if (static_cast<int>(g_pools.size()) <= device) {
        g_pools.resize(static_cast<size_t>(device) + 1, nullptr);
        g_pool_engines.resize(static_cast<size_t>(device) + 1, 0);
    }
    if (!g_pools[device]) {
        int supported = 0;
        if (cudaDeviceGetAttribute(&supported, cudaDevAttrMemoryPoolsSupported, device) != cudaSuccess || !supported) {
            cudaGetLastError();
            return nullptr;
        }
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = UINT64_MAX;   // freed memory stays in the pool until the last engine goes
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        g_pools[device] = pool;
    }
    return g_pools[device];
}

void pool_engine_added(int device) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (device >= 0 && device < static_cast<int>(g_pool_engines.size())) ++g_pool_engines[device];
}

void pool_engine_removed(int device) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (device < 0 || device >= static_cast<int>(g_pool_engines.size())) return;
    if (--g_pool_engines[device] == 0 && g_pools[device]) cudaMemPoolTrimTo(g_pools[device], 0);
}

}  // namespace apxb

extern "C" {

int apxb_engine_destroy(apxb_engine* e) {
    if (!e) return APXB_OK;
    if (e->children > 0) {
        e->closing = true;
        return APXB_OK;
    }
    engine_free(e);
    return APXB_OK;
}

int apxb_engine_sync(apxb_engine* e) {
    if (!e) return fail(APXB_ERR_INVALID, "engine is NULL");
    APXB_CK(cudaStreamSynchronize(e->stream));
    return e->take_error();
}

void* apxb_engine_stream(apxb_engine* e) { return e ? static_cast<void*>(e->stream) : nullptr; }

int apxb_engine_set_spin_budget(apxb_engine* e, uint64_t ns) {
    if (!e || ns == 0) return fail(APXB_ERR_INVALID, "bad spin budget");
    e->budget_ns = ns;
    return APXB_OK;
}

int apxb_engine_set_memory_budget(apxb_engine* e, uint64_t bytes) {
    if (!e) return fail(APXB_ERR_INVALID, "engine is NULL");
    e->mem_budget = bytes;
    return APXB_OK;
}

uint64_t apxb_engine_memory_used(apxb_engine* e) { return e ? e->mem_used : 0; }

int apxb_engine_set_sweep_grid(apxb_engine* e, int blocks) {
    if (!e || blocks < 0) return fail(APXB_ERR_INVALID, "bad sweep grid");
    e->sweep_grid = blocks;
    return APXB_OK;
}

int apxb_prepare_host(uint32_t n, const uint32_t* colptr, const uint32_t* rowidx, const float* vals,
                      const uint32_t* perm, int sddm, const uint64_t* rounds, uint32_t n_rounds,
                      double drop_rel, uint32_t* m, uint64_t* nnz_stored, int32_t* levels,
                      uint32_t* csr_ptr, uint32_t* csr_idx, float* csr_val,
                      uint32_t* csc_ptr, uint32_t* csc_idx, float* csc_val,
                      uint8_t* fwd_thin, uint8_t* bck_thin) {
    return guarded([&]() -> int {
        if (!colptr || !rowidx || !vals || !perm || !m || !nnz_stored) return fail(APXB_ERR_INVALID, "NULL argument");
        if (n_rounds && !rounds) return fail(APXB_ERR_INVALID, "rounds is NULL");
        apxb::prepared_factor h;
        const std::string why = apxb::prepare_factor(n, colptr, rowidx, vals, perm, sddm != 0, rounds, n_rounds,
                                                     drop_rel, h);
        if (!why.empty()) return fail(APXB_ERR_BAD_FACTOR, why);
        *m = h.m;
        *nnz_stored = h.nnz_stored;
        if (levels) { levels[0] = h.fwd_levels; levels[1] = h.bck_levels; }
        if (csr_ptr) std::memcpy(csr_ptr, h.csr_ptr.data(), 4 * h.csr_ptr.size());
        if (csr_idx) std::memcpy(csr_idx, h.csr_idx.data(), 4 * h.csr_idx.size());
        if (csr_val) std::memcpy(csr_val, h.csr_val.data(), 4 * h.csr_val.size());
        if (csc_ptr) std::memcpy(csc_ptr, h.csc_ptr.data(), 4 * h.csc_ptr.size());
        if (csc_idx) std::memcpy(csc_idx, h.csc_idx.data(), 4 * h.csc_idx.size());
        if (csc_val) std::memcpy(csc_val, h.csc_val.data(), 4 * h.csc_val.size());
        for (uint32_t r = 0; r < h.m; ++r) {
            if (fwd_thin) fwd_thin[r] = (h.fwd_thin_bits[r >> 5] >> (r & 31)) & 1u;
            if (bck_thin) bck_thin[r] = (h.bck_thin_bits[r >> 5] >> (r & 31)) & 1u;
        }
        return APXB_OK;
    });
}

int apxb_prepare_host_fp16(uint32_t n, const uint32_t* colptr, const uint32_t* rowidx, const float* vals,
                           const uint32_t* perm, int sddm, const uint64_t* rounds, uint32_t n_rounds,
                           double drop_rel, uint32_t* m, uint64_t* nnz_stored,
                           uint32_t* csc_ptr, uint32_t* csc_idx, uint16_t* csc_val16,
                           uint32_t* csr_ptr, uint32_t* csr_idx, uint16_t* csr_val16,
                           float* diag, float* inv_scale, uint64_t* stats) {
    return guarded([&]() -> int {
        if (!colptr || !rowidx || !vals || !perm || !m || !nnz_stored) return fail(APXB_ERR_INVALID, "NULL argument");
        if (n_rounds && !rounds) return fail(APXB_ERR_INVALID, "rounds is NULL");
        apxb::prepared_factor h;
        const std::string why = apxb::prepare_factor(n, colptr, rowidx, vals, perm, sddm != 0, rounds, n_rounds,
                                                     drop_rel, h, true);
        if (!why.empty()) return fail(APXB_ERR_BAD_FACTOR, why);
        *m = h.m;
        *nnz_stored = h.nnz_stored;
        if (csc_ptr) std::memcpy(csc_ptr, h.csc_ptr.data(), 4 * h.csc_ptr.size());
        if (csc_idx) std::memcpy(csc_idx, h.csc_idx.data(), 4 * h.csc_idx.size());
        if (csc_val16) std::memcpy(csc_val16, h.csc_h.data(), 2 * h.csc_h.size());
        if (csr_ptr) std::memcpy(csr_ptr, h.csr_ptr.data(), 4 * h.csr_ptr.size());
        if (csr_idx) std::memcpy(csr_idx, h.csr_idx.data(), 4 * h.csr_idx.size());
        if (csr_val16) std::memcpy(csr_val16, h.csr_h.data(), 2 * h.csr_h.size());
        if (diag) std::memcpy(diag, h.diag16.data(), 4 * h.diag16.size());
        if (inv_scale) std::memcpy(inv_scale, h.inv_scale.data(), 4 * h.inv_scale.size());
        if (stats) { stats[0] = h.dropped; stats[1] = h.dropped_flush; stats[2] = h.flushed; }
        return APXB_OK;
    });
}

// ---------------------------------------------------------------- factor

int apxb_factor_create(apxb_engine* e, uint32_t n, const uint32_t* colptr, const uint32_t* rowidx,
                       const float* vals, const uint32_t* perm, int sddm, const uint64_t* rounds,
                       uint32_t n_rounds, double drop_rel, int precision, apxb_factor** out) {
    return guarded([&]() -> int {
        if (!e || !out || !colptr || !rowidx || !vals || !perm) return fail(APXB_ERR_INVALID, "NULL argument");
        if (precision != APXB_PREC_FP64 && precision != APXB_PREC_FP32 && precision != APXB_PREC_FP16)
            return fail(APXB_ERR_INVALID, "bad precision");
        if (n_rounds && !rounds) return fail(APXB_ERR_INVALID, "rounds is NULL");
        *out = nullptr;
        const bool fp16 = precision == APXB_PREC_FP16;
        APXB_CK(cudaSetDevice(e->device));
        std::unique_ptr<apxb_factor> f(new (std::nothrow) apxb_factor);
        if (!f) return fail(APXB_ERR_INVALID, "host allocation failed");
        f->e = e;
        f->precision = precision;
        f->drop_rel = drop_rel < 0.0 ? apxb::kDropRelDefault : drop_rel;
        // Factors with round sizes and fp32 / fp64 storage are prepared by kernels
        // (devprep.cu); the others on the host. Both give the same arrays.
        const bool on_device = apxb::device_prep_applies(fp16, n_rounds);
        if (on_device) {
            int arc = 0;
            const std::string why = apxb::prepare_factor_device(f.get(), n, colptr, rowidx, vals, perm, sddm != 0,
                                                                rounds, n_rounds, drop_rel, &arc);
            if (arc) return arc;
            if (!why.empty()) return fail(APXB_ERR_BAD_FACTOR, why);
        } else {
            const std::string why = apxb::prepare_factor(n, colptr, rowidx, vals, perm, sddm != 0, rounds, n_rounds,
                                                         drop_rel, f->h, fp16);
            if (!why.empty()) return fail(APXB_ERR_BAD_FACTOR, why);
        }
        const auto& h = f->h;
        const size_t m = h.m, nnz = h.nnz_stored;
        if (nnz >= 0xffffffffull) return fail(APXB_ERR_BAD_FACTOR, "factor nnz exceeds the 32-bit offset range");
        // fp16 storage: (1 / s)^2 in fp64 (an fp32 square overflows for s below
        // ~5e-20), and a column the storage cannot represent fails here, loudly
        // (cuda.h:339-358)
        std::vector<double> inv_scale2;
        if (fp16) {
            inv_scale2.resize(m);
            for (size_t j = 0; j < m; ++j) {
                const double r = static_cast<double>(h.inv_scale[j]);
                inv_scale2[j] = r * r;
                if (!(std::isfinite(h.diag16[j]) && h.diag16[j] != 0.0f && std::isfinite(inv_scale2[j])))
                    return fail(APXB_ERR_BAD_FACTOR, "fp16 factor storage cannot represent column " + std::to_string(j) +
                                                         " (diag " + std::to_string(h.diag16[j]) + ", inv_scale^2 " +
                                                         std::to_string(inv_scale2[j]) + ")");
            }
        }
        int rc;
        cudaStream_t s = e->stream;
        if ((rc = f->dalloc(&f->ctl, 2))) return rc;
        APXB_CK(cudaMemsetAsync(f->ctl, 0, sizeof(apxb::sweep_ctl) * 2, s));
        if (!on_device) {
            if ((rc = f->dalloc(&f->perm, n))) return rc;
            APXB_CK(cudaMemcpyAsync(f->perm, h.perm.data(), 4 * static_cast<size_t>(n), cudaMemcpyHostToDevice, s));
        }
        for (int dir = 0; dir < 2 && !on_device; ++dir) {
            const apxb::sweep_plan& pl = dir == 0 ? h.fwd_plan : h.bck_plan;
            if ((rc = f->dalloc(&f->info[dir], pl.info.size())) || (rc = f->dalloc(&f->ord[dir], pl.ord.size())) ||
                (rc = f->dalloc(&f->ptr[dir], pl.ptr.size())) || (rc = f->dalloc(&f->idx[dir], pl.idx.size())) ||
                (rc = fp16 ? f->dalloc(&f->val16[dir], pl.val16.size()) : f->dalloc(&f->val[dir], pl.val.size())) ||
                (rc = f->dalloc(&f->chunk[dir], pl.chunk.size())))
                return rc;
            f->n_chunks[dir] = static_cast<uint32_t>(pl.chunk.size() - 1);
            APXB_CK(cudaMemcpyAsync(f->chunk[dir], pl.chunk.data(), 4 * pl.chunk.size(), cudaMemcpyHostToDevice, s));
            APXB_CK(cudaMemcpyAsync(f->info[dir], pl.info.data(), 4 * pl.info.size(), cudaMemcpyHostToDevice, s));
            APXB_CK(cudaMemcpyAsync(f->ord[dir], pl.ord.data(), 4 * pl.ord.size(), cudaMemcpyHostToDevice, s));
            APXB_CK(cudaMemcpyAsync(f->ptr[dir], pl.ptr.data(), 4 * pl.ptr.size(), cudaMemcpyHostToDevice, s));
            APXB_CK(cudaMemcpyAsync(f->idx[dir], pl.idx.data(), 4 * pl.idx.size(), cudaMemcpyHostToDevice, s));
            if (fp16)
                APXB_CK(cudaMemcpyAsync(f->val16[dir], pl.val16.data(), 2 * pl.val16.size(), cudaMemcpyHostToDevice, s));
            else
                APXB_CK(cudaMemcpyAsync(f->val[dir], pl.val.data(), 4 * pl.val.size(), cudaMemcpyHostToDevice, s));
            if (pl.seg_rows) {
                if ((rc = f->dalloc(&f->seg_row[dir], pl.seg_row.size())) ||
                    (rc = f->dalloc(&f->seg_lvl[dir], pl.seg_lvl.size())) ||
                    (rc = f->dalloc(&f->seg_ptr[dir], pl.seg_ptr.size())) ||
                    (rc = f->dalloc(&f->seg_idx[dir], pl.seg_idx.size())) ||
                    (rc = f->dalloc(&f->seg_val[dir], pl.seg_val.size())))
                    return rc;
                APXB_CK(cudaMemcpyAsync(f->seg_row[dir], pl.seg_row.data(), 4 * pl.seg_row.size(), cudaMemcpyHostToDevice, s));
                APXB_CK(cudaMemcpyAsync(f->seg_lvl[dir], pl.seg_lvl.data(), 4 * pl.seg_lvl.size(), cudaMemcpyHostToDevice, s));
                APXB_CK(cudaMemcpyAsync(f->seg_ptr[dir], pl.seg_ptr.data(), 4 * pl.seg_ptr.size(), cudaMemcpyHostToDevice, s));
                APXB_CK(cudaMemcpyAsync(f->seg_idx[dir], pl.seg_idx.data(), 4 * pl.seg_idx.size(), cudaMemcpyHostToDevice, s));
                APXB_CK(cudaMemcpyAsync(f->seg_val[dir], pl.seg_val.data(), 4 * pl.seg_val.size(), cudaMemcpyHostToDevice, s));
            }
        }
        if (fp16) {
            if ((rc = f->dalloc(&f->diag16, m)) || (rc = f->dalloc(&f->inv_scale2, m))) return rc;
            APXB_CK(cudaMemcpyAsync(f->diag16, h.diag16.data(), 4 * m, cudaMemcpyHostToDevice, s));
            APXB_CK(cudaMemcpyAsync(f->inv_scale2, inv_scale2.data(), 8 * m, cudaMemcpyHostToDevice, s));
        }
        if ((rc = f->dalloc(&f->Y, n)) || (rc = f->dalloc(&f->Z, n)) || (rc = f->dalloc(&f->zp, n))) return rc;
        // Z[m] (the grounded entry of a Laplacian) is 0 for good; rows < m start armed.
        APXB_CK(cudaMemsetAsync(f->Z, 0, 8 * static_cast<size_t>(n), s));
        apxb::launch_fill_sent64(f->Y, m, s);
        apxb::launch_fill_sent64(f->Z, m, s);
        f->y_armed = f->z_armed = true;
        APXB_CK(cudaGetLastError());
        f->grid64 = apxb::sweep_grid64(e->num_sms);
        APXB_CK(cudaStreamSynchronize(s));
        e->children++;
        *out = f.release();
        return APXB_OK;
    });
}

int apxb_factor_destroy(apxb_factor* f) {
    if (!f) return APXB_OK;
    apxb_engine* e = f->e;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    delete f;
    release_child(e);
    return APXB_OK;
}

int apxb_factor_info_get(const apxb_factor* f, apxb_factor_info* info) {
    if (!f || !info) return fail(APXB_ERR_INVALID, "NULL argument");
    info->n = f->h.n; info->m = f->h.m;
    info->nnz_factor = f->h.nnz_factor; info->nnz_stored = f->h.nnz_stored; info->dropped = f->h.dropped;
    info->fwd_levels = f->h.fwd_levels; info->bck_levels = f->h.bck_levels;
    info->precision = f->precision; info->sddm = f->h.sddm ? 1 : 0;
    info->device_bytes = f->dev_bytes; info->apply_count = f->apply_count;
    info->drop_rel = f->drop_rel;
    info->dropped_flush = f->h.dropped_flush;
    info->sweep_grid = f->e->sweep_grid > 0 ? f->e->sweep_grid
                     : f->precision == APXB_PREC_FP64 ? f->grid64 : apxb::sweep_grid32(1, f->e->num_sms);
    info->reserved = 0;
    return APXB_OK;
}

int apxb_factor_arrays(const apxb_factor* f, uint32_t* csr_ptr, uint32_t* csr_idx, float* csr_val,
                       uint32_t* csc_ptr, uint32_t* csc_idx, float* csc_val, uint8_t* fwd_thin,
                       uint8_t* bck_thin) {
    if (!f) return fail(APXB_ERR_INVALID, "factor is NULL");
    if (!f->host_arrays) {   // prepared on the device: the host copies on first request
        const std::string why = apxb::factor_host_arrays(const_cast<apxb_factor*>(f));
        if (!why.empty()) return fail(APXB_ERR_CUDA, why);
    }
    const auto& h = f->h;
    if (csr_ptr) std::memcpy(csr_ptr, h.csr_ptr.data(), 4 * h.csr_ptr.size());
    if (csr_idx) std::memcpy(csr_idx, h.csr_idx.data(), 4 * h.csr_idx.size());
    if (csr_val) std::memcpy(csr_val, h.csr_val.data(), 4 * h.csr_val.size());
    if (csc_ptr) std::memcpy(csc_ptr, h.csc_ptr.data(), 4 * h.csc_ptr.size());
    if (csc_idx) std::memcpy(csc_idx, h.csc_idx.data(), 4 * h.csc_idx.size());
    if (csc_val) std::memcpy(csc_val, h.csc_val.data(), 4 * h.csc_val.size());
    for (uint32_t r = 0; r < h.m; ++r) {
        if (fwd_thin) fwd_thin[r] = (h.fwd_thin_bits[r >> 5] >> (r & 31)) & 1u;
        if (bck_thin) bck_thin[r] = (h.bck_thin_bits[r >> 5] >> (r & 31)) & 1u;
    }
    return APXB_OK;
}

int apxb_factor_reset_apply_count(apxb_factor* f) {
    if (!f) return fail(APXB_ERR_INVALID, "factor is NULL");
    f->apply_count = 0;
    return APXB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- sweeps (internal)

namespace {

int grid64_of(const apxb_factor* f) { return f->e->sweep_grid > 0 ? f->e->sweep_grid : f->grid64; }

apxb::sweep_args<double> sweep64_args(apxb_factor* f, int dir) {
    apxb::sweep_args<double> a{};
    plan_args(f, dir, a);
    a.ctl = f->ctl + dir;
    a.err = f->e->d_err;
    a.budget_ns = f->e->budget_ns;
    a.k = 1;
    return a;
}

// Forward: in -> Y (re-arms Z). Backward: in -> Z (re-arms Y).
int run_sweep64(apxb_factor* f, int dir, const double* in, double* copy_out, const double* rhs_sub,
                const int* skip) {
    cudaStream_t s = f->e->stream;
    double* out = dir == 0 ? f->Y : f->Z;
    bool& armed = dir == 0 ? f->y_armed : f->z_armed;
    bool& other = dir == 0 ? f->z_armed : f->y_armed;
    if (!armed) apxb::launch_fill_sent64(out, f->h.m, s);
    apxb::sweep_args<double> a = sweep64_args(f, dir);
    a.in = in;
    a.out = out;
    a.reset = dir == 0 ? f->Z : f->Y;
    a.copy_out = copy_out;
    a.rhs_sub = rhs_sub;
    a.skip = skip;
    apxb::launch_sweep64(dir, a, grid64_of(f), s);
    armed = false;
    other = true;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(APXB_ERR_CUDA, std::string("sweep launch: ") + cudaGetErrorString(e));
    return APXB_OK;
}

// After a failed call the tracked buffers are in an unknown state.
void disarm(apxb_factor* f) {
    f->y_armed = f->z_armed = false;
    f->yf_armed = f->zf_armed = false;
    cudaMemsetAsync(f->ctl, 0, sizeof(apxb::sweep_ctl) * 2, f->e->stream);
    cudaMemsetAsync(f->e->d_counters, 0, sizeof(unsigned) * 16, f->e->stream);
}

int finish(apxb_factor* f) {
    const int rc = f->e->take_error();
    if (rc) disarm(f);
    return rc;
}

int sweep32_one(apxb_factor* f, int dir, const double* d_in, double* d_out);

}  // namespace

extern "C" {

int apxb_sweep(apxb_engine* e, apxb_factor* f, int dir, const double* d_in, double* d_out) {
    if (!e || !f || !d_in || !d_out || (dir != 0 && dir != 1)) return fail(APXB_ERR_INVALID, "bad argument");
    if (f->e != e) return fail(APXB_ERR_INVALID, "factor belongs to another engine");
    APXB_CK(cudaSetDevice(e->device));
    int rc = f->precision == APXB_PREC_FP64 ? run_sweep64(f, dir, d_in, d_out, nullptr, nullptr)
                                            : sweep32_one(f, dir, d_in, d_out);
    if (rc) return rc;
    return finish(f);
}

}  // extern "C"

namespace {

int pair_fp64(apxb_factor* f, const double* d_in, double* d_out) {
    int rc = run_sweep64(f, 0, d_in, nullptr, nullptr, nullptr);
    if (rc) return rc;
    return run_sweep64(f, 1, f->Y, d_out, nullptr, nullptr);
}

int ensure_f32(apxb_factor* f, int k) {
    const size_t need = static_cast<size_t>(f->h.n) * k;
    if (f->f32_cap < need) {
        for (auto it = f->owned.begin(); it != f->owned.end();) {
            if (it->first == f->Yf || it->first == f->Zf) {
                f->e->release(it->first, it->second);
                f->dev_bytes -= it->second;
                it = f->owned.erase(it);
            } else {
                ++it;
            }
        }
        f->Yf = f->Zf = nullptr;
        f->f32_cap = 0;
        int rc;
        if ((rc = f->dalloc(&f->Yf, need)) || (rc = f->dalloc(&f->Zf, need))) return rc;
        f->f32_cap = need;
        f->yf_armed = f->zf_armed = false;
        f->f32_k = 0;
    }
    if (f->f32_k != k) {
        f->yf_armed = f->zf_armed = false;
        APXB_CK(cudaMemsetAsync(f->Zf, 0, sizeof(float) * need, f->e->stream));
        f->f32_k = k;
    }
    return APXB_OK;
}

}  // namespace

namespace apxb {
void launch_cast32to64(const float* in, double* out, size_t n, cudaStream_t s);
void launch_cast64to32(const double* in, float* out, size_t n, cudaStream_t s);
}

namespace {

int pair_fp32(apxb_factor* f, int k, const double* d_in, double* d_out) {
    int rc = ensure_f32(f, k);
    if (rc) return rc;
    cudaStream_t s = f->e->stream;
    const size_t mk = static_cast<size_t>(f->h.m) * k;
    if (!f->yf_armed) apxb::launch_fill_sent32(f->Yf, mk, s);
    if (!f->zf_armed) apxb::launch_fill_sent32(f->Zf, mk, s);
    const int grid = f->e->sweep_grid > 0 ? f->e->sweep_grid : apxb::sweep_grid32(k, f->e->num_sms);
    apxb::sweep_args<float> a{};
    a.k = k;
    a.err = f->e->d_err; a.budget_ns = f->e->budget_ns;
    plan_args(f, 0, a);
    a.ctl = f->ctl;
    a.out = f->Yf; a.reset = f->Zf;
    apxb::launch_sweep32_from64(0, a, d_in, grid, s);
    plan_args(f, 1, a);
    a.ctl = f->ctl + 1;
    a.in = f->Yf; a.out = f->Zf; a.reset = f->Yf;
    a.in_scale2 = f->inv_scale2;   // fp16 factors: the backward reads D^-2 y'
    apxb::launch_sweep32(1, a, grid, s);
    f->yf_armed = true;
    f->zf_armed = false;
    apxb::launch_cast32to64(f->Zf, d_out, mk, s);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(APXB_ERR_CUDA, std::string("sweep launch: ") + cudaGetErrorString(e));
    return APXB_OK;
}

// One fp32 sweep of an fp32 / fp16 factor, fp64 in and out (m entries).
// Forward: in -> Yf (re-arms Zf). Backward: in is narrowed into Yf, which the
// sweep reads as its right-hand side (fp16: times inv_scale^2) and re-arms
// row by row; -> Zf.
int sweep32_one(apxb_factor* f, int dir, const double* d_in, double* d_out) {
    int rc = ensure_f32(f, 1);
    if (rc) return rc;
    cudaStream_t s = f->e->stream;
    const size_t m = f->h.m;
    const int grid = f->e->sweep_grid > 0 ? f->e->sweep_grid : apxb::sweep_grid32(1, f->e->num_sms);
    apxb::sweep_args<float> a{};
    a.k = 1;
    a.err = f->e->d_err; a.budget_ns = f->e->budget_ns;
    plan_args(f, dir, a);
    a.ctl = f->ctl + dir;
    if (dir == 0) {
        if (!f->yf_armed) apxb::launch_fill_sent32(f->Yf, m, s);
        a.out = f->Yf; a.reset = f->Zf;
        apxb::launch_sweep32_from64(0, a, d_in, grid, s);
        f->yf_armed = false;
        f->zf_armed = true;
        apxb::launch_cast32to64(f->Yf, d_out, m, s);
    } else {
        if (!f->zf_armed) apxb::launch_fill_sent32(f->Zf, m, s);
        apxb::launch_cast64to32(d_in, f->Yf, m, s);
        a.in = f->Yf; a.out = f->Zf; a.reset = f->Yf;
        a.in_scale2 = f->inv_scale2;
        apxb::launch_sweep32(1, a, grid, s);
        f->zf_armed = false;
        f->yf_armed = true;
        apxb::launch_cast32to64(f->Zf, d_out, m, s);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(APXB_ERR_CUDA, std::string("sweep launch: ") + cudaGetErrorString(e));
    return APXB_OK;
}

}  // namespace

extern "C" {

int apxb_sweep_pair(apxb_engine* e, apxb_factor* f, const double* d_in, double* d_out) {
    if (!e || !f || !d_in || !d_out) return fail(APXB_ERR_INVALID, "bad argument");
    if (f->e != e) return fail(APXB_ERR_INVALID, "factor belongs to another engine");
    APXB_CK(cudaSetDevice(e->device));
    const int rc = f->precision == APXB_PREC_FP64 ? pair_fp64(f, d_in, d_out) : pair_fp32(f, 1, d_in, d_out);
    if (rc) return rc;
    return finish(f);
}

int apxb_sweep_pair_multi(apxb_engine* e, apxb_factor* f, int k, const double* d_in, double* d_out) {
    if (!e || !f || !d_in || !d_out) return fail(APXB_ERR_INVALID, "bad argument");
    if (f->e != e) return fail(APXB_ERR_INVALID, "factor belongs to another engine");
    if (k != 1 && k != 2 && k != 4 && k != 8 && k != 16) return fail(APXB_ERR_INVALID, "k must be 1, 2, 4, 8 or 16");
    APXB_CK(cudaSetDevice(e->device));
    const int rc = pair_fp32(f, k, d_in, d_out);
    if (rc) return rc;
    return finish(f);
}

int apxb_sweep_pair_host(apxb_engine* e, apxb_factor* f, const double* in, double* out) {
    if (!e || !f || !in || !out) return fail(APXB_ERR_INVALID, "bad argument");
    if (f->e != e) return fail(APXB_ERR_INVALID, "factor belongs to another engine");
    APXB_CK(cudaSetDevice(e->device));
    const size_t m = f->h.m;
    int rc = e->ensure_stage(f->h.n);
    if (rc) return rc;
    std::memcpy(e->h_stage_a, in, 8 * m);
    APXB_CK(cudaMemcpyAsync(e->d_stage_a, e->h_stage_a, 8 * m, cudaMemcpyHostToDevice, e->stream));
    rc = f->precision == APXB_PREC_FP64 ? pair_fp64(f, e->d_stage_a, e->d_stage_b)
                                        : pair_fp32(f, 1, e->d_stage_a, e->d_stage_b);
    if (rc) return rc;
    APXB_CK(cudaMemcpyAsync(e->h_stage_b, e->d_stage_b, 8 * m, cudaMemcpyDeviceToHost, e->stream));
    rc = finish(f);
    if (rc) return rc;
    std::memcpy(out, e->h_stage_b, 8 * m);
    return APXB_OK;
}

// ---------------------------------------------------------------- apply (original ordering)

int apxb_apply(apxb_engine* e, apxb_factor* f, const double* b, double* z, int flags, double* rz_out) {
    if (!e || !f || !b || !z) return fail(APXB_ERR_INVALID, "bad argument");
    if (f->e != e) return fail(APXB_ERR_INVALID, "factor belongs to another engine");
    APXB_CK(cudaSetDevice(e->device));
    const uint32_t n = f->h.n;
    const bool dev = flags & APXB_DEVICE_PTRS;
    bool center = false;
    if (!f->h.sddm) {
        if (flags & APXB_CENTER_ALWAYS) center = true;
        else if (flags & APXB_CENTER_NEVER) center = false;
        else center = (++f->apply_count % static_cast<uint64_t>(e->center_k)) == 0;
    }
    int rc = 0;
    const double* db = b;
    double* dz = z;
    if (!dev) {
        if ((rc = e->ensure_stage(n))) return rc;
        std::memcpy(e->h_stage_a, b, 8 * static_cast<size_t>(n));
        APXB_CK(cudaMemcpyAsync(e->d_stage_a, e->h_stage_a, 8 * static_cast<size_t>(n), cudaMemcpyHostToDevice,
                                e->stream));
        db = e->d_stage_a;
        dz = e->d_stage_b;
    }
    apxb::apply_ptrs a{};
    a.perm = f->perm; a.b = db; a.zp = f->zp; a.z = dz; a.scal = e->d_scal;
    a.center = center ? 1 : 0; a.partials = e->d_partials; a.counters = e->d_counters; a.n = n;
    a.grid = e->vec_grid;
    cudaStream_t s = e->stream;
    apxb::launch_apply_bsum(a, s);
    apxb::launch_apply_permute(a, s);
    if (f->precision == APXB_PREC_FP64) {
        if ((rc = pair_fp64(f, f->zp, nullptr))) return rc;
        a.zsol = f->Z;
    } else {
        // fp32 sweeps write Zf; widen into zp (rows < m), zp[m] = 0 for a Laplacian.
        if ((rc = pair_fp32(f, 1, f->zp, f->zp))) return rc;
        if (!f->h.sddm) APXB_CK(cudaMemsetAsync(f->zp + f->h.m, 0, 8, s));
        a.zsol = f->zp;
    }
    apxb::launch_apply_zsum(a, s);
    apxb::launch_apply_gather(a, s);
    APXB_CK(cudaGetLastError());
    if (rz_out) APXB_CK(cudaMemcpyAsync(e->h_scal, e->d_scal, sizeof(double) * 4, cudaMemcpyDeviceToHost, s));
    if (!dev) APXB_CK(cudaMemcpyAsync(e->h_stage_b, dz, 8 * static_cast<size_t>(n), cudaMemcpyDeviceToHost, s));
    if ((rc = finish(f))) return rc;
    if (rz_out) *rz_out = e->h_scal[2];
    if (!dev) std::memcpy(z, e->h_stage_b, 8 * static_cast<size_t>(n));
    return APXB_OK;
}

// ---------------------------------------------------------------- operator

int apxb_operator_create(apxb_engine* e, uint32_t n, const int32_t* colptr, const int32_t* rowidx,
                         const double* vals, const uint32_t* perm, apxb_operator** out) {
    return guarded([&]() -> int {
        if (!e || !colptr || !rowidx || !vals || !perm || !out || n == 0) return fail(APXB_ERR_INVALID, "bad argument");
        *out = nullptr;
        APXB_CK(cudaSetDevice(e->device));
        std::unique_ptr<apxb_operator> a(new (std::nothrow) apxb_operator);
        if (!a) return fail(APXB_ERR_INVALID, "host allocation failed");
        a->e = e;
        a->n = n;
        std::vector<int32_t> ptr;
        cudaStream_t s = e->stream;
        int rc;
        const char* hp = std::getenv("APXB_HOST_PREP");
        if (hp && *hp && *hp != '0') {   // P A P^T on the host threads
            apxb::plan_vec<int32_t> idx;
            apxb::plan_vec<double> val;
            const std::string why = apxb::permute_operator(n, colptr, rowidx, vals, perm, ptr, idx, val);
            if (!why.empty()) return fail(APXB_ERR_INVALID, why);
            a->nnz = idx.size();
            if ((rc = a->dalloc(&a->ptr, n + 1)) || (rc = a->dalloc(&a->idx, a->nnz)) || (rc = a->dalloc(&a->val, a->nnz)))
                return rc;
            APXB_CK(cudaMemcpyAsync(a->ptr, ptr.data(), 4 * (static_cast<size_t>(n) + 1), cudaMemcpyHostToDevice, s));
            APXB_CK(cudaMemcpyAsync(a->idx, idx.data(), 4 * a->nnz, cudaMemcpyHostToDevice, s));
            APXB_CK(cudaMemcpyAsync(a->val, val.data(), 8 * a->nnz, cudaMemcpyHostToDevice, s));
            APXB_CK(cudaStreamSynchronize(s));   // the host arrays go out of scope
        } else {                          // P A P^T by kernels (devprep.cu): the same arrays
            int arc = 0;
            const std::string why = apxb::permute_operator_device(a.get(), n, colptr, rowidx, vals, perm, ptr, &arc);
            if (arc) return arc;
            if (!why.empty()) return fail(APXB_ERR_INVALID, why);
        }
        {   // storage precision: fp32 iff every value is fp32-exact; APXCHOL_GPU_FP32_OPERATOR overrides
            // ("0": fp64, any other value: fp32), the reference's rule (pcg_cuda.h:100-111)
            const char* ev = std::getenv("APXCHOL_GPU_FP32_OPERATOR");
            const int want = ev && std::string(ev) == "0" ? 0 : (ev && *ev ? 1 : -1);
            int arc = 0;
            const std::string why = apxb::operator_precision_device(a.get(), want, &arc);
            if (arc) return arc;
            if (!why.empty()) return fail(APXB_ERR_CUDA, why);
        }
        if ((rc = a->dalloc(&a->perm, n)) || (rc = a->dalloc(&a->x, n)) || (rc = a->dalloc(&a->r, n)) ||
            (rc = a->dalloc(&a->p, n)) || (rc = a->dalloc(&a->Ap, n)) || (rc = a->dalloc(&a->b_orig, n)) ||
            (rc = a->dalloc(&a->x_orig, n)) || (rc = a->dalloc(&a->st, 1)))
            return rc;
        APXB_CK(cudaMallocHost(&a->h_st, sizeof(apxb::pcg_state)));
        APXB_CK(cudaMemcpyAsync(a->perm, perm, 4 * static_cast<size_t>(n), cudaMemcpyHostToDevice, s));
        {   // long rows: cut into chunks summed by one block each (power-law hubs)
            std::vector<uint32_t> lrow, lfirst, clo, chi;
            for (uint32_t r = 0; r < n; ++r) {
                const uint32_t b0 = static_cast<uint32_t>(ptr[r]), e0 = static_cast<uint32_t>(ptr[r + 1]);
                if (e0 - b0 <= apxb::kLongRowPlain) continue;
                lrow.push_back(r);
                lfirst.push_back(static_cast<uint32_t>(clo.size()));
                for (uint32_t q = b0; q < e0; q += apxb::kChunkNnzPlain) {
                    clo.push_back(q);
                    chi.push_back(std::min(e0, q + apxb::kChunkNnzPlain));
                }
            }
            if (!lrow.empty()) {
                lfirst.push_back(static_cast<uint32_t>(clo.size()));
                a->n_long = static_cast<uint32_t>(lrow.size());
                a->n_chunks = static_cast<uint32_t>(clo.size());
                if ((rc = a->dalloc(&a->lr_row, lrow.size())) || (rc = a->dalloc(&a->lr_first, lfirst.size())) ||
                    (rc = a->dalloc(&a->ch_lo, clo.size())) || (rc = a->dalloc(&a->ch_hi, chi.size())) ||
                    (rc = a->dalloc(&a->ch_part, clo.size())))
                    return rc;
                APXB_CK(cudaMemcpyAsync(a->lr_row, lrow.data(), 4 * lrow.size(), cudaMemcpyHostToDevice, s));
                APXB_CK(cudaMemcpyAsync(a->lr_first, lfirst.data(), 4 * lfirst.size(), cudaMemcpyHostToDevice, s));
                APXB_CK(cudaMemcpyAsync(a->ch_lo, clo.data(), 4 * clo.size(), cudaMemcpyHostToDevice, s));
                APXB_CK(cudaMemcpyAsync(a->ch_hi, chi.data(), 4 * chi.size(), cudaMemcpyHostToDevice, s));
            }
        }
        APXB_CK(cudaStreamSynchronize(s));
        e->children++;
        *out = a.release();
        return APXB_OK;
    });
}

int apxb_operator_destroy(apxb_operator* a) {
    if (!a) return APXB_OK;
    apxb_engine* e = a->e;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    delete a;
    release_child(e);
    return APXB_OK;
}

int apxb_operator_fp32(const apxb_operator* a, int* fp32) {
    if (!a || !fp32) return fail(APXB_ERR_INVALID, "bad argument");
    *fp32 = a->valf != nullptr ? 1 : 0;
    return APXB_OK;
}

}  // extern "C"

namespace apxb {
void launch_perm_in(const uint32_t* perm, const double* src, double* dst, unsigned n, int grid, cudaStream_t s);
void launch_perm_out(const uint32_t* perm, const double* src, double* dst, unsigned n, int grid, cudaStream_t s);
void launch_resid(const uint32_t* perm, const double* b_orig, const double* y_perm, double* scal, double* partials,
                  unsigned* counter, unsigned n, int grid, cudaStream_t s);
}

extern "C" {

int apxb_operator_matvec(apxb_engine* e, apxb_operator* a, const double* x, double* y) {
    if (!e || !a || !x || !y) return fail(APXB_ERR_INVALID, "bad argument");
    APXB_CK(cudaSetDevice(e->device));
    const size_t n = a->n;
    int rc = e->ensure_stage(n);
    if (rc) return rc;
    cudaStream_t s = e->stream;
    std::memcpy(e->h_stage_a, x, 8 * n);
    APXB_CK(cudaMemcpyAsync(e->d_stage_a, e->h_stage_a, 8 * n, cudaMemcpyHostToDevice, s));
    apxb::launch_perm_in(a->perm, e->d_stage_a, a->Ap, a->n, e->vec_grid, s);
    apxb::launch_spmv_plain(a->ptr, a->idx, a->val, a->valf, a->Ap, a->r, a->n, e->vec_grid, s);
    apxb::launch_perm_out(a->perm, a->r, e->d_stage_b, a->n, e->vec_grid, s);
    APXB_CK(cudaMemcpyAsync(e->h_stage_b, e->d_stage_b, 8 * n, cudaMemcpyDeviceToHost, s));
    APXB_CK(cudaStreamSynchronize(s));
    std::memcpy(y, e->h_stage_b, 8 * n);
    return e->take_error();
}

}  // extern "C"

// ---------------------------------------------------------------- PCG

namespace {

apxb::pcg_ptrs pcg_ptrs_of(apxb_operator* a, apxb_factor* f) {
    apxb::pcg_ptrs p{};
    p.a_ptr = a->ptr; p.a_idx = a->idx; p.a_val = a->val; p.a_valf = a->valf; p.perm = a->perm;
    p.x = a->x; p.r = a->r; p.p = a->p; p.Ap = a->Ap; p.z = f->Z;
    p.b_orig = a->b_orig; p.x_orig = a->x_orig;
    p.st = a->st; p.err = a->e->d_err; p.partials = a->e->d_partials; p.counters = a->e->d_counters;
    p.n = a->n; p.grid = a->e->vec_grid;
    // lanes per SpMV row from the average row length: a thread per row keeps a
    // short row's gathers in flight together; long rows share lanes
    const double avg = a->n ? static_cast<double>(a->nnz) / a->n : 0.0;
    p.spmv_lanes = avg <= 16.0 ? 1 : (avg <= 64.0 ? 8 : 32);
    p.lr_row = a->lr_row; p.lr_first = a->lr_first; p.ch_lo = a->ch_lo; p.ch_hi = a->ch_hi;
    p.n_long = a->n_long; p.n_chunks = a->n_chunks; p.ch_part = a->ch_part;
    return p;
}

// One preconditioner application inside the loop: fwd + bck sweeps, centring
// shift, r.z / beta, p update. `skip` makes every launch a no-op after `done`.
int enqueue_apply(apxb_operator* a, apxb_factor* f, const apxb::pcg_ptrs& p, unsigned long long handle,
                  int use_cond) {
    cudaStream_t s = a->e->stream;
    const int* skip = &a->st->done;
    // The sweeps read mean_in as the rhs shift (0 on non-centring applications).
    const double* mean_in = &a->st->mean_in;
    {
        apxb::sweep_args<double> fa = sweep64_args(f, 0);
        fa.in = a->r; fa.out = f->Y; fa.reset = f->Z; fa.rhs_sub = mean_in; fa.skip = skip;
        apxb::launch_sweep64(0, fa, grid64_of(f), s);
        apxb::sweep_args<double> ba = sweep64_args(f, 1);
        ba.in = f->Y; ba.out = f->Z; ba.reset = f->Y; ba.skip = skip;
        apxb::launch_sweep64(1, ba, grid64_of(f), s);
    }
    apxb::launch_pcg_zsum(p, s);
    apxb::launch_pcg_rz(p, s);
    apxb::launch_pcg_update_p(p, s, handle, use_cond);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(APXB_ERR_CUDA, std::string("pcg launch: ") + cudaGetErrorString(e));
    return APXB_OK;
}

int enqueue_iteration(apxb_operator* a, apxb_factor* f, const apxb::pcg_ptrs& p, unsigned long long handle,
                      int use_cond) {
    apxb::launch_pcg_spmv(p, a->e->stream);
    apxb::launch_pcg_update_xr(p, a->e->stream);
    return enqueue_apply(a, f, p, handle, use_cond);
}

// APXB_NO_GRAPH=1: no conditional graph (the loop falls back to one-iteration
// graphs launched by the host), so a profiler sees every kernel.
bool conditional_graph_off() {
    const char* v = std::getenv("APXB_NO_GRAPH");
    return v && *v && *v != '0';
}

// Graph of the whole iteration loop: a conditional WHILE node whose body is one
// iteration; the body's last kernel clears the condition once `done` is set.
int build_loop_graph(apxb_operator* a, apxb_factor* f) {
    if (a->loop) {
        cudaGraphExecDestroy(a->loop);
        a->loop = nullptr;
    }
    cudaStream_t s = a->e->stream;
    const apxb::pcg_ptrs p = pcg_ptrs_of(a, f);
    cudaGraph_t g = nullptr;
    APXB_CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    cudaError_t err = conditional_graph_off() ? cudaErrorNotSupported
                                              : cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    if (err == cudaSuccess) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        err = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
        if (err == cudaSuccess) {
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            err = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
            if (err == cudaSuccess) {
                const int rc = enqueue_iteration(a, f, p, static_cast<unsigned long long>(h), 1);
                cudaGraph_t captured = nullptr;
                err = cudaStreamEndCapture(s, &captured);
                if (rc) { cudaGraphDestroy(g); return rc; }
            }
        }
        if (err == cudaSuccess) err = cudaGraphInstantiate(&a->loop, g, 0);
    }
    cudaGraphDestroy(g);
    if (err == cudaSuccess) {
        a->loop_conditional = true;
        a->graph_factor = f;
        return APXB_OK;
    }
    cudaGetLastError();
    // Fallback: a plain graph of one iteration, launched repeatedly by the host.
    a->loop = nullptr;
    APXB_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_iteration(a, f, p, 0, 0);
    cudaGraph_t one = nullptr;
    APXB_CK(cudaStreamEndCapture(s, &one));
    if (rc) { cudaGraphDestroy(one); return rc; }
    APXB_CK(cudaGraphInstantiate(&a->loop, one, 0));
    cudaGraphDestroy(one);
    a->loop_conditional = false;
    a->graph_factor = f;
    return APXB_OK;
}

}  // namespace

extern "C" {

int apxb_pcg(apxb_engine* e, apxb_factor* f, apxb_operator* a, const double* b, double* x, double tol,
             int max_iter, int flags, int want_true_residual, apxb_pcg_result* res) {
    if (!e || !f || !a || !b || !x || !res) return fail(APXB_ERR_INVALID, "bad argument");
    if (f->e != e || a->e != e) return fail(APXB_ERR_INVALID, "objects belong to another engine");
    if (a->n != f->h.n) return fail(APXB_ERR_INVALID, "operator and factor dimensions differ");
    if (f->precision != APXB_PREC_FP64) return fail(APXB_ERR_INVALID, "apxb_pcg needs an fp64 factor (use the batch engine for fp32)");
    if (!(tol >= 0.0)) return fail(APXB_ERR_INVALID, "tol must be >= 0");
    APXB_CK(cudaSetDevice(e->device));
    cudaStream_t s = e->stream;
    const size_t n = a->n;
    const bool dev = flags & APXB_DEVICE_PTRS;
    if (dev) APXB_CK(cudaMemcpyAsync(a->b_orig, b, 8 * n, cudaMemcpyDeviceToDevice, s));
    else APXB_CK(cudaMemcpyAsync(a->b_orig, b, 8 * n, cudaMemcpyHostToDevice, s));
    // Fixed fields of the state; k_pcg_init sets the rest.
    apxb::pcg_state& hs = *a->h_st;
    std::memset(&hs, 0, sizeof(hs));
    hs.tol = tol; hs.max_iter = max_iter; hs.laplacian = f->h.sddm ? 0 : 1; hs.stag_window = 50;
    hs.center_k = e->center_k; hs.n = a->n; hs.m = f->h.m;
    APXB_CK(cudaMemcpyAsync(a->st, &hs, sizeof(hs), cudaMemcpyHostToDevice, s));
    if (!f->y_armed) apxb::launch_fill_sent64(f->Y, f->h.m, s);
    if (!f->z_armed) apxb::launch_fill_sent64(f->Z, f->h.m, s);
    f->y_armed = true;   // the loop ends on a backward sweep, which re-arms Y
    f->z_armed = false;
    if (a->graph_factor != f || !a->loop) {
        const int rc = build_loop_graph(a, f);
        if (rc) { disarm(f); return rc; }
    }
    const apxb::pcg_ptrs p = pcg_ptrs_of(a, f);
    APXB_CK(cudaEventRecord(e->ev0, s));
    apxb::launch_pcg_init(p, s);
    int rc = enqueue_apply(a, f, p, 0, 0);
    if (rc) { disarm(f); return rc; }
    if (max_iter > 0) {
        if (a->loop_conditional) {
            APXB_CK(cudaGraphLaunch(a->loop, s));
        } else {
            // Host-driven: launch iterations in chunks, poll `done` between them.
            int launched = 0;
            for (;;) {
                const int chunk = 4;
                for (int i = 0; i < chunk && launched < max_iter; ++i, ++launched) APXB_CK(cudaGraphLaunch(a->loop, s));
                APXB_CK(cudaMemcpyAsync(a->h_st, a->st, sizeof(apxb::pcg_state), cudaMemcpyDeviceToHost, s));
                APXB_CK(cudaStreamSynchronize(s));
                if (a->h_st->done || launched >= max_iter || e->h_err->code) break;
            }
        }
    }
    apxb::launch_pcg_finish(p, s);
    APXB_CK(cudaEventRecord(e->ev1, s));
    APXB_CK(cudaGetLastError());
    if (dev) APXB_CK(cudaMemcpyAsync(x, a->x_orig, 8 * n, cudaMemcpyDeviceToDevice, s));
    else APXB_CK(cudaMemcpyAsync(x, a->x_orig, 8 * n, cudaMemcpyDeviceToHost, s));
    APXB_CK(cudaMemcpyAsync(a->h_st, a->st, sizeof(apxb::pcg_state), cudaMemcpyDeviceToHost, s));
    if ((rc = finish(f))) return rc;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    res->iterations = a->h_st->iters;
    res->status = a->h_st->status;
    res->residual = a->h_st->rnorm;
    res->seconds = ms * 1e-3;
    res->true_residual = -1.0;
    if (want_true_residual) {
        // ||b - A x|| / ||b|| in fp64 on the device, from the permuted x.
        apxb::launch_spmv_plain(a->ptr, a->idx, a->val, a->valf, a->x, a->Ap, a->n, e->vec_grid, s);
        apxb::launch_resid(a->perm, a->b_orig, a->Ap, e->d_scal, e->d_partials, e->d_counters + 8, a->n,
                           e->vec_grid, s);
        APXB_CK(cudaMemcpyAsync(e->h_scal, e->d_scal, sizeof(double) * 8, cudaMemcpyDeviceToHost, s));
        if ((rc = finish(f))) return rc;
        const double bn = std::sqrt(e->h_scal[5]);
        res->true_residual = bn > 0.0 ? std::sqrt(e->h_scal[4]) / bn : 0.0;
        // Laplacian x was centred after the permuted x: A 1 = 0, so the residual is unchanged.
    }
    return APXB_OK;
}

}  // extern "C"

extern "C" int apxb_test_stalled_sweep(apxb_engine* e, apxb_factor* f, uint64_t budget_ns) {
    if (!e || !f || f->e != e || budget_ns == 0) return fail(APXB_ERR_INVALID, "bad argument");
    if (f->precision != APXB_PREC_FP64) return fail(APXB_ERR_INVALID, "needs an fp64 factor");
    APXB_CK(cudaSetDevice(e->device));
    cudaStream_t s = e->stream;
    int rc = e->ensure_stage(f->h.n);
    if (rc) return rc;
    APXB_CK(cudaMemsetAsync(e->d_stage_a, 0, 8 * static_cast<size_t>(f->h.n), s));
    // Start the forward work counter past claim unit 0: its rows are never solved.
    const apxb::sweep_ctl start{1u, 0u};
    APXB_CK(cudaMemcpyAsync(f->ctl, &start, sizeof(start), cudaMemcpyHostToDevice, s));
    const unsigned long long saved = e->budget_ns;
    e->budget_ns = budget_ns;
    rc = run_sweep64(f, 0, e->d_stage_a, e->d_stage_b, nullptr, nullptr);
    e->budget_ns = saved;
    APXB_CK(cudaStreamSynchronize(s));
    if (rc) { disarm(f); return rc; }
    rc = finish(f);
    disarm(f);
    return rc;
}

extern "C" int apxb_sweep_pair_timed(apxb_engine* e, apxb_factor* f, const double* d_in, double* d_out, int reps,
                                     double* seconds) {
    if (!e || !f || !d_in || !d_out || reps < 1 || !seconds) return fail(APXB_ERR_INVALID, "bad argument");
    if (f->e != e) return fail(APXB_ERR_INVALID, "factor belongs to another engine");
    APXB_CK(cudaSetDevice(e->device));
    APXB_CK(cudaEventRecord(e->ev0, e->stream));
    for (int i = 0; i < reps; ++i) {
        const int rc = f->precision == APXB_PREC_FP64 ? pair_fp64(f, d_in, d_out) : pair_fp32(f, 1, d_in, d_out);
        if (rc) { disarm(f); return rc; }
    }
    APXB_CK(cudaEventRecord(e->ev1, e->stream));
    const int rc = finish(f);
    if (rc) return rc;
    float ms = 0.0f;
    APXB_CK(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
    *seconds = ms * 1e-3 / reps;
    return APXB_OK;
}
