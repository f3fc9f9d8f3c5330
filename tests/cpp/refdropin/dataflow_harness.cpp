// TEST INFRASTRUCTURE: the reference's raw dataflow-sweep contract end to end.
// The reference's own host side -- cuda_host.h's L11 extraction, drop, fp16
// narrowing, transpose and dataflow_build_plan / dataflow_plan_check, the
// steps of its GPU test (tests/test_sptrsv_drop.cpp:1228-1290) -- prepares a
// factor and its batch plans; apxb200's apxchol::dataflow_solve /
// dataflow_solve_fp16 (replacement cuda_dataflow.h) run the sweeps; a serial
// fp64 sweep over the same arrays (after the reference test's
// host_reference_sweep) is the check. C entry points for tests/test_gpu_dataflow.py:
//   dap_df_create  factor (CSC u32/f32) -> both storages, both directions' plans
//                  for one segmentation setting, uploaded
//   dap_df_sweep   one GPU sweep (fp32 or fp16 storage, a grid) of host rhs
//   dap_df_serial  the serial fp64 sweep of the same arrays
//   dap_df_info    plan sizes (batches, split rows, slots) per direction
#include "apxchol/solver/sptrsv/cuda_host.h"
#include "apxchol/solver/sptrsv/cuda_dataflow.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "apxb200.h"

namespace {
thread_local std::string g_err;

namespace ch = apxchol::cuda_host;

template <class T>
T* upload(const T* h, size_t n) {
    T* d = nullptr;
    if (cudaMalloc(&d, sizeof(T) * (n ? n : 1)) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
    if (n && cudaMemcpy(d, h, sizeof(T) * n, cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("cudaMemcpy failed");
    return d;
}

struct dir_plan {
    int* bs = nullptr;
    int* sel = nullptr;
    int4* spec = nullptr;
    int nb = 0, slots = 0, split = 0;
};

struct df_handle {
    int m = 0;
    ch::csr_int<float> LT, Lc;                 // CSR of L^T (back), CSR of L (forward)
    ch::csr_int<std::uint16_t> LT16, L16;
    ch::fp16_scaled_arrays h16;
    std::vector<double> is2;
    dir_plan plan[2];                          // 0 forward, 1 back
    int *d_Lp = nullptr, *d_Li = nullptr, *d_Tp = nullptr, *d_Ti = nullptr;
    float *d_Lv = nullptr, *d_Tv = nullptr, *d_diag = nullptr;
    std::uint16_t *d_Lv16 = nullptr, *d_Tv16 = nullptr;
    double* d_is2 = nullptr;
    unsigned long long* tag = nullptr;
    int* ctrl = nullptr;                       // 2 per direction
    float *d_rhs = nullptr, *d_out = nullptr;
    unsigned epoch = 0;
    ~df_handle() {
        for (void* p : {(void*)d_Lp, (void*)d_Li, (void*)d_Tp, (void*)d_Ti, (void*)d_Lv, (void*)d_Tv, (void*)d_diag,
                        (void*)d_Lv16, (void*)d_Tv16, (void*)d_is2, (void*)tag, (void*)ctrl, (void*)d_rhs,
                        (void*)d_out})
            cudaFree(p);
        for (auto& p : plan) { cudaFree(p.bs); cudaFree(p.sel); cudaFree(p.spec); }
    }
};

ch::csr_int<std::uint16_t> with_values(const ch::csr_int<float>& a, const std::uint16_t* v) {
    ch::csr_int<std::uint16_t> o;
    o.m = a.m; o.nnz = a.nnz; o.ptr = a.ptr;
    o.idx = std::make_unique<int[]>(static_cast<size_t>(a.nnz));
    std::copy_n(a.idx.get(), a.nnz, o.idx.get());
    o.vals = std::make_unique<std::uint16_t[]>(static_cast<size_t>(a.nnz));
    std::copy_n(v, a.nnz, o.vals.get());
    return o;
}
}  // namespace

extern "C" {

const char* dap_df_last_error() { return g_err.c_str(); }

int dap_df_create(int n, const uint32_t* f_colptr, const uint32_t* f_rowidx, const float* f_vals, int m, int seg,
                  int split_min, int max_seg, double drop_rel, void** out) {
    try {
        apxchol::sparse_csc L;
        L.resize(static_cast<uint32_t>(n), static_cast<uint32_t>(n));
        std::memcpy(L.outer_.data(), f_colptr, sizeof(uint32_t) * (static_cast<size_t>(n) + 1));
        L.resizeNonZeros(f_colptr[n]);
        std::memcpy(L.inner_.data(), f_rowidx, sizeof(uint32_t) * f_colptr[n]);
        std::memcpy(L.vals_.data(), f_vals, sizeof(float) * f_colptr[n]);
        auto h = std::make_unique<df_handle>();
        h->m = m;
        h->LT = ch::build_L11_csc_int<float>(L, m);
        const std::vector<float> scales = ch::column_scales(h->LT);
        ch::apply_factor_drop(h->LT, scales, drop_rel, false);
        h->Lc = ch::transpose_csr(h->LT);
        h->h16 = ch::narrow_fp16_scaled(h->LT, scales);
        h->LT16 = with_values(h->LT, h->h16.vals.get());
        h->L16 = ch::transpose_csr(h->LT16);
        h->is2.resize(static_cast<size_t>(m));
        for (int j = 0; j < m; ++j)
            h->is2[j] = static_cast<double>(h->h16.inv_scale[j]) * static_cast<double>(h->h16.inv_scale[j]);
        const int pre = apxchol::dataflow_prefetch_depth();
        const ch::dataflow_seg_params prm{seg, split_min, max_seg};
        int max_slots = 0;
        for (int d = 0; d < 2; ++d) {
            const bool reverse = d == 1;
            const auto& A = reverse ? h->LT : h->Lc;
            const std::vector<int> len = ch::csr_row_lengths(m, A.ptr.data());
            const ch::dataflow_plan pl = ch::dataflow_build_plan(m, reverse, A.ptr.data(), A.idx.get(), len.data(), pre, prm);
            const std::string bad = ch::dataflow_plan_check(pl, m, reverse, len.data(), pre);
            if (!bad.empty()) throw std::runtime_error("dataflow_plan_check: " + bad);
            dir_plan& p = h->plan[d];
            p.bs = upload(pl.batch_start.data(), pl.batch_start.size());
            p.sel = upload(pl.batch_spec.data(), pl.batch_spec.size());
            if (!pl.spec.empty()) p.spec = upload(reinterpret_cast<const int4*>(pl.spec.data()), pl.spec.size());
            p.nb = pl.n_batches();
            p.slots = pl.n_slots;
            p.split = pl.n_split;
            max_slots = std::max(max_slots, pl.n_slots);
        }
        h->d_Lp = upload(h->Lc.ptr.data(), h->Lc.ptr.size());
        h->d_Li = upload(h->Lc.idx.get(), static_cast<size_t>(h->Lc.nnz));
        h->d_Lv = upload(h->Lc.vals.get(), static_cast<size_t>(h->Lc.nnz));
        h->d_Tp = upload(h->LT.ptr.data(), h->LT.ptr.size());
        h->d_Ti = upload(h->LT.idx.get(), static_cast<size_t>(h->LT.nnz));
        h->d_Tv = upload(h->LT.vals.get(), static_cast<size_t>(h->LT.nnz));
        h->d_Lv16 = upload(h->L16.vals.get(), static_cast<size_t>(h->L16.nnz));
        h->d_Tv16 = upload(h->LT16.vals.get(), static_cast<size_t>(h->LT16.nnz));
        h->d_diag = upload(h->h16.diag.data(), h->h16.diag.size());
        h->d_is2 = upload(h->is2.data(), h->is2.size());
        const size_t words = static_cast<size_t>(m) + static_cast<size_t>(max_slots);
        if (cudaMalloc(&h->tag, 8 * words) != cudaSuccess || cudaMemset(h->tag, 0, 8 * words) != cudaSuccess ||
            cudaMalloc(&h->ctrl, 4 * sizeof(int)) != cudaSuccess || cudaMemset(h->ctrl, 0, 4 * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&h->d_rhs, 4 * static_cast<size_t>(m)) != cudaSuccess ||
            cudaMalloc(&h->d_out, 4 * static_cast<size_t>(m)) != cudaSuccess)
            throw std::runtime_error("device allocation failed");
        *out = h.release();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

void dap_df_free(void* h) { delete static_cast<df_handle*>(h); }

int dap_df_info(void* hv, int* m, int* nb, int* split, int* slots) {
    const auto* h = static_cast<const df_handle*>(hv);
    *m = h->m;
    for (int d = 0; d < 2; ++d) { nb[d] = h->plan[d].nb; split[d] = h->plan[d].split; slots[d] = h->plan[d].slots; }
    return 0;
}

// One GPU sweep: reverse 0 solves L y = rhs (CSR of L), 1 solves L^T z = rhs
// (CSR of L^T; fp16 storage: rhs times inv_scale^2). grid 0: dataflow_grid_size.
int dap_df_sweep(void* hv, int reverse, int fp16, int grid, const float* rhs, float* out) {
    try {
        auto* h = static_cast<df_handle*>(hv);
        const dir_plan& p = h->plan[reverse ? 1 : 0];
        if (cudaMemcpy(h->d_rhs, rhs, 4 * static_cast<size_t>(h->m), cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("rhs upload failed");
        const int g = grid > 0 ? grid : apxchol::dataflow_grid_size(fp16 != 0);
        const unsigned e = ++h->epoch;
        int* ctrl = h->ctrl + (reverse ? 2 : 0);
        if (fp16)
            apxchol::dataflow_solve_fp16(0, h->m, reverse != 0, reverse ? h->d_Tp : h->d_Lp, reverse ? h->d_Ti : h->d_Li,
                                         reverse ? h->d_Tv16 : h->d_Lv16, h->d_diag, reverse ? h->d_is2 : nullptr, p.bs,
                                         p.sel, p.spec, p.nb, h->tag, e, ctrl, g, h->d_rhs, h->d_out);
        else
            apxchol::dataflow_solve(0, h->m, reverse != 0, reverse ? h->d_Tp : h->d_Lp, reverse ? h->d_Ti : h->d_Li,
                                    reverse ? h->d_Tv : h->d_Lv, p.bs, p.sel, p.spec, p.nb, h->tag, e, ctrl, g,
                                    h->d_rhs, h->d_out);
        const cudaError_t rc = cudaDeviceSynchronize();
        if (rc != cudaSuccess) throw std::runtime_error(std::string("sweep: ") + cudaGetErrorString(rc));
        if (apxb_dataflow_status() != APXB_OK) throw std::runtime_error(apxb_last_error());
        int c[2] = {1, 1};
        if (cudaMemcpy(c, ctrl, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess || c[0] != 0 || c[1] != 0)
            throw std::runtime_error("ctrl not reset to zero after the sweep");
        if (cudaMemcpy(out, h->d_out, 4 * static_cast<size_t>(h->m), cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("out download failed");
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// The serial fp64 sweep over the same arrays: out[i] = (rhs[i] (* is2[i]) -
// sum_{j != i} w_ij out[j]) / d_i, rows in sweep order; w and d the fp32
// values (d the diagonal slot) or the widened binary16 values and diag16.
int dap_df_serial(void* hv, int reverse, int fp16, const float* rhs, double* out) {
    try {
        const auto* h = static_cast<const df_handle*>(hv);
        const int m = h->m;
        const auto& A = reverse ? h->LT : h->Lc;
        const std::uint16_t* v16 = reverse ? h->LT16.vals.get() : h->L16.vals.get();
        for (int q = 0; q < m; ++q) {
            const int i = reverse ? m - 1 - q : q;
            double s = 0.0, d = 0.0;
            for (int p = A.ptr[i]; p < A.ptr[i + 1]; ++p) {
                const int j = A.idx[p];
                if (j == i) { d = A.vals[p]; continue; }
                const double w = fp16 ? static_cast<double>(ch::widen_fp16(v16[p])) : static_cast<double>(A.vals[p]);
                s += w * out[j];
            }
            if (fp16) d = h->h16.diag[i];
            const double r = fp16 && reverse ? static_cast<double>(rhs[i]) * h->is2[i] : static_cast<double>(rhs[i]);
            out[i] = (r - s) / d;
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

}  // extern "C"
