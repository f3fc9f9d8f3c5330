// apxb200 replacement of the apxchol reference's raw dataflow-sweep header,
// include/apxchol/solver/sptrsv/cuda_dataflow.h (cuda_dataflow.h:150-208): the
// same four functions, implemented by libapxb200 (csrc/tagflow.cu) with the
// reference's contract -- CSR of the triangle with the diagonal inside every
// row, the batch tables of cuda_host::dataflow_build_plan, 64-bit {value,
// epoch} tagged words, ctrl = {ticket, finished warps} zero at entry and exit.
// The replacement cuda_sptrsv of this tree does not use them (it sweeps its
// own plans); callers that drive the kernel with the reference's plans do,
// the reference's GPU tests among them.
//
// One difference: every wait is bounded. A launch whose wait makes no
// progress for one second (a plan or an epoch that breaks the contract) ends
// instead of hanging and records it; apxb_dataflow_status() (apxb200.h)
// returns and clears that record.
#pragma once
#include <cuda_runtime.h>

#include "apxb200.h"

namespace apxchol {

// The device-side value type of the sweep: fp32.
using sptrsv_gpu_value_t = float;

// Threads per block of the persistent kernel.
inline constexpr int kDataflowBlock = 256;

// Entries of a row each lane holds in flight; the host's batch packing
// (cuda_host::dataflow_batches / dataflow_build_plan) takes it as `pre`.
int dataflow_prefetch_depth();

// The persistent grid: resident blocks per SM x SMs of the current device
// (APXCHOL_GPU_DATAFLOW_BLOCKS=<n> overrides).
int dataflow_grid_size(bool fp16);

// One sweep T out = rhs (fp32 values); arguments as cuda_dataflow.h:174-192.
void dataflow_solve(cudaStream_t stream, int m, bool reverse, const int* rowptr, const int* colidx,
                    const sptrsv_gpu_value_t* vals, const int* batch_start, const int* batch_spec, const int4* spec,
                    int n_batches, unsigned long long* tag, unsigned epoch, int* ctrl, int grid,
                    const sptrsv_gpu_value_t* rhs, sptrsv_gpu_value_t* out);

// The same over the fp16 column-scaled storage: binary16 values (the
// diagonal slot skipped), the fp32 diagonal diag[i], and rhs[i] * in_scale[i]
// formed in double when in_scale is given (cuda_dataflow.h:194-206).
void dataflow_solve_fp16(cudaStream_t stream, int m, bool reverse, const int* rowptr, const int* colidx,
                         const unsigned short* vals16, const float* diag, const double* in_scale,
                         const int* batch_start, const int* batch_spec, const int4* spec, int n_batches,
                         unsigned long long* tag, unsigned epoch, int* ctrl, int grid,
                         const sptrsv_gpu_value_t* rhs, sptrsv_gpu_value_t* out);

}  // namespace apxchol
