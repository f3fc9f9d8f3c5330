// apxb_sweep_pair_noalloc: the fp64 sweep pair out = (L L^T)^-1 in without
// any device allocation in the call.
//
// Some callers cannot allocate device memory at the moment they need a
// preconditioner application: a host application that reserves the GPU's
// memory up front for its own pool and forbids allocations outside it, or a
// latency-bound loop that cannot afford the device-wide synchronisation that
// cudaMalloc / cudaFree can cause. apxb_sweep_pair keeps its intermediate
// vectors in buffers of the factor (allocated lazily and re-armed between
// calls); this variant keeps them -- the forward result, the backward result
// and the two work-claim counters -- in one fixed array of device memory
// that belongs to the library, so the call itself allocates nothing (the
// engine and the factor, created beforehand, hold everything else).
//
// The array: kNoAllocMaxRows rows, 256 + 16 * kNoAllocMaxRows bytes
// (1 MiB + 256 B), held by every GPU that loads this code until the process
// exits. Its host-side name is not a device address: the address is taken with
// cudaGetSymbolAddress once per device, with that device current, on the first
// call that runs on it, and kept for the life of the process: after a
// cudaDeviceReset the module is loaded again and the kept address is stale,
// so this entry point must not be used on a device that has been reset.
// Every call ends by reading the engine's error word, which waits for the
// engine stream.
#include <mutex>

#include "objects.hpp"

namespace {

constexpr uint32_t kNoAllocMaxRows = 65536;
constexpr size_t kHeadWords = 32;   // 256 bytes: the two sweep_ctl counters, padded
constexpr size_t kScratchWords = kHeadWords + 2 * static_cast<size_t>(kNoAllocMaxRows);
constexpr int kMaxDevices = 64;

// [0, 256 B): sweep_ctl[2]; then Y[kNoAllocMaxRows]; then Z[kNoAllocMaxRows].
static __device__ __align__(256) double g_sweep_scratch[kScratchWords];

std::mutex g_scratch_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Every call re-arms what it uses: both counters to zero and both result
// vectors to the not-yet-solved marker (the array keeps the previous call's
// contents).
__global__ void k_noalloc_arm(uint32_t m) {
    const double sent = apxb::sent_of(0.0);
    double* y = g_sweep_scratch + kHeadWords;
    double* z = y + kNoAllocMaxRows;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        y[i] = sent;
        z[i] = sent;
    }
    if (blockIdx.x == 0 && threadIdx.x < 2 * sizeof(apxb::sweep_ctl) / sizeof(unsigned))
        reinterpret_cast<unsigned*>(g_sweep_scratch)[threadIdx.x] = 0u;
}

// Device address of the scratch array on `device` (current); set up once per device.
int scratch_on(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) return fail(APXB_ERR_INVALID, "device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&p, g_sweep_scratch);
        if (rc != cudaSuccess || !p)
            return fail(APXB_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(rc));
        g_scratch_ptr[device] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[device];
    return APXB_OK;
}

apxb::sweep_args<double> noalloc_args(const apxb_factor* f, int dir, apxb::sweep_ctl* ctl) {
    apxb::sweep_args<double> a{};
    plan_args(f, dir, a);
    a.ctl = ctl + dir;
    a.err = f->e->d_err;
    a.budget_ns = f->e->budget_ns;
    a.k = 1;
    return a;
}

}  // namespace

extern "C" int apxb_sweep_pair_noalloc(apxb_engine* e, apxb_factor* f, const double* d_in, double* d_out) {
    if (!e || !f || !d_in || !d_out) return fail(APXB_ERR_INVALID, "bad argument");
    if (f->e != e) return fail(APXB_ERR_INVALID, "factor belongs to another engine");
    if (f->precision != APXB_PREC_FP64) return fail(APXB_ERR_INVALID, "apxb_sweep_pair_noalloc needs an fp64 factor");
    if (f->h.m > kNoAllocMaxRows)
        return fail(APXB_ERR_INVALID, "factor has " + std::to_string(f->h.m) +
                                          " rows; apxb_sweep_pair_noalloc handles at most " +
                                          std::to_string(kNoAllocMaxRows));
    APXB_CK(cudaSetDevice(e->device));
    double* base = nullptr;
    int rc = scratch_on(e->device, &base);
    if (rc) return rc;
    auto* ctl = reinterpret_cast<apxb::sweep_ctl*>(base);
    double* y = base + kHeadWords;
    double* z = y + kNoAllocMaxRows;
    cudaStream_t s = e->stream;
    const uint32_t m = f->h.m;
    k_noalloc_arm<<<std::max(1u, std::min((m + 255u) / 256u, 4u * static_cast<unsigned>(e->num_sms))), 256, 0, s>>>(m);
    const int grid = e->sweep_grid > 0 ? e->sweep_grid : f->grid64;
    apxb::sweep_args<double> a = noalloc_args(f, 0, ctl);
    a.in = d_in; a.out = y;
    apxb::launch_sweep64(0, a, grid, s);
    a = noalloc_args(f, 1, ctl);
    a.in = y; a.out = z; a.copy_out = d_out;
    apxb::launch_sweep64(1, a, grid, s);
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return fail(APXB_ERR_CUDA, std::string("sweep launch: ") + cudaGetErrorString(le));
    return e->take_error();
}
