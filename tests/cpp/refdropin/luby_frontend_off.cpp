// TEST INFRASTRUCTURE (drop-in build): the reference's optional GPU Luby
// selector of its factorization (include/apxchol/solver/gpu_luby_frontend.h,
// src/cuda_luby_frontend.cu) is part of the setup phase, which stays the
// reference's CPU code here. Its CUDA build references the selector's class;
// this definition keeps it off: configured_mode() is `disabled` (the
// reference's own default, APXCHOL_GPU_LUBY_FRONTEND unset), so the
// factorization never constructs it, and anything that would is an error.
#include "apxchol/solver/gpu_luby_frontend.h"

#include <stdexcept>

namespace apxchol::detail {

struct gpu_luby_frontend::impl {};

namespace {
[[noreturn]] void off() {
    throw std::runtime_error("the GPU Luby selector of the factorization is not part of this build "
                             "(the setup phase runs on the CPU)");
}
}  // namespace

gpu_luby_frontend::mode gpu_luby_frontend::configured_mode() { return mode::disabled; }
bool gpu_luby_frontend::automatic_worthwhile(node_index, std::size_t, std::size_t) { return false; }
gpu_luby_frontend::runtime_probe gpu_luby_frontend::probe_runtime(node_index, std::size_t) { return {}; }
gpu_luby_frontend::gpu_luby_frontend(node_index, std::span<const gpu_topology_edge>) { off(); }
gpu_luby_frontend::~gpu_luby_frontend() = default;
gpu_luby_frontend::gpu_luby_frontend(gpu_luby_frontend&&) noexcept = default;
gpu_luby_frontend& gpu_luby_frontend::operator=(gpu_luby_frontend&&) noexcept = default;
gpu_luby_frontend::prepare_result gpu_luby_frontend::prepare(std::span<const node_index>, const partition_options&) { off(); }
std::span<const node_index> gpu_luby_frontend::host_candidates() const { off(); }
std::span<const node_index> gpu_luby_frontend::host_active_degrees() const { off(); }
const partition_result& gpu_luby_frontend::select(unsigned, std::uint64_t) { off(); }
void gpu_luby_frontend::advance(std::span<const node_index>, std::span<const gpu_topology_edge>) { off(); }

}  // namespace apxchol::detail
