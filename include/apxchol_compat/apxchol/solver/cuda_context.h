// apxb200 replacement of the apxchol reference's device-initialisation
// header, include/apxchol/solver/cuda_context.h (namespace cuda_ctx), which
// preconditioner.h calls around its factorization: prewarm() before the host
// elimination (preconditioner.h:194), ensure_context() before the SpTRSV
// setup (preconditioner.h:279-283).
//
// Here the first device touch is the process's apxb200 engine (stream, error
// word, workspaces on the calling thread's current device), the object every
// replacement class of this tree shares. prewarm() creates it on a helper
// thread while the elimination runs; ensure_context() waits for it and returns
// the seconds the caller waited; context_seconds() is how long the creation
// itself took. Creation errors are not thrown here: the setup's own first
// library call reports them with the library's message. Without
// APXCHOL_USE_CUDA the functions do nothing, as the reference's.
#pragma once

#include <chrono>
#include <mutex>

#if defined(APXCHOL_USE_CUDA)
#include <cuda_runtime.h>
#include <thread>

#include "apxb200.hpp"
#endif

namespace apxchol::cuda_ctx {

#if defined(APXCHOL_USE_CUDA)

namespace detail {

struct prewarm_state {
    std::mutex mu;
    std::thread worker;
    bool started = false;
    double ctx_seconds = 0.0;
    ~prewarm_state() {
        if (worker.joinable()) worker.join();
    }
};

inline prewarm_state& state() {
    static prewarm_state s;
    return s;
}

// Creates the shared engine on `device`, timed; failures stay silent (see above).
inline double create_engine(int device) {
    const auto t0 = std::chrono::steady_clock::now();
    if (cudaSetDevice(device) == cudaSuccess) {
        try {
            (void)apxb::engine::shared(device);
        } catch (...) {
        }
    }
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace detail

inline void prewarm() {
    auto& s = detail::state();
    std::lock_guard<std::mutex> lock(s.mu);
    if (s.started) return;
    s.started = true;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) device = 0;   // the caller's current device
    s.worker = std::thread([&s, device] { s.ctx_seconds = detail::create_engine(device); });
}

inline double ensure_context() {
    auto& s = detail::state();
    const auto t0 = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lock(s.mu);
    if (s.worker.joinable()) {
        s.worker.join();
    } else if (!s.started) {
        s.started = true;
        int device = 0;
        if (cudaGetDevice(&device) != cudaSuccess) device = 0;
        s.ctx_seconds = detail::create_engine(device);
    }
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

inline double context_seconds() {
    auto& s = detail::state();
    std::lock_guard<std::mutex> lock(s.mu);
    return s.ctx_seconds;
}

#else

inline void prewarm() {}
inline double ensure_context() { return 0.0; }
inline double context_seconds() { return 0.0; }

#endif

}  // namespace apxchol::cuda_ctx
