// Shared device-side definitions for the T-BLAEQ B200 traversal kernels.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace tblaeq {

// Error bits a kernel may raise in the device status word; the host turns them into
// TBLAEQ_ERR_OVERFLOW / TBLAEQ_ERR_TIMEOUT before any result is read.
enum DeviceStatus : uint32_t {
    kStatusOverflowEntries = 1u << 0,   // output frontier / result capacity exceeded
    kStatusOverflowItems = 1u << 1,     // next-level work items exceed the tile-start capacity
    kStatusOverflowSum = 1u << 2,       // 32-bit child-prefix overflow
    kStatusLookbackTimeout = 1u << 3,   // a decoupled look-back spin gave up
    kStatusWindowOverflow = 1u << 4,    // a tile spanned more frontier entries than it can stage
};
// After any of these the frontiers that follow are not to be read (a wrapped child prefix, a
// look-back that gave up): the kernels of the rest of the batch return at once.
constexpr uint32_t kStatusInconsistent = kStatusOverflowSum | kStatusLookbackTimeout | kStatusWindowOverflow;

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const std::string& what) : std::runtime_error(what), code(c) {}
};

// Kernel launches issued by this library since load (a launch captured into a CUDA graph counts
// once, at capture; replays of the graph do not count here).
extern std::atomic<uint64_t> gKernelLaunches;

// A batch whose traversal does not fit the 32-bit item and entry space; smaller batches do.
struct SplitBatch : CudaError {
    explicit SplitBatch(const std::string& what) : CudaError(cudaErrorMemoryAllocation, what) {}
};

#define TBLAEQ_CUDA(call)                                                                                     \
    do {                                                                                                      \
        cudaError_t e_ = (call);                                                                              \
        if (e_ != cudaSuccess) {                                                                              \
            throw ::tblaeq::CudaError(e_, std::string(#call) + " failed: " + cudaGetErrorString(e_) + " at " + \
                                              __FILE__ + ":" + std::to_string(__LINE__));                      \
        }                                                                                                     \
    } while (0)

// Error check after a kernel launch; counts the launch.
#define TBLAEQ_LAUNCHED()                                                     \
    do {                                                                      \
        ::tblaeq::gKernelLaunches.fetch_add(1, std::memory_order_relaxed);    \
        TBLAEQ_CUDA(cudaGetLastError());                                      \
    } while (0)

}  // namespace tblaeq
