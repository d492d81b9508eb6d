// Allocation-free per-level range step (see noalloc.cu for who needs it and its limits).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>

namespace tblaeq {

struct Runtime;

constexpr uint64_t kNoAllocMaxGrid = 16384;    // input grid entries per call
constexpr uint64_t kNoAllocMaxOut = 1u << 20;  // output entries per call

struct NoAllocOverflow : std::runtime_error {
    explicit NoAllocOverflow(uint64_t needed)
        : std::runtime_error("no-alloc level step needs " + std::to_string(needed) +
                             " output entries, more than the caller's capacity or the fixed limit") {}
};

// Bytes of the file-scope device scratch array.
uint64_t noAllocScratchBytes();

// Same result as B200Strategy::runLevel for a range query (ids and vals in the reference's order),
// written into caller buffers; returns the number of entries written. Throws NoAllocOverflow when
// the output does not fit, std::invalid_argument beyond the fixed limits.
uint64_t runLevelRangeNoAlloc(Runtime& rt, uint64_t l, const uint64_t* dIds, const double* dVals, uint64_t p,
                              const double* lo, const double* hi, uint64_t* outIds, double* outVals, uint64_t outCap);

}  // namespace tblaeq
