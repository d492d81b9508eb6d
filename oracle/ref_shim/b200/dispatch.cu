// See dispatch.cuh.
#include "dispatch.cuh"

#include <atomic>

#include "B200Strategy.cuh"
#include "src/core/strategies/L0Strategy.cuh"

namespace {
std::atomic<tblaeq_handle*> gHandle{nullptr};
std::atomic<uint64_t> gDispatched{0};
}  // namespace

void b200UseHandleForL0(tblaeq_handle* h) { gHandle.store(h); }

uint64_t b200LevelsDispatched() { return gDispatched.load(); }

std::unique_ptr<IQueryStrategy> b200StrategyForL0(IndexData& idx) {
    tblaeq_handle* h = gHandle.load();
    if (!h) return std::make_unique<L0Strategy>(idx);
    ++gDispatched;
    return std::make_unique<B200Strategy>(idx, h);
}
