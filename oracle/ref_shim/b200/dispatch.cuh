// The hook a maintainer adds to PolicyScheduler::makeForLevel (src/core/MemoryPolicy.cu:303-316):
// levels whose policy is L0 go to the B200 strategy while a handle is registered. oracle/Makefile
// compiles the reference's MemoryPolicy.cu with its L0 case in makeForLevel pointed here (and this
// header force-included); nothing else of the reference changes.
#pragma once

#include <cstdint>
#include <memory>

#include "tblaeq.h"

class IndexData;
class IQueryStrategy;

// Registers the handle every L0 level dispatches to (nullptr: back to the reference's L0Strategy).
void b200UseHandleForL0(tblaeq_handle* h);
// Levels dispatched to the B200 strategy so far.
uint64_t b200LevelsDispatched();
// makeForLevel's L0 case.
std::unique_ptr<IQueryStrategy> b200StrategyForL0(IndexData& idx);
