// Reference-side adapter (compiled against the reference's own headers): the B200 library as one
// more IQueryStrategy (src/core/strategies/IQueryStrategy.cuh:73-107). This is the code a
// maintainer adds to the reference tree to adopt the per-level plugin; the B200 library is reached
// only through its C ABI (include/tblaeq.h).
//
// Every level runs through tblaeq_level: the input grid's device pointers go in as they are (the
// coarsest view QueryEngine builds from IndexData, or the previous level's B200 output), and the
// returned grid points into buffers the handle owns, like the reference's L0 strategy
// (ownsIds = ownsVals = false, src/core/strategies/L0Strategy.cu:190): valid until the next call
// for the same level, so QueryEngine frees only the SparseGrid object.
#pragma once

#include <cstdint>
#include <ostream>
#include <stdexcept>
#include <string>

#include "tblaeq.h"
#include "src/core/IndexData.cuh"
#include "src/core/strategies/IQueryStrategy.cuh"

class B200Strategy final : public IQueryStrategy {
public:
    B200Strategy(IndexData& idx, tblaeq_handle* h) : idx_(idx), h_(h) {}
    ~B200Strategy() override = default;

    // The handle was opened on the same index directory; the device copy is made once.
    void prepare(std::ostream& reportOs) override {
        tblaeq_index_info info{};
        check(tblaeq_info(h_, &info), "tblaeq_info");
        if (info.N != idx_.N || info.D != idx_.D || info.intervals != idx_.intervals)
            throw std::runtime_error("B200Strategy: the handle holds another index");
        if (!info.prepared) check(tblaeq_prepare(h_, nullptr, 0), "tblaeq_prepare");
        reportOs << "B200 strategy: " << info.deviceBytes << " bytes of index on the device\n";
    }

    LevelResult runLevel(size_t l, SparseGrid* cur, QueryType qType, const double* lo, const double* hi,
                         const double* queryPoint, size_t K) override {
        const tblaeq_grid in{cur->get_num_rows(), cur->get_dimensions(), cur->get_nnz_nums(),
                             reinterpret_cast<const uint64_t*>(cur->get_ids_()), cur->get_vals_()};
        tblaeq_grid out{};
        const int qt = (qType == QueryType::RANGE) ? TBLAEQ_RANGE : TBLAEQ_POINT;
        check(tblaeq_level(h_, l, &in, qt, lo, hi, queryPoint, K, &out), "tblaeq_level");
        auto* g = new SparseGrid(out.numRows, out.dim, out.nnz, reinterpret_cast<size_t*>(const_cast<uint64_t*>(out.ids)),
                                 const_cast<double*>(out.vals));
        return {g, /*ownsIds=*/false, /*ownsVals=*/false, /*onHost=*/false};
    }

private:
    static void check(int rc, const char* what) {
        if (rc != TBLAEQ_OK) throw std::runtime_error(std::string(what) + ": " + tblaeq_last_error());
    }
    IndexData& idx_;
    tblaeq_handle* h_;
};
