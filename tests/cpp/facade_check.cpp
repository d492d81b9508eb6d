// C++ caller of the B200 library's facade (t-blaeq_b200/csrc/handler.hpp), written like a caller of
// the reference's QueryHandler (src/core/QueryHandler.cuh:189-216): load an index directory,
// prepareForQuery, then performQuery over a query file in both result modes and the single-query
// forms. Used by tests/test_gpu_drop_in.py.
//
// usage: facade_check <index_dir> <query_file> <0=range|1=knn> <K> <out.txt>
// out.txt: per mode (ref-parity, exact) and query: "<mode> <query> <level sizes...> | <ids...>"
#include <cstdio>
#include <string>
#include <vector>

#include "handler.hpp"

using namespace tblaeq;

int main(int argc, char** argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s index_dir query_file type K out.txt\n", argv[0]);
        return 2;
    }
    const QueryType t = std::atoi(argv[3]) == 1 ? QueryType::POINT : QueryType::RANGE;
    const size_t K = std::strtoull(argv[4], nullptr, 10);
    FILE* out = std::fopen(argv[5], "w");
    if (!out) return 1;
    try {
        QueryHandler h(argv[1], /*loadFromIndex=*/true);
        h.prepareForQuery(LevelPolicy::L0);
        for (int mode : {kModeRefParity, kModeExact}) {
            h.setMode(mode);
            const QueryResult r = h.performQuery(argv[2], t, /*saveFineMesh=*/true, static_cast<size_t>(-1), K);
            for (size_t q = 0; q < r.ids.size(); ++q) {
                std::fprintf(out, "%d %zu", mode, q);
                for (size_t v : r.levelFineMeshSize[q]) std::fprintf(out, " %zu", v);
                std::fprintf(out, " |");
                for (uint64_t id : r.ids[q]) std::fprintf(out, " %llu", static_cast<unsigned long long>(id));
                std::fprintf(out, "\n");
            }
        }
        // The single-query forms agree with performQuery (upper bound first for ranges).
        const Query q = loadQueryFile(argv[2], t);
        h.setMode(kModeExact);
        const QueryResult all = h.performQuery(argv[2], t, true, static_cast<size_t>(-1), K);
        for (size_t i = 0; i < q.length; ++i) {
            QueryResult one;
            if (t == QueryType::RANGE) {
                const std::vector<double> lo(q.getQueryLo(i), q.getQueryLo(i) + q.dim);
                const std::vector<double> hi(q.getQueryHi(i), q.getQueryHi(i) + q.dim);
                one = h.performSingleRangeQuery(hi, lo, true);
            } else {
                one = h.performSingleKNNQuery(std::vector<double>(q.getQueryPoint(i), q.getQueryPoint(i) + q.dim), K,
                                              true);
            }
            if (one.ids.at(0) != all.ids.at(i)) {
                std::fprintf(stderr, "single query %zu differs from performQuery\n", i);
                return 3;
            }
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    std::fclose(out);
    return 0;
}
