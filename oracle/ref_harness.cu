// Test-infrastructure harness linked against the reference T-BLAEQ objects (built from the
// reference sources by oracle/Makefile into oracle/_ref/). It is never part of the product.
//
// It runs the reference's own public API one query at a time, exactly as its HTTP server does
// (src/HTTPServer.cu:498,525 -> QueryHandler::performSingle{KNN,Range}Query with
// saveFineMesh=true), and dumps each query's final candidate-id set so the parity tests can
// compare the B200 path against the reference CUDA build on the same index and queries.
//
// usage: ref_harness <index_dir> <query_file> <0=range|1=knn> <K> <policy L0..L3> <out.bin>
//        (b200_drop_in: the same arguments)
//
// out.bin (little endian):
//   u64 nq, u64 intervals
//   per query: u64 levelSizes[intervals], f64 query_us, u64 count, u64 ids[count] (ascending)
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdint>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>
#include "src/core/QueryHandler.cuh"
#include "src/core/MemoryPolicy.cuh"
#include "src/Data_Structures/File.cuh"
#ifdef TBLAEQ_DROP_IN
// Built as b200_drop_in: the same driver, with every L0 level of the reference's QueryEngine
// dispatched to the B200 library through the reference-side adapter (ref_shim/b200). It also
// writes <out.bin>.levels: the number of levels the B200 strategy ran.
#include "b200/dispatch.cuh"
#endif

int main(int argc, char** argv) {
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s index_dir query_file type K policy out.bin\n", argv[0]);
        return 2;
    }
    const std::string indexDir = argv[1];
    const std::string queryFile = argv[2];
    const int type = std::atoi(argv[3]);
    const size_t K = std::strtoull(argv[4], nullptr, 10);
    const std::string policy = argv[5];
    const std::string outPath = argv[6];

    // Silence the reference's per-level logging; results go to out.bin.
    std::ostringstream sink;
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());

    QueryHandler handler(indexDir, /*loadFromIndex=*/true);
    handler.prepareForQuery(IndexPolicy::parseLevel(policy));
#ifdef TBLAEQ_DROP_IN
    tblaeq_handle* b200 = nullptr;
    if (tblaeq_open(indexDir.c_str(), &b200) != TBLAEQ_OK || tblaeq_prepare(b200, nullptr, 0) != TBLAEQ_OK) {
        std::cout.rdbuf(old);
        std::fprintf(stderr, "B200 library: %s\n", tblaeq_last_error());
        return 1;
    }
    b200UseHandleForL0(b200);
#endif

    const Query q = (type == 1) ? loadQueryPointFromFile(queryFile) : loadQueryRangeFromFile(queryFile);
    FILE* f = std::fopen(outPath.c_str(), "wb");
    if (!f) {
        std::cout.rdbuf(old);
        std::fprintf(stderr, "cannot open %s\n", outPath.c_str());
        return 1;
    }
    const uint64_t nq = static_cast<uint64_t>(q.length);
    uint64_t intervals = 0;
    std::fwrite(&nq, 8, 1, f);
    const long intervalsPos = std::ftell(f);
    std::fwrite(&intervals, 8, 1, f);

    for (int i = 0; i < q.length; ++i) {
        const auto t0 = std::chrono::steady_clock::now();
        QueryResult r = (type == 1)
            ? handler.performSingleKNNQuery(q.getQueryPoint(i), K, /*saveFineMesh=*/true)
            : [&] {
                  auto [lo, hi] = q.getQueryRange(i);
                  return handler.performSingleRangeQuery(hi, lo, /*saveFineMesh=*/true);
              }();
        const auto t1 = std::chrono::steady_clock::now();
        const double us = std::chrono::duration<double, std::micro>(t1 - t0).count();
        const SparseGrid* g = r.fineMesh.at(0);
        const size_t n = g->get_nnz_nums();
        std::vector<uint64_t> ids(n);
        if (n) {
            if (r.fineMeshOnHost.at(0)) {
                std::copy(g->get_ids_(), g->get_ids_() + n, ids.begin());
            } else {
                cudaMemcpy(ids.data(), g->get_ids_(), n * sizeof(uint64_t), cudaMemcpyDeviceToHost);
            }
        }
        std::sort(ids.begin(), ids.end());
        const auto& lv = r.levelFineMeshSize.at(0);
        intervals = lv.size();
        for (size_t l = 0; l < lv.size(); ++l) {
            const uint64_t v = lv[l];
            std::fwrite(&v, 8, 1, f);
        }
        std::fwrite(&us, 8, 1, f);
        const uint64_t cnt = n;
        std::fwrite(&cnt, 8, 1, f);
        if (n) {
            std::fwrite(ids.data(), 8, n, f);
        }
    }
    std::fseek(f, intervalsPos, SEEK_SET);
    std::fwrite(&intervals, 8, 1, f);
    std::fclose(f);
    std::cout.rdbuf(old);
#ifdef TBLAEQ_DROP_IN
    b200UseHandleForL0(nullptr);
    if (FILE* lv = std::fopen((outPath + ".levels").c_str(), "w")) {
        std::fprintf(lv, "%llu\n", static_cast<unsigned long long>(b200LevelsDispatched()));
        std::fclose(lv);
    }
#endif
    return 0;
}
