// Test-infrastructure harness linked against the reference T-BLAEQ objects and its JSONL/payload
// tool sources (built from the reference sources by oracle/Makefile into oracle/_ref/). It is never
// part of the product.
//
// It calls the reference's own refine service, tblaeq::file_index::run_query_service
// (src/file_index/IndexJsonTblaeqQuery.cu:294-380), once per request over one QueryHandler
// prepared with policy L3, as the reference tool's own query does (src/file_index/IndexJsonTblaeqQuery.cu:387):
// the service reads the final grid's ids on the host, which only L3's host-resident grids allow
// (with L0 the grid is device memory). The results go out as text so the parity tests can compare
// the B200 refine service with them.
//
// usage: file_index_harness <index_root> <requests.txt> <out.txt>
//
// requests.txt, one request per line:
//   knn   <timestamp> <knn_k> <include_padding 0|1> <seq>
//   range <start> <end> <range_limit> <include_padding 0|1> <n_seqs> <seq>...
// out.txt, per request:
//   R <candidate_count> <record_count> <slot_count> <n_matches>
//   M <rank> <item_no> <seq> <dtype> <slot> <timestamp %.17g> <diff_us> <payload_offset> <payload_size> <data_file>
// or, when the reference throws:
//   E <message>
// The output is flushed after every request, so a run that dies leaves the requests before it.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "src/core/MemoryPolicy.cuh"
#include "src/core/QueryHandler.cuh"
#include "src/file_index/IndexJsonTblaeqQuery.cuh"

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s index_root requests.txt out.txt\n", argv[0]);
        return 2;
    }
    using namespace tblaeq::file_index;
    const std::string root = argv[1];
    std::ifstream req(argv[2]);
    FILE* out = std::fopen(argv[3], "w");
    if (!req || !out) {
        std::fprintf(stderr, "cannot open the request or output file\n");
        return 1;
    }
    std::ostringstream sink;
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
    QueryHandler handler(root + "/" + kDefaultTblaeqDir, /*loadFromIndex=*/true);
    handler.prepareForQuery(LevelPolicy::L3);

    std::string line;
    while (std::getline(req, line)) {
        if (line.empty()) continue;
        std::istringstream in(line);
        QueryArgs a;
        a.index_root = root;
        std::string mode;
        in >> mode;
        a.mode = mode;
        int pad = 0;
        if (mode == "knn") {
            int seq = 0;
            in >> a.timestamp >> a.knn_k >> pad >> seq;
            a.has_timestamp = true;
            a.seqs = {static_cast<uint8_t>(seq)};
        } else {
            size_t n = 0;
            in >> a.start >> a.end >> a.range_limit >> pad >> n;
            a.has_start = a.has_end = true;
            for (size_t i = 0; i < n; ++i) {
                int s = 0;
                in >> s;
                a.seqs.push_back(static_cast<uint8_t>(s));
            }
        }
        a.has_seq = !a.seqs.empty();
        a.include_padding = pad != 0;
        try {
            const QueryServiceResult r = run_query_service(a, handler);
            std::fprintf(out, "R %zu %zu %zu %zu\n", r.candidate_count, r.record_count, r.slot_count,
                         r.matches.size());
            for (const QueryPayloadMatch& m : r.matches)
                std::fprintf(out, "M %zu %zu %d %d %d %.17g %lld %llu %llu %s\n", m.rank, m.item_no,
                             static_cast<int>(m.seq), static_cast<int>(m.dtype), static_cast<int>(m.slot), m.timestamp,
                             static_cast<long long>(m.diff_us), static_cast<unsigned long long>(m.payload_offset),
                             static_cast<unsigned long long>(m.payload_size), m.data_file.c_str());
        } catch (const std::exception& e) {
            std::string msg = e.what();
            for (char& c : msg)
                if (c == '\n') c = ' ';
            std::fprintf(out, "E %s\n", msg.c_str());
        }
        std::fflush(out);  // a request's lines are complete on disk before the next one runs
    }
    std::fclose(out);
    std::cout.rdbuf(old);
    return 0;
}
