// Serving loop: continuous batching of range and KNN requests on one GPU.
//
// Requests are submitted from any thread and queue per lane. In the default two-lane layout, range
// and KNN requests have separate lanes, each a worker thread with its own batch engine (device
// workspace, kept resident between batches) and CUDA stream, so the two kinds of work overlap on
// the device. Each lane batches continuously: whatever arrived while its previous batch was on the
// GPU forms the next batch, up to the lane's slot limit, which shrinks when the engine's workspace
// per query would exceed the lane's device-memory budget (the admission rule). A KNN batch that
// does not fit one traversal is split in halves. Latency is measured from each request's arrival
// time to the moment its result is posted.
//
// The reference serves one query at a time behind its HTTP front end (src/HTTPServer.cu:414-550);
// this is the batched replacement for that loop, without the HTTP layer.
#pragma once

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.hpp"

namespace tblaeq {

struct Runtime;

struct ServeConfig {
    uint32_t maxBatch = 4096;   // requests per batch and lane
    uint64_t memoryBudget = 0;  // traversal workspace bytes per lane (0: a quarter of free memory)
    int mode = kModeExact;      // range mode; KNN is always exact
    bool learned = true;        // rank KNN frontiers with the trained scorer, when there is one
    int lanes = 2;              // 2: range and KNN lanes; 1: one lane serves both, in arrival order
    bool levels = false;        // also record every request's generated-children count per level
};

struct ServeStats {
    uint64_t submitted = 0, completed = 0, failed = 0, batches = 0, maxBatch = 0;
    double meanBatch = 0, p50Us = 0, p99Us = 0, meanUs = 0, maxUs = 0;
    double spanS = 0;  // first arrival to last completion of the measured requests
};

class Server {
public:
    using Clock = std::chrono::steady_clock;

    struct Result {
        int status = 0;  // 0 ok, otherwise a tblaeq status code
        std::string error;
        std::vector<uint64_t> ids;
        std::vector<double> dist2;  // KNN
        double latencyUs = 0;
        std::vector<uint32_t> levels;  // per interval, coarsest first (ServeConfig::levels)
    };

    Server(Runtime& rt, const ServeConfig& cfg);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    // qtype 0 = KNN (point[D], K), 1 = range (lo[D] hi[D]). Returns the request's ticket.
    uint64_t submit(int qtype, const double* query, uint32_t K, Clock::time_point arrival);
    // Submits n requests, each at its arrival time (µs after the call), from the calling thread.
    std::vector<uint64_t> replay(uint64_t n, const int* qtypes, const double* queries, const uint64_t* offsets,
                                 const uint32_t* K, const double* arrivalUs);
    // true: the result is moved into `out` and the ticket released. false: not done within waitMs.
    bool poll(uint64_t ticket, Result& out, int waitMs);
    // Puts a polled result back (a caller whose buffer was too small polls it again).
    void repost(uint64_t ticket, Result&& r);
    bool known(uint64_t ticket) const;
    // Blocks until every submitted request has completed (or waitMs passes); true when idle.
    bool waitIdle(int waitMs);
    ServeStats stats(bool reset);
    void stop();

private:
    struct Request {
        uint64_t ticket;
        int qtype;
        std::vector<double> q;
        uint32_t K;
        Clock::time_point arrival;
    };
    struct Lane {
        std::deque<Request> pending;
        std::thread worker;
        std::unique_ptr<BatchEngine> engine;
        cudaStream_t stream = nullptr;
        DeviceMem dq, dk;
        uint32_t cap = 0;   // current admission limit (slots)
        uint64_t maxN = 0;  // largest batch this lane has run
    };

    void work(Lane& lane);
    void runGroup(Lane& lane, std::vector<Request>& batch, size_t begin, size_t end);
    void post(std::vector<Request>& batch, size_t begin, size_t end, const std::vector<uint32_t>& levels,
              const std::vector<uint64_t>& offs,
              const std::vector<uint64_t>& ids, const std::vector<double>& d2, int status, const std::string& err);

    Runtime& rt_;
    ServeConfig cfg_;
    int device_ = 0;
    uint64_t D_ = 0;
    mutable std::mutex mu_;
    std::condition_variable cvWork_, cvDone_;
    bool stopping_ = false;
    uint64_t nextTicket_ = 1;
    std::vector<std::unique_ptr<Lane>> lanes_;
    std::unordered_map<uint64_t, Result> done_;
    std::unordered_map<uint64_t, bool> inFlight_;
    // statistics since the last reset
    std::vector<double> latUs_;
    uint64_t submitted_ = 0, completed_ = 0, failed_ = 0, batches_ = 0, batched_ = 0, maxBatchSeen_ = 0;
    Clock::time_point firstArrival_{}, lastDone_{};
    bool haveFirst_ = false;
};

}  // namespace tblaeq
