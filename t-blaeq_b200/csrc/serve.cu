// Serving loop (see serve.hpp).
#include "serve.hpp"

#include <algorithm>
#include <stdexcept>

#include "handler.hpp"
#include "scorer.hpp"

namespace tblaeq {

namespace {

constexpr int kQtypePoint = 0;
constexpr int kQtypeRange = 1;

double percentile(std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const size_t i = std::min(v.size() - 1, static_cast<size_t>(p * static_cast<double>(v.size() - 1) + 0.5));
    return v[i];
}

}  // namespace

Server::Server(Runtime& rt, const ServeConfig& cfg) : rt_(rt), cfg_(cfg) {
    if (cfg_.maxBatch == 0) throw std::invalid_argument("serving needs max_batch >= 1");
    if (cfg_.lanes != 1 && cfg_.lanes != 2) throw std::invalid_argument("serving lanes must be 1 or 2");
    TBLAEQ_CUDA(cudaGetDevice(&device_));
    D_ = rt_.dev->D;
    if (cfg_.memoryBudget == 0) {
        size_t freeB = 0, totalB = 0;
        TBLAEQ_CUDA(cudaMemGetInfo(&freeB, &totalB));
        cfg_.memoryBudget = freeB / 4;
    }
    for (int l = 0; l < cfg_.lanes; ++l) {
        auto lane = std::make_unique<Lane>();
        TBLAEQ_CUDA(cudaStreamCreateWithFlags(&lane->stream, cudaStreamNonBlocking));
        lane->engine = std::make_unique<BatchEngine>(*rt_.dev, lane->stream);
        if (cfg_.learned && scorerTrained(rt_)) attachScorer(rt_, *lane->engine);
        lane->cap = cfg_.maxBatch;
        lanes_.push_back(std::move(lane));
    }
    for (auto& lane : lanes_) {
        Lane* l = lane.get();
        l->worker = std::thread([this, l] { work(*l); });
    }
}

Server::~Server() {
    try {
        stop();
    } catch (...) {
    }
}

void Server::stop() {
    {
        std::lock_guard<std::mutex> g(mu_);
        if (stopping_ && lanes_.empty()) return;
        stopping_ = true;
    }
    cvWork_.notify_all();
    for (auto& lane : lanes_) {
        if (lane->worker.joinable()) lane->worker.join();
    }
    for (auto& lane : lanes_) {
        lane->engine.reset();
        lane->dq = DeviceMem();
        lane->dk = DeviceMem();
        if (lane->stream) cudaStreamDestroy(lane->stream);
        lane->stream = nullptr;
    }
    lanes_.clear();
    cvDone_.notify_all();
}

uint64_t Server::submit(int qtype, const double* query, uint32_t K, Clock::time_point arrival) {
    if (qtype != kQtypePoint && qtype != kQtypeRange) throw std::invalid_argument("bad query type");
    if (!query) throw std::invalid_argument("null query");
    Request r;
    r.qtype = qtype;
    r.q.assign(query, query + (qtype == kQtypeRange ? 2 * D_ : D_));
    r.K = K;
    r.arrival = arrival;
    uint64_t t;
    {
        std::lock_guard<std::mutex> g(mu_);
        if (stopping_) throw std::logic_error("the server is stopping");
        t = r.ticket = nextTicket_++;
        Lane& lane = *lanes_[(cfg_.lanes == 2 && qtype == kQtypePoint) ? 1 : 0];
        lane.pending.push_back(std::move(r));
        inFlight_[t] = true;
        ++submitted_;
        if (!haveFirst_ || arrival < firstArrival_) {
            firstArrival_ = arrival;
            haveFirst_ = true;
        }
    }
    cvWork_.notify_all();
    return t;
}

std::vector<uint64_t> Server::replay(uint64_t n, const int* qtypes, const double* queries, const uint64_t* offsets,
                                     const uint32_t* K, const double* arrivalUs) {
    std::vector<uint64_t> tickets(n);
    const Clock::time_point t0 = Clock::now();
    for (uint64_t i = 0; i < n; ++i) {
        const Clock::time_point at =
            t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::micro>(arrivalUs[i]));
        // Sleep while the next arrival is far, spin for the last stretch.
        for (;;) {
            const Clock::time_point now = Clock::now();
            if (now >= at) break;
            if (at - now > std::chrono::microseconds(200))
                std::this_thread::sleep_for(at - now - std::chrono::microseconds(100));
        }
        tickets[i] = submit(qtypes[i], queries + offsets[i], K ? K[i] : 0, at);
    }
    return tickets;
}

bool Server::known(uint64_t ticket) const {
    std::lock_guard<std::mutex> g(mu_);
    return inFlight_.count(ticket) || done_.count(ticket);
}

bool Server::poll(uint64_t ticket, Result& out, int waitMs) {
    std::unique_lock<std::mutex> g(mu_);
    if (!inFlight_.count(ticket) && !done_.count(ticket)) throw std::out_of_range("unknown ticket");
    const auto ready = [&] { return done_.count(ticket) > 0; };
    if (!ready()) {
        if (waitMs <= 0) return false;
        if (!cvDone_.wait_for(g, std::chrono::milliseconds(waitMs), ready)) return false;
    }
    auto it = done_.find(ticket);
    out = std::move(it->second);
    done_.erase(it);
    return true;
}

void Server::repost(uint64_t ticket, Result&& r) {
    {
        std::lock_guard<std::mutex> g(mu_);
        done_[ticket] = std::move(r);
    }
    cvDone_.notify_all();
}

bool Server::waitIdle(int waitMs) {
    std::unique_lock<std::mutex> g(mu_);
    return cvDone_.wait_for(g, std::chrono::milliseconds(std::max(waitMs, 0)), [&] { return inFlight_.empty(); });
}

ServeStats Server::stats(bool reset) {
    std::lock_guard<std::mutex> g(mu_);
    ServeStats s;
    s.submitted = submitted_;
    s.completed = completed_;
    s.failed = failed_;
    s.batches = batches_;
    s.maxBatch = maxBatchSeen_;
    s.meanBatch = batches_ ? static_cast<double>(batched_) / static_cast<double>(batches_) : 0.0;
    s.p50Us = percentile(latUs_, 0.50);
    s.p99Us = percentile(latUs_, 0.99);
    double sum = 0.0, mx = 0.0;
    for (double v : latUs_) {
        sum += v;
        mx = std::max(mx, v);
    }
    s.meanUs = latUs_.empty() ? 0.0 : sum / static_cast<double>(latUs_.size());
    s.maxUs = mx;
    s.spanS = (haveFirst_ && completed_) ? std::chrono::duration<double>(lastDone_ - firstArrival_).count() : 0.0;
    if (reset) {
        latUs_.clear();
        submitted_ = completed_ = failed_ = batches_ = batched_ = maxBatchSeen_ = 0;
        haveFirst_ = false;
    }
    return s;
}

void Server::work(Lane& lane) {
    if (cudaSetDevice(device_) != cudaSuccess) return;
    for (;;) {
        std::vector<Request> batch;
        {
            std::unique_lock<std::mutex> g(mu_);
            cvWork_.wait(g, [&] { return stopping_ || !lane.pending.empty(); });
            if (lane.pending.empty()) return;  // stopping and drained
            const size_t n = std::min<size_t>(lane.cap, lane.pending.size());
            batch.reserve(n);
            for (size_t i = 0; i < n; ++i) {
                batch.push_back(std::move(lane.pending.front()));
                lane.pending.pop_front();
            }
            ++batches_;
            batched_ += n;
            maxBatchSeen_ = std::max<uint64_t>(maxBatchSeen_, n);
        }
        // One lane serving both kinds runs consecutive runs of one kind as one batch each.
        size_t b = 0;
        while (b < batch.size()) {
            size_t e = b + 1;
            while (e < batch.size() && batch[e].qtype == batch[b].qtype) ++e;
            runGroup(lane, batch, b, e);
            b = e;
        }
        // Admission by memory: the engine's workspace was sized by the largest batch so far, so
        // scale that batch size by budget / workspace to get the slots the next batch may take.
        lane.maxN = std::max<uint64_t>(lane.maxN, batch.size());
        const uint64_t ws = std::max<uint64_t>(1, lane.engine->workspaceBytes());
        const double fit = static_cast<double>(lane.maxN) * static_cast<double>(cfg_.memoryBudget) / static_cast<double>(ws);
        lane.cap = static_cast<uint32_t>(std::max(1.0, std::min(static_cast<double>(cfg_.maxBatch), fit)));
    }
}

void Server::runGroup(Lane& lane, std::vector<Request>& batch, size_t begin, size_t end) {
    const size_t n = end - begin;
    const int qtype = batch[begin].qtype;
    const size_t row = (qtype == kQtypeRange) ? 2 * D_ : D_;
    std::vector<uint64_t> offs, ids;
    std::vector<double> d2;
    std::vector<uint32_t> lv;
    const unsigned flags = cfg_.levels ? kWantLevels : 0u;
    try {
        std::vector<double> hq(n * row);
        std::vector<uint32_t> hk(n);
        uint64_t sumK = 0;
        for (size_t i = 0; i < n; ++i) {
            std::copy(batch[begin + i].q.begin(), batch[begin + i].q.end(), hq.begin() + i * row);
            hk[i] = batch[begin + i].K;
            sumK += hk[i];
        }
        if (lane.dq.bytes() < hq.size() * 8) lane.dq.alloc(hq.size() * 8);
        TBLAEQ_CUDA(cudaMemcpyAsync(lane.dq.get(), hq.data(), hq.size() * 8, cudaMemcpyHostToDevice, lane.stream));
        BatchOutput o;
        if (qtype == kQtypeRange) {
            o = lane.engine->runRange(lane.dq.as<double>(), static_cast<uint32_t>(n), cfg_.mode, flags);
        } else {
            if (lane.dk.bytes() < n * 4) lane.dk.alloc(n * 4);
            TBLAEQ_CUDA(cudaMemcpyAsync(lane.dk.get(), hk.data(), n * 4, cudaMemcpyHostToDevice, lane.stream));
            try {
                o = lane.engine->runKnn(lane.dq.as<double>(), static_cast<uint32_t>(n), lane.dk.as<uint32_t>(), sumK,
                                        flags);
            } catch (const SplitBatch&) {
                if (n == 1) throw;
                const size_t mid = begin + n / 2;
                runGroup(lane, batch, begin, mid);
                runGroup(lane, batch, mid, end);
                return;
            }
        }
        offs.resize(n + 1);
        TBLAEQ_CUDA(cudaMemcpyAsync(offs.data(), o.offsets, (n + 1) * 8, cudaMemcpyDeviceToHost, lane.stream));
        TBLAEQ_CUDA(cudaStreamSynchronize(lane.stream));
        ids.resize(offs[n]);
        if (offs[n]) TBLAEQ_CUDA(cudaMemcpyAsync(ids.data(), o.ids, offs[n] * 8, cudaMemcpyDeviceToHost, lane.stream));
        if (qtype == kQtypePoint && offs[n]) {
            d2.resize(offs[n]);
            TBLAEQ_CUDA(cudaMemcpyAsync(d2.data(), o.dist2, offs[n] * 8, cudaMemcpyDeviceToHost, lane.stream));
        }
        if (o.levelItems) {  // [l * n + q]
            lv.resize(rt_.dev->intervals * n);
            TBLAEQ_CUDA(cudaMemcpyAsync(lv.data(), o.levelItems, lv.size() * 4, cudaMemcpyDeviceToHost, lane.stream));
        }
        TBLAEQ_CUDA(cudaStreamSynchronize(lane.stream));
    } catch (const CudaError& e) {
        post(batch, begin, end, lv, offs, ids, d2, e.code == cudaErrorMemoryAllocation ? 4 : 3, e.what());
        return;
    } catch (const std::exception& e) {
        post(batch, begin, end, lv, offs, ids, d2, 3, e.what());
        return;
    }
    post(batch, begin, end, lv, offs, ids, d2, 0, "");
}

void Server::post(std::vector<Request>& batch, size_t begin, size_t end, const std::vector<uint32_t>& levels,
                  const std::vector<uint64_t>& offs,
                  const std::vector<uint64_t>& ids, const std::vector<double>& d2, int status,
                  const std::string& err) {
    const Clock::time_point now = Clock::now();
    {
        std::lock_guard<std::mutex> g(mu_);
        for (size_t i = begin; i < end; ++i) {
            Result r;
            r.status = status;
            r.error = err;
            if (status == 0) {
                const size_t q = i - begin;
                r.ids.assign(ids.begin() + static_cast<ptrdiff_t>(offs[q]), ids.begin() + static_cast<ptrdiff_t>(offs[q + 1]));
                if (!d2.empty())
                    r.dist2.assign(d2.begin() + static_cast<ptrdiff_t>(offs[q]), d2.begin() + static_cast<ptrdiff_t>(offs[q + 1]));
                const size_t n = end - begin, L = n ? levels.size() / n : 0;
                for (size_t l = 0; l < L; ++l) r.levels.push_back(levels[l * n + q]);
            }
            r.latencyUs = std::chrono::duration<double, std::micro>(now - batch[i].arrival).count();
            latUs_.push_back(r.latencyUs);
            if (status == 0) {
                ++completed_;
            } else {
                ++failed_;
            }
            inFlight_.erase(batch[i].ticket);
            done_[batch[i].ticket] = std::move(r);
        }
        lastDone_ = now;
    }
    cvDone_.notify_all();
}

}  // namespace tblaeq
