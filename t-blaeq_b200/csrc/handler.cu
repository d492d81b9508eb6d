// C++ host facade: QueryHandler, PolicyScheduler and the B200 per-level strategy.
#include "handler.hpp"

#include "knn.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <stdexcept>

namespace tblaeq {

const char* levelPolicyName(LevelPolicy p) {
    switch (p) {
        case LevelPolicy::L0: return "L0";
        case LevelPolicy::L1: return "L1";
        case LevelPolicy::L2: return "L2";
        case LevelPolicy::L3: return "L3";
    }
    return "?";
}

LevelPolicy IndexPolicy::parseLevel(const std::string& s) {
    if (s == "L0" || s == "l0") return LevelPolicy::L0;
    if (s == "L1" || s == "l1") return LevelPolicy::L1;
    if (s == "L2" || s == "l2") return LevelPolicy::L2;
    if (s == "L3" || s == "l3") return LevelPolicy::L3;
    throw std::invalid_argument("Unknown policy level '" + s + "'. Valid values: L0, L1, L2, L3.");
}

MemoryStats computeStats(const HostIndex& idx) {
    MemoryStats s;
    for (const auto& t : idx.pTensors)
        s.hostPTensors += t.nnz * t.D * 8 + t.cols * 8 + (t.cols + 1) * 8 + t.nnz * 8;
    for (uint64_t m = 1; m < idx.height; ++m)
        if (!idx.maps[m].empty()) s.hostMaps += idx.meshSizes[idx.intervals - m] * 8;
    for (uint64_t i = 0; i < idx.intervals; ++i) s.hostRadius += idx.meshSizes[idx.intervals - i] * 8;
    s.hostCoarsestMesh = idx.coarsest.nnz * 8 + idx.coarsest.nnz * idx.coarsest.dim * 8;
    s.hostTotal = s.hostPTensors + s.hostMaps + s.hostRadius + s.hostCoarsestMesh;
    for (const auto& t : idx.pTensors) s.devicePTensorVals += t.nnz * t.D * 8;
    s.deviceMaps = s.hostMaps;
    s.deviceRadius = s.hostRadius;
    s.deviceCoarsestMesh = s.hostCoarsestMesh;
    for (const auto& t : idx.pTensors) s.deviceSpTSpMBufs += 3 * t.rows * 8;
    s.deviceTotal = s.devicePTensorVals + s.deviceMaps + s.deviceRadius + s.deviceCoarsestMesh;
    s.grandTotal = s.hostTotal + s.deviceTotal;
    return s;
}

IndexPolicy PolicyScheduler::recommend(const HostIndex& idx, uint64_t freeBytes) {
    const MemoryStats st = computeStats(idx);
    uint64_t budget = static_cast<uint64_t>(static_cast<double>(freeBytes) * kSafetyFactor);
    const uint64_t permanent = st.deviceCoarsestMesh + st.deviceMaps;
    IndexPolicy policy;
    if (budget <= permanent) {
        policy.levels.assign(idx.intervals, LevelPolicy::L3);
        return policy;
    }
    budget -= permanent;
    policy.levels.resize(idx.intervals);
    for (uint64_t l = 0; l < idx.intervals; ++l) {
        const uint64_t nnz = idx.pTensors[l].nnz, col = idx.pTensors[l].cols, D = idx.D;
        const uint64_t pVals = nnz * D * 8, radius = col * 8, spBuf = 3 * nnz * 8;
        const uint64_t costL0 = pVals + radius + spBuf + pVals;
        const uint64_t costL1 = pVals + radius + spBuf + pVals;
        const uint64_t costL2 = 2 * pVals + spBuf;
        if (budget >= costL0) {
            policy.levels[l] = LevelPolicy::L0;
            budget -= costL0;
        } else if (budget >= costL1) {
            policy.levels[l] = LevelPolicy::L1;
            budget -= costL1;
        } else if (budget >= costL2) {
            policy.levels[l] = LevelPolicy::L2;
        } else {
            policy.levels[l] = LevelPolicy::L3;
        }
    }
    return policy;
}

Runtime::~Runtime() {
    scorer.reset();
    invMapFinest.release();
    parentFinest.release();
    engine.reset();
    pluginEngine.reset();
    levelOut.clear();
    pluginMask.release();
    knnKeys.release();
    knnKeys2.release();
    knnLabels.release();
    knnLabels2.release();
    knnCnt.release();
    knnRr.release();
    scratchQuery.release();
    dev.reset();
    if (stream) cudaStreamDestroy(stream);
}

QueryHandler::QueryHandler(const std::string& indexPath, bool loadFromIndex) {
    if (!loadFromIndex) throw std::invalid_argument("Use QueryHandler(datasetPath) to build a new index.");
    host_ = std::make_unique<HostIndex>(loadIndex(indexPath));
}

QueryHandler::QueryHandler(const GenParams& gen) { host_ = std::make_unique<HostIndex>(generateRandomIndex(gen)); }

QueryHandler::QueryHandler(HostIndex&& built) { host_ = std::make_unique<HostIndex>(std::move(built)); }

QueryHandler::~QueryHandler() = default;

void QueryHandler::saveIndex(const std::string& dirPath) const { tblaeq::saveIndex(*host_, dirPath); }

Runtime& QueryHandler::runtime() {
    if (!prepared_) prepareForQuery();
    return *rt_;
}

void QueryHandler::prepareForQuery() {
    if (prepared_) return;
    size_t freeB = 0, totalB = 0;
    TBLAEQ_CUDA(cudaMemGetInfo(&freeB, &totalB));
    prepareForQuery(PolicyScheduler::recommend(*host_, freeB));
}

void QueryHandler::prepareForQuery(LevelPolicy level) {
    if (prepared_) return;
    prepareForQuery(IndexPolicy::uniform(host_->intervals, level));
}

void QueryHandler::prepareForQuery(const IndexPolicy& policy) {
    if (prepared_) return;
    if (policy.levels.size() != host_->intervals)
        throw std::invalid_argument("prepareForQuery: policy must name one level policy per interval");
    policy_ = policy;
    auto rt = std::make_unique<Runtime>();
    rt->host = host_.get();
    TBLAEQ_CUDA(cudaStreamCreateWithFlags(&rt->stream, cudaStreamNonBlocking));
    const DerivedArrays der = computeDerived(*host_);
    std::vector<int> residency(host_->intervals, kResident);
    for (size_t l = 0; l < residency.size(); ++l) {
        if (policy.levels[l] == LevelPolicy::L2) residency[l] = kRowsOnHost;
        if (policy.levels[l] == LevelPolicy::L3) residency[l] = kRowsAndMapOnHost;
    }
    rt->dev = buildDeviceIndex(*host_, der, rt->stream, residency);
    rt->engine = std::make_unique<BatchEngine>(*rt->dev, rt->stream);
    rt->pluginEngine = std::make_unique<BatchEngine>(*rt->dev, rt->stream);
    rt->levelOut.resize(host_->intervals);
    rt->scratchQuery.alloc(2 * host_->D * 8);
    rt_ = std::move(rt);
    prepared_ = true;
}

void B200Strategy::prepare(std::ostream& reportOs) {
    size_t streamed = 0;
    for (uint8_t o : rt_.dev->rowsOnHost) streamed += o;
    reportOs << "B200 strategy: " << rt_.dev->deviceBytes() << " bytes on the device; " << streamed
             << " interval(s) read from mapped host memory\n";
}

LevelResult B200Strategy::runLevel(size_t l, SparseGrid* curGrid, QueryType qType, const double* lo, const double* hi,
                                   const double* queryPoint, size_t K) {
    const HostIndex& h = *rt_.host;
    if (!curGrid) throw std::invalid_argument("runLevel: null grid");
    const SparseGrid& cur = *curGrid;
    if (l >= h.intervals) throw std::out_of_range("runLevel: level out of range");
    if (cur.dim != h.D) throw std::invalid_argument("runLevel: grid dimension mismatch");
    const uint64_t D = h.D;
    auto& out = rt_.levelOut[l];
    const uint64_t cap = h.meshCount(l + 1);
    if (out.cap < cap) {
        out.ids.alloc(std::max<uint64_t>(cap, 1) * 8);
        out.vals.alloc(std::max<uint64_t>(cap, 1) * D * 8);
        out.cap = cap;
    }
    uint64_t n = 0;
    if (qType == QueryType::RANGE) {
        TBLAEQ_CUDA(cudaMemcpyAsync(rt_.scratchQuery.as<double>(), lo, D * 8, cudaMemcpyHostToDevice, rt_.stream));
        TBLAEQ_CUDA(cudaMemcpyAsync(rt_.scratchQuery.as<double>() + D, hi, D * 8, cudaMemcpyHostToDevice, rt_.stream));
        n = rt_.pluginEngine->runGridLevel(static_cast<int>(l), cur.ids, cur.vals, cur.nnz, true,
                                           rt_.scratchQuery.as<double>(), nullptr, out.ids.as<uint64_t>(),
                                           out.vals.as<double>(), cap);
    } else {
        // The reference's KNN level: lower bounds, sort, STEP -> mask, then the same expansion.
        const uint64_t p = cur.nnz;
        if (p > 0) {
            if (rt_.knnCap < p) {
                rt_.knnKeys.alloc(p * 8);
                rt_.knnKeys2.alloc(p * 8);
                rt_.knnLabels.alloc(p * 4);
                rt_.knnLabels2.alloc(p * 4);
                rt_.knnCnt.alloc(p * 4);
                rt_.knnRr.alloc(p * 8);
                rt_.pluginMask.alloc(p);
                rt_.knnCap = p;
            }
            TBLAEQ_CUDA(cudaMemcpyAsync(rt_.scratchQuery.as<double>(), queryPoint, D * 8, cudaMemcpyHostToDevice,
                                        rt_.stream));
            TBLAEQ_CUDA(cudaMemsetAsync(rt_.pluginMask.get(), 0, p, rt_.stream));
            launchKnnLowerBound(cur.ids, cur.vals, p, static_cast<int>(D), rt_.scratchQuery.as<double>(),
                                rt_.dev->nodeOrig[l].as<NodeRec>(), rt_.knnKeys.as<uint64_t>(),
                                rt_.knnLabels.as<uint32_t>(), rt_.knnCnt.as<uint32_t>(), rt_.knnRr.as<double>(),
                                rt_.stream);
            sortPairs(rt_.knnKeys.as<uint64_t>(), rt_.knnLabels.as<uint32_t>(), rt_.knnKeys2.as<uint64_t>(),
                      rt_.knnLabels2.as<uint32_t>(), p, rt_.stream);
            launchStep(rt_.knnKeys.as<uint64_t>(), rt_.knnLabels.as<uint32_t>(), rt_.knnCnt.as<uint32_t>(),
                       rt_.knnRr.as<double>(), p, K, rt_.pluginMask.as<uint8_t>(), rt_.stream);
        }
        n = rt_.pluginEngine->runGridLevel(static_cast<int>(l), cur.ids, cur.vals, p, false, nullptr,
                                           rt_.pluginMask.as<uint8_t>(), out.ids.as<uint64_t>(),
                                           out.vals.as<double>(), cap);
    }
    LevelResult r;
    r.grid = new SparseGrid{h.meshCount(l + 1), D, n, out.ids.as<uint64_t>(), out.vals.as<double>()};
    return r;
}

// ---- the reference's query API on the facade -------------------------------------------------------

Query loadQueryFile(const std::string& path, QueryType type) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("Cannot open query file: " + path);
    Query q;
    q.type = type;
    long long n = -1, d = -1;
    if (!(in >> n >> d) || n < 0 || d <= 0) throw std::runtime_error("Invalid query file header: " + path);
    q.length = static_cast<size_t>(n);
    q.dim = static_cast<size_t>(d);
    const size_t per = (type == QueryType::RANGE ? 2 : 1) * q.dim;
    q.data.resize(q.length * per);
    for (size_t i = 0; i < q.data.size(); ++i)
        if (!(in >> q.data[i]))
            throw std::runtime_error("Query file ended after " + std::to_string(i / per) + " of " +
                                     std::to_string(q.length) + " rows: " + path);
    return q;
}

LevelResult QueryEngine::runSingleQuery(QueryHandler& qh, QueryType qType, const double* lo, const double* hi,
                                        const double* queryPoint, size_t K, size_t* levelFineMeshSize) {
    Runtime& rt = qh.runtime();
    const HostIndex& h = *rt.host;
    // The coarsest mesh as the first grid (QueryEngine.cu:66-70), device-resident.
    SparseGrid coarsest{h.coarsest.rows, h.D, h.coarsest.nnz, rt.dev->coarseIds.as<uint64_t>(),
                        rt.dev->coarseVals.as<double>()};
    B200Strategy strategy(rt);
    SparseGrid* cur = &coarsest;
    LevelResult last{};
    for (size_t l = 0; l < h.intervals; ++l) {
        LevelResult r = strategy.runLevel(l, cur, qType, lo, hi, queryPoint, K);
        if (levelFineMeshSize) levelFineMeshSize[l] = r.grid->nnz;
        if (cur != &coarsest) delete cur;  // the strategy keeps the buffers (ownsIds = ownsVals = false)
        cur = r.grid;
        last = r;
    }
    return last;
}

namespace {
double rangeLogVolume(const double* lo, const double* hi, size_t D) {
    double v = 0.0;
    for (size_t i = 0; i < D; ++i) {
        const double s = hi[i] - lo[i];
        if (s <= 0.0) return -std::numeric_limits<double>::infinity();
        v += std::log(s);
    }
    return v;
}
}  // namespace

QueryResult QueryEngine::run(QueryHandler& qh, const Query& q, const RunConfig& cfg) {
    if (!qh.prepared()) throw std::logic_error("call prepareForQuery before querying");
    Runtime& rt = qh.runtime();
    const HostIndex& h = *rt.host;
    if (q.dim != h.D) throw std::invalid_argument("query dimension does not match the index");
    QueryResult res;
    res.type = q.type;
    res.datasetName = h.datasetName;
    res.datasetSize = h.N;
    res.datasetDim = h.D;
    res.queryParam = q.type == QueryType::POINT ? "K=" + std::to_string(cfg.K) : "";
    for (size_t l = 0; l < h.intervals; ++l) res.levelOriginalSize.push_back(h.meshCount(l + 1));
    const size_t count = std::min(q.length, cfg.maxQueryCount);
    const bool range = q.type == QueryType::RANGE;
    long totalUs = 0, maxUs = 0, minUs = std::numeric_limits<long>::max();
    std::vector<double> row(2 * h.D);
    for (size_t i = 0; i < count; ++i) {
        const double* lo = range ? q.getQueryLo(i) : nullptr;
        const double* hi = range ? q.getQueryHi(i) : nullptr;
        const double* pt = range ? nullptr : q.getQueryPoint(i);
        std::vector<size_t> lv(h.intervals, 0);
        std::vector<uint64_t> ids;
        std::vector<double> d2;
        const auto t0 = std::chrono::steady_clock::now();
        size_t n = 0;
        if (qh.mode() == kModeRefParity) {
            LevelResult r = runSingleQuery(qh, q.type, lo, hi, pt, cfg.K, lv.data());
            n = r.grid->nnz;
            if (cfg.saveFineMesh && n) {
                ids.resize(n);
                TBLAEQ_CUDA(cudaMemcpyAsync(ids.data(), r.grid->ids, n * 8, cudaMemcpyDeviceToHost, rt.stream));
                TBLAEQ_CUDA(cudaStreamSynchronize(rt.stream));
            }
            delete r.grid;
        } else {
            // Exact answers: the batched engine with one query (its own per-level counts).
            const size_t w = range ? 2 * h.D : h.D;
            std::copy(range ? lo : pt, (range ? lo : pt) + w, row.begin());
            TBLAEQ_CUDA(cudaMemcpyAsync(rt.scratchQuery.get(), row.data(), w * 8, cudaMemcpyHostToDevice, rt.stream));
            BatchOutput o;
            if (range) {
                o = rt.engine->runRange(rt.scratchQuery.as<double>(), 1, kModeExact, kWantLevels);
            } else {
                const uint32_t k32 = static_cast<uint32_t>(cfg.K);
                TBLAEQ_CUDA(cudaMemcpyAsync(rt.scratchQuery.as<double>() + h.D, &k32, 4, cudaMemcpyHostToDevice,
                                            rt.stream));
                o = rt.engine->runKnn(rt.scratchQuery.as<double>(), 1,
                                      reinterpret_cast<const uint32_t*>(rt.scratchQuery.as<double>() + h.D), cfg.K,
                                      kWantLevels);
            }
            n = o.total;
            std::vector<uint32_t> items(h.intervals);
            TBLAEQ_CUDA(cudaMemcpyAsync(items.data(), o.levelItems, h.intervals * 4, cudaMemcpyDeviceToHost, rt.stream));
            if (cfg.saveFineMesh && n) {
                ids.resize(n);
                TBLAEQ_CUDA(cudaMemcpyAsync(ids.data(), o.ids, n * 8, cudaMemcpyDeviceToHost, rt.stream));
                if (o.dist2) {
                    d2.resize(n);
                    TBLAEQ_CUDA(cudaMemcpyAsync(d2.data(), o.dist2, n * 8, cudaMemcpyDeviceToHost, rt.stream));
                }
            }
            TBLAEQ_CUDA(cudaStreamSynchronize(rt.stream));
            for (size_t l = 0; l < h.intervals; ++l) lv[l] = items[l];
        }
        const long us = std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0)
                            .count();
        maxUs = std::max(maxUs, us);
        minUs = std::min(minUs, us);
        totalUs += us;
        res.queryTimeUs.push_back(us);
        res.levelFineMeshSize.push_back(std::move(lv));
        res.fineMeshSize.push_back(n);
        res.queryRangeVolume.push_back(range ? rangeLogVolume(lo, hi, h.D) : 1.0);
        if (cfg.saveFineMesh) {
            res.ids.push_back(std::move(ids));
            res.dist2.push_back(std::move(d2));
        }
    }
    long cnt = static_cast<long>(count);
    if (cnt > 2) {  // the reference drops the fastest and the slowest query (QueryEngine.cu:216-220)
        totalUs -= maxUs + minUs;
        cnt -= 2;
    }
    res.totalTimeUs = totalUs;
    res.queryCount = static_cast<size_t>(cnt);
    for (size_t l = 0; l < h.intervals; ++l) {
        if (l) res.memoryPolicy += "-";
        res.memoryPolicy += levelPolicyName(qh.activePolicy().levels[l]);
    }
    return res;
}

QueryResult QueryHandler::performQuery(const std::string& path, QueryType type, bool saveFineMesh,
                                       size_t maxQueryCount, size_t K) {
    Query q = loadQueryFile(path, type);
    RunConfig cfg;
    cfg.maxQueryCount = maxQueryCount;
    cfg.K = K;
    cfg.saveFineMesh = saveFineMesh;
    return QueryEngine::run(*this, q, cfg);
}

QueryResult QueryHandler::performSingleKNNQuery(const std::vector<double>& point, size_t K, bool saveFineMesh) {
    Query q;
    q.type = QueryType::POINT;
    q.length = 1;
    q.dim = point.size();
    q.data = point;
    RunConfig cfg;
    cfg.K = K;
    cfg.saveFineMesh = saveFineMesh;
    return QueryEngine::run(*this, q, cfg);
}

QueryResult QueryHandler::performSingleRangeQuery(const std::vector<double>& upper, const std::vector<double>& lower,
                                                  bool saveFineMesh) {
    if (upper.size() != lower.size()) throw std::invalid_argument("range bounds of different dimensions");
    Query q;
    q.type = QueryType::RANGE;
    q.length = 1;
    q.dim = lower.size();
    q.data = lower;
    q.data.insert(q.data.end(), upper.begin(), upper.end());
    RunConfig cfg;
    cfg.saveFineMesh = saveFineMesh;
    QueryResult r = QueryEngine::run(*this, q, cfg);
    r.queryParam = "single-range-query";
    return r;
}

}  // namespace tblaeq
