// C++ host facade: QueryHandler, PolicyScheduler and the B200 per-level strategy.
#include "handler.hpp"

#include "knn.cuh"

#include <algorithm>
#include <iomanip>
#include <iostream>
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

LevelResult B200Strategy::runLevel(size_t l, const Grid& cur, QueryType qType, const double* lo, const double* hi,
                                   const double* queryPoint, size_t K) {
    const HostIndex& h = *rt_.host;
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
    r.grid.numRows = h.meshCount(l + 1);
    r.grid.dim = D;
    r.grid.nnz = n;
    r.grid.ids = out.ids.as<uint64_t>();
    r.grid.vals = out.vals.as<double>();
    return r;
}

}  // namespace tblaeq
