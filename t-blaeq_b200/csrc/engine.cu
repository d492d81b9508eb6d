// Batched traversal engine (range queries; see engine.hpp).
#include "engine.hpp"

#include <exception>
#include <limits>

#include "knn.cuh"

#include <algorithm>

namespace tblaeq {

namespace {
// Resets the engine's workspace when the scope it guards exits by an exception.
class WorkspaceGuard {
public:
    explicit WorkspaceGuard(BatchEngine& e) : e_(e), n_(std::uncaught_exceptions()) {}
    ~WorkspaceGuard() {
        if (std::uncaught_exceptions() > n_) e_.resetWorkspace();
    }
    WorkspaceGuard(const WorkspaceGuard&) = delete;
    WorkspaceGuard& operator=(const WorkspaceGuard&) = delete;

private:
    BatchEngine& e_;
    int n_;
};
}  // namespace

void BatchEngine::resetWorkspace() noexcept {
    dropGraph();
    for (auto& f : f_)
        for (DeviceMem* m : {&f.q, &f.node, &f.cbeg, &f.cpre, &f.x, &f.tileStart}) m->release();
    for (DeviceMem* m : {&nmNodeOff_, &nmUnitOff_, &nmUnitNode_, &nmList_, &rawIds_, &rawQ_, &rawVals_, &pairQ_[0], &pairQ_[1],
                         &pairNode_[0], &pairNode_[1], &pairList_, &pairNodeOff_, &pairUnitOff_, &pairUnitNode_, &candQ_, &candId_,
                         &candD2_, &excl_, &probeK_, &resIds_, &resVals_, &resQ_, &resDist_, &zeroBlock_, &cmpCnt_,
                         &cmpKids_, &cmpEntryOff_, &cmpKidOff_, &offsets_, &boxF_, &tau_, &candOff_, &knnCount_,
                         &knnOff_, &knnIds_, &knnD2_, &lbE_, &scoreE_, &sel_, &offF_, &waveM_, &selCount_, &selOff_,
                         &selIds_, &selD2_, &candOffB_, &candOffS_, &resIdsB_, &resQB_, &resDistB_})
        m->release();
    caps_ = EngineCaps{};
    qcap_ = 0;
    haveVals_ = false;
    nmEntryCap_ = nmResultCap_ = 0;
    nmVals_ = false;
    pairCap_ = candCap_ = 0;
    knnCap_ = 0;
    entryCap_ = resCapB_ = 0;
    knnQcap_ = 0;
    tileCap_ = 0;
    zeroBytes_ = 0;
}


namespace {
size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
}  // namespace

BatchEngine::BatchEngine(const DeviceIndex& di, cudaStream_t stream)
    : di_(di), stream_(stream), tile_(expandTile(static_cast<int>(di.D))),
      variants_(static_cast<size_t>(di.height), kVariantDirect), grids_(static_cast<size_t>(di.height), 100) {}

void BatchEngine::setLaunchShapes(const std::vector<int>& v, const std::vector<int>& g) {
    if (g.size() != grids_.size()) throw std::invalid_argument("setLaunchShapes: one grid percentage per expand launch");
    for (int x : g)
        if (x < 1 || x > 100) throw std::invalid_argument("setLaunchShapes: grid percentage must be in [1, 100]");
    setVariants(v);
    if (g != grids_) dropGraph();
    grids_ = g;
}

void BatchEngine::setVariants(const std::vector<int>& v) {
    if (v.size() != variants_.size()) throw std::invalid_argument("setVariants: one variant per expand launch");
    for (int x : v)
        if (x != kVariantDirect && x != kVariantStaged && x != kVariantNodeMajor)
            throw std::invalid_argument("setVariants: unknown variant");
    if (v != variants_) dropGraph();
    variants_ = v;
}

std::vector<float> BatchEngine::autotuneRange(const double* dBoxes, uint32_t nq, int mode, unsigned flags, int reps) {
    WorkspaceGuard guard(*this);
    const int H = static_cast<int>(di_.height);
    const bool wasTiming = timing_;
    setTiming(true);
    runRange(dBoxes, nq, mode, flags & ~kUseGraph);  // sizes the workspace
    struct Shape {
        int variant, grid;
    };
    std::vector<Shape> candidates;
    const bool nm = useNodeMajor(mode);
    for (int v : {kVariantDirect, kVariantStaged, kVariantNodeMajor}) {
        if (v == kVariantNodeMajor && !nm) continue;
        for (int g : {100, 75, 50, 25}) candidates.push_back({v, g});
    }
    std::vector<std::vector<float>> med(candidates.size(), std::vector<float>(H, 0.f));
    for (size_t c = 0; c < candidates.size(); ++c) {
        setLaunchShapes(std::vector<int>(H, candidates[c].variant), std::vector<int>(H, candidates[c].grid));
        enqueueRange(dBoxes, nq, mode, flags & ~kUseGraph);
        status();
        std::vector<std::vector<float>> samples(H);
        for (int r = 0; r < std::max(1, reps); ++r) {
            enqueueRange(dBoxes, nq, mode, flags & ~kUseGraph);
            if (status() != 0) throw CudaError(cudaErrorLaunchFailure, "autotune batch reported a device status");
            const std::vector<float> t = stageTimes();
            for (int m = 0; m < H; ++m) samples[m].push_back(t[1 + m]);
        }
        for (int m = 0; m < H; ++m) {
            std::sort(samples[m].begin(), samples[m].end());
            med[c][m] = samples[m][samples[m].size() / 2];
        }
    }
    std::vector<int> best(H, kVariantDirect), bestG(H, 100);
    std::vector<float> bestT(H, 0.f);
    for (int m = 0; m < H; ++m) {
        size_t bi = 0;
        for (size_t c = 1; c < candidates.size(); ++c)
            if (med[c][m] < med[bi][m]) bi = c;
        best[m] = candidates[bi].variant;
        bestG[m] = candidates[bi].grid;
        bestT[m] = med[bi][m];
    }
    setLaunchShapes(best, bestG);
    setTiming(wasTiming);
    return bestT;
}

BatchEngine::~BatchEngine() {
    dropGraph();
    for (cudaEvent_t e : events_) cudaEventDestroy(e);
}

void BatchEngine::dropGraph() {
    if (graphExec_) cudaGraphExecDestroy(graphExec_);
    graphExec_ = nullptr;
    graphKey_ = GraphKey{};
}

void BatchEngine::record(int i) {
    // Inside stream capture an event must become an external event-record node to stay usable
    // for cudaEventElapsedTime after the graph replays.
    if (capturing_) {
        TBLAEQ_CUDA(cudaEventRecordWithFlags(events_[i], stream_, cudaEventRecordExternal));
    } else {
        TBLAEQ_CUDA(cudaEventRecord(events_[i], stream_));
    }
}

void BatchEngine::setTiming(bool on) {
    timing_ = on;
    if (on && events_.empty()) {
        events_.resize(static_cast<size_t>(di_.height) + 3);
        for (auto& e : events_) TBLAEQ_CUDA(cudaEventCreate(&e));
    }
}

std::vector<float> BatchEngine::stageTimes() {
    std::vector<float> t;
    if (!timing_ || events_.empty()) return t;
    TBLAEQ_CUDA(cudaEventSynchronize(events_.back()));
    for (size_t i = 0; i + 1 < events_.size(); ++i) {
        float ms = 0.f;
        TBLAEQ_CUDA(cudaEventElapsedTime(&ms, events_[i], events_[i + 1]));
        t.push_back(ms);
    }
    return t;
}

void BatchEngine::levelCounts(std::vector<uint64_t>& entries, std::vector<uint64_t>& items, uint64_t& results) {
    const int H = static_cast<int>(di_.height);
    std::vector<uint32_t> h((H + 2) * 2);
    TBLAEQ_CUDA(cudaMemcpyAsync(h.data(), hdrPtr(0), h.size() * 4, cudaMemcpyDeviceToHost, stream_));
    TBLAEQ_CUDA(cudaStreamSynchronize(stream_));
    entries.clear();
    items.clear();
    for (int lv = 0; lv < H; ++lv) {
        entries.push_back(h[2 * lv]);
        items.push_back(h[2 * lv + 1]);
    }
    results = h[2 * H];
}

uint64_t BatchEngine::lastTotal(uint32_t nq) {
    uint64_t total = 0;
    const uint64_t* off = lastKnn_ ? knnOff_.as<uint64_t>() : offsets_.as<uint64_t>();
    TBLAEQ_CUDA(cudaMemcpyAsync(&total, off + nq, 8, cudaMemcpyDeviceToHost, stream_));
    TBLAEQ_CUDA(cudaStreamSynchronize(stream_));
    return total;
}

size_t BatchEngine::workspaceBytes() const {
    size_t t = zeroBlock_.bytes() + offsets_.bytes() + resIds_.bytes() + resVals_.bytes() + resQ_.bytes() +
               resDist_.bytes() + nmList_.bytes() + nmNodeOff_.bytes() + nmUnitOff_.bytes() + rawIds_.bytes() +
               rawQ_.bytes() + rawVals_.bytes();
    for (const auto& f : f_) t += f.q.bytes() + f.node.bytes() + f.cbeg.bytes() + f.cpre.bytes() + f.x.bytes() +
                                  f.tileStart.bytes();
    return t;
}

void BatchEngine::reserve(const EngineCaps& want, uint32_t nq, unsigned flags) {
    const uint64_t H = di_.height, D = di_.D;
    const bool wantVals = (flags & kWantVals) != 0;
    EngineCaps c = caps_;
    bool growF = false, growR = false, growZ = false;
    if (want.entries > c.entries || f_[0].q.bytes() == 0) {
        c.entries = std::max(c.entries, want.entries);
        growF = true;
    }
    // One root entry per query must fit as well.
    if (nq > c.entries) {
        c.entries = nq;
        growF = true;
    }
    if (want.items > c.items || f_[0].tileStart.bytes() == 0) {
        c.items = std::max(c.items, want.items);
        growF = true;
        growZ = true;
    }
    const uint64_t rootItems = static_cast<uint64_t>(nq) * di_.meshCount[0];
    if (rootItems > c.items) {
        c.items = rootItems;
        growF = true;
        growZ = true;
    }
    if (want.results > c.results || resIds_.bytes() == 0 || (wantVals && !haveVals_)) {
        c.results = std::max(c.results, want.results);
        growR = true;
    }
    if (nq > qcap_ || zeroBlock_.bytes() == 0) growZ = true;
    if (c.entries > 0xffffffffull || c.items > 0xffffffffull || c.results > 0xffffffffull)
        throw SplitBatch("batch exceeds 32-bit traversal capacities; split the batch");
    // Frontier and result buffers that would not fit in device memory (beside what this engine
    // already holds and will release) also call for a smaller batch, not an allocation failure.
    {
        const uint64_t needF = growF ? 2 * (c.entries * (16 + 8 * D) + (c.items / tile_ + 2) * 4) : 0;
        const uint64_t needR = growR ? c.results * (20 + ((wantVals || haveVals_) ? 8 * D : 0)) : 0;
        size_t freeB = 0, totalB = 0;
        TBLAEQ_CUDA(cudaMemGetInfo(&freeB, &totalB));
        const uint64_t held = workspaceBytes(), margin = 512ull << 20;
        if (needF + needR > freeB + held && needF + needR > margin)
            throw SplitBatch("batch workspace (" + std::to_string((needF + needR) >> 20) +
                             " MiB) exceeds free device memory; split the batch");
    }
    if (growF || growR || growZ) dropGraph();  // captured launches hold the old buffer addresses

    if (growF) {
        const uint64_t tileCap = c.items / tile_ + 2;
        for (auto& f : f_) {
            f.q.alloc(c.entries * 4);
            f.node.alloc(c.entries * 4);
            f.cbeg.alloc(c.entries * 4);
            f.cpre.alloc(c.entries * 4);
            f.x.alloc(c.entries * D * 8);
            f.tileStart.alloc(tileCap * 4);
        }
        tileCap_ = tileCap;
    }
    if (growR) {
        resIds_.alloc(c.results * 8);
        resQ_.alloc(c.results * 4);
        resDist_.alloc(c.results * 8);
        if (wantVals || haveVals_) {
            resVals_.alloc(c.results * D * 8);
            haveVals_ = true;
        }
    }
    if (growZ) {
        qcap_ = std::max(qcap_, nq);
        size_t off = 0;
        offDesc_ = off;
        off = align256(off + (H + 1) * tileCap_ * 8);
        offTickets_ = off;
        off = align256(off + (H + 1) * 4);
        offStatus_ = off;
        off = align256(off + 4);
        offHdr_ = off;
        off = align256(off + (H + 4) * 2 * 4);  // levels 0..H-1, results, wave 2, compaction, point groups
        offQcount_ = off;
        off = align256(off + static_cast<size_t>(qcap_) * 4);
        offLevels_ = off;
        off = align256(off + static_cast<size_t>(di_.intervals) * qcap_ * 4);
        offQcountF_ = off;
        off = align256(off + static_cast<size_t>(qcap_) * 4);
        offQcountB_ = off;
        off = align256(off + static_cast<size_t>(qcap_) * 4);
        offWork_ = off;
        off = align256(off + 2 * 8);
        // Node-major range levels: a packed survivor counter (64 bits) and a unit ticket per level,
        // the per-node entry counts and cursors of every inner level, and the per-query result cursors.
        offNm_ = off;
        off = align256(off + H * 8 + H * 4);
        offNodeCnt_.assign(H, 0);
        for (uint64_t m = 1; m + 1 < H; ++m) {
            offNodeCnt_[m] = off;
            off = align256(off + 2 * di_.meshCount[m - 1] * 4);
        }
        offRcursor_ = off;
        off = align256(off + static_cast<size_t>(qcap_) * 4);
        // Node-major KNN completion: H+1 tickets, H pair counts and the candidate count; the probe's
        // per-level query counts; per-node counts and cursors of meshes 0..H-2; the per-query
        // candidate cursors.
        offKnnTick_ = off;
        // H+1 tickets, H pair counts, candidates, then a ticket and a candidate count per refine stage
        off = align256(off + (2 * H + 2 + 3 * kMaxRefineStages) * 4);  // ... and a filtered-pair count per stage
        offQcountP_ = off;
        off = align256(off + H * static_cast<size_t>(qcap_) * 4);
        offKnnNodeCnt_.assign(H, 0);
        for (uint64_t m = 0; m + 1 < H; ++m) {
            offKnnNodeCnt_[m] = off;
            off = align256(off + 2 * di_.meshCount[m] * 4);
        }
        offCandCursor_ = off;
        off = align256(off + static_cast<size_t>(qcap_) * 4);
        zeroBytes_ = off;
        zeroBlock_.alloc(zeroBytes_);
        offsets_.alloc((static_cast<size_t>(qcap_) + 1) * 8);
        boxF_.alloc(static_cast<size_t>(qcap_) * 4 * D * 4);  // rounded outward, then inward
    }
    caps_ = c;
}

uint32_t* BatchEngine::hdrPtr(int level) const {
    return reinterpret_cast<uint32_t*>(zeroBlock_.as<char>() + offHdr_) + 2 * level;
}

FrontierIn BatchEngine::inView(int b, uint32_t* hdr) const {
    const FrontierBufs& f = f_[b];
    return FrontierIn{f.q.as<uint32_t>(),         f.cbeg.as<uint32_t>(), f.cpre.as<uint32_t>(), f.x.as<double>(),
                      f.tileStart.as<uint32_t>(), hdr,                   static_cast<uint32_t>(caps_.entries),
                      static_cast<uint32_t>(tileCap_)};
}

FrontierOut BatchEngine::outView(int b, uint32_t* hdr) const {
    const FrontierBufs& f = f_[b];
    return FrontierOut{f.q.as<uint32_t>(),    f.node.as<uint32_t>(),     f.cbeg.as<uint32_t>(),
                       f.cpre.as<uint32_t>(), f.x.as<double>(),          f.tileStart.as<uint32_t>(),
                       hdr,                   static_cast<uint32_t>(caps_.entries), static_cast<uint32_t>(tileCap_)};
}

void BatchEngine::enqueueRange(const double* dBoxes, uint32_t nq, int mode, unsigned flags) {
    if (!(flags & kUseGraph)) {
        enqueueLaunches(dBoxes, nq, mode, flags);
        return;
    }
    const GraphKey key{dBoxes, nq, mode, flags & ~kUseGraph, timing_};
    if (!graphExec_ || !(key == graphKey_)) {
        dropGraph();
        cudaGraph_t g = nullptr;
        TBLAEQ_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        capturing_ = true;
        try {
            enqueueLaunches(dBoxes, nq, mode, flags);
            capturing_ = false;
        } catch (...) {
            capturing_ = false;
            cudaStreamEndCapture(stream_, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        TBLAEQ_CUDA(cudaStreamEndCapture(stream_, &g));
        size_t nNodes = 0;
        cudaGraphGetNodes(g, nullptr, &nNodes);
        std::vector<cudaGraphNode_t> nodes(nNodes);
        uint64_t nKernels = 0;
        if (nNodes && cudaGraphGetNodes(g, nodes.data(), &nNodes) == cudaSuccess) {
            for (size_t i = 0; i < nNodes; ++i) {
                cudaGraphNodeType t;
                if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++nKernels;
            }
        }
        const cudaError_t e = cudaGraphInstantiate(&graphExec_, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            graphExec_ = nullptr;
            throw CudaError(e, std::string("cudaGraphInstantiate failed: ") + cudaGetErrorString(e));
        }
        graphKey_ = key;
        graphKernels_ = nKernels;
        graphNodes_ = nNodes;
    }
    TBLAEQ_CUDA(cudaGraphLaunch(graphExec_, stream_));
}

bool BatchEngine::useNodeMajor(int mode) const {
    if (!nodeMajor_ || mode != kModeExact || di_.height < 2) return false;
    for (uint64_t m = 0; m + 1 < di_.height; ++m)
        if (!di_.aabb[m].bytes()) return false;
    return true;
}

void BatchEngine::reserveNodeMajor(unsigned flags) {
    const uint64_t D = di_.D;
    if (nmEntryCap_ < caps_.entries) {
        dropGraph();
        nmList_.alloc(caps_.entries * 4);
        uint64_t maxM = 1;
        for (uint64_t m = 0; m + 2 < di_.height; ++m) maxM = std::max<uint64_t>(maxM, di_.meshCount[m]);
        nmNodeOff_.alloc((maxM + 1) * 4);
        nmUnitOff_.alloc((maxM + 1) * 4);
        nmUnitNode_.alloc((caps_.entries / 32 + maxM + 2) * 4);  // units <= entries / 32 + nodes
        nmEntryCap_ = caps_.entries;
    }
    const bool vals = (flags & kWantVals) != 0;
    if (nmResultCap_ < caps_.results || (vals && !nmVals_)) {
        dropGraph();
        rawIds_.alloc(caps_.results * 8);
        rawQ_.alloc(caps_.results * 4);
        if (vals || nmVals_) {
            rawVals_.alloc(caps_.results * D * 8);
            nmVals_ = true;
        }
        nmResultCap_ = caps_.results;
    }
}

// Records of the children of level m (mesh m) in an exact range batch: the subtree radii with the
// children's own children, or, for the finest clusters when this batch tests point groups, with
// their groups.
const NodeRec* BatchEngine::innerRecords(int m) const {
    if (groupsThisBatch_ && m == static_cast<int>(di_.height) - 2) return di_.clusterGroups.as<NodeRec>();
    return di_.nodeSub[m].as<NodeRec>();
}

// Level m of an exact range batch, node-major: group frontier `buf` by node (m >= 1), test every
// node's children against the query boxes holding it, and append the survivors to the next frontier
// (1 - buf).
void BatchEngine::enqueueNodeMajorLevel(int m, int buf, const double* dBoxes, uint32_t nq, bool wantLevels) {
    const int D = static_cast<int>(di_.D);
    char* z = zeroBlock_.as<char>();
    auto* nmCounter = reinterpret_cast<unsigned long long*>(z + offNm_);
    auto* nmTicket = reinterpret_cast<uint32_t*>(z + offNm_ + di_.height * 8);
    auto* status = reinterpret_cast<uint32_t*>(z + offStatus_);
    const FrontierBufs& in = f_[buf];
    NodeMajorArgs n{};
    n.inQ = in.q.as<uint32_t>();
    n.inX = in.x.as<double>();
    n.inHdr = hdrPtr(m);
    n.inCap = static_cast<uint32_t>(caps_.entries);
    if (m == 0) {
        n.nNodes = 0;
        n.rootChildren = static_cast<uint32_t>(di_.meshCount[0]);
        // About 4,096 units (32 entries and a chunk of at least 4 of the root's children each).
        const uint64_t qUnits = (static_cast<uint64_t>(nq) + 31) / 32;
        const uint64_t maxChunks = std::max<uint64_t>(1, (n.rootChildren + 3) / 4);
        const uint64_t chunks = std::min<uint64_t>(maxChunks, std::max<uint64_t>(1, (4096 + qUnits - 1) / qUnits));
        n.rootChunk = static_cast<uint32_t>((n.rootChildren + chunks - 1) / chunks);
    } else {
        const uint32_t M = static_cast<uint32_t>(di_.meshCount[m - 1]);
        auto* nodeCnt = reinterpret_cast<uint32_t*>(z + offNodeCnt_[m]);
        launchNodeTranspose(in.node.as<uint32_t>(), hdrPtr(m), n.inCap, M, nodeCnt, nmNodeOff_.as<uint32_t>(),
                            nmUnitOff_.as<uint32_t>(), nodeCnt + M, nmList_.as<uint32_t>(), stream_,
                            nmUnitNode_.as<uint32_t>(), static_cast<uint32_t>(nmUnitNode_.bytes() / 4));
        n.list = nmList_.as<uint32_t>();
        n.nodeOff = nmNodeOff_.as<uint32_t>();
        n.unitOff = nmUnitOff_.as<uint32_t>();
        n.unitNode = nmUnitNode_.as<uint32_t>();
        n.nNodes = M;
        n.parents = di_.nodeSub[m - 1].as<NodeRec>();
    }
    n.rows = (m == 0) ? di_.coarseVals.as<double>() : di_.rows[m - 1];
    n.rowsOnHost = (m == 0) ? 0 : di_.rowsOnHost[m - 1];
    n.aabb = di_.aabb[m].as<float>();
    n.children = innerRecords(m);
    n.boxes = dBoxes;
    n.boxesF = boxF_.as<float>();
    n.out = outView(1 - buf, hdrPtr(m + 1));
    n.counter = nmCounter + m;
    n.ticket = nmTicket + m;
    n.status = status;
    n.levelItems = (wantLevels && m > 0)
                       ? reinterpret_cast<uint32_t*>(z + offLevels_) + static_cast<size_t>(m - 1) * nq
                       : nullptr;
    n.D = D;
    launchNodeMajorRange(n, grids_[m], stream_);
    launchFrontierHeader(n.counter, hdrPtr(m + 1), n.out.cap, n.out.tileCap, status, stream_);
}

void BatchEngine::enqueueLaunches(const double* dBoxes, uint32_t nq, int mode, unsigned flags) {
    lastKnn_ = false;
    lastCompletion_ = false;
    const int H = static_cast<int>(di_.height);
    const int D = static_cast<int>(di_.D);
    char* z = zeroBlock_.as<char>();
    auto* desc = reinterpret_cast<unsigned long long*>(z + offDesc_);
    auto* tickets = reinterpret_cast<uint32_t*>(z + offTickets_);
    auto* status = reinterpret_cast<uint32_t*>(z + offStatus_);
    auto* qcount = reinterpret_cast<uint32_t*>(z + offQcount_);
    auto* levels = reinterpret_cast<uint32_t*>(z + offLevels_);
    const bool wantLevels = (flags & kWantLevels) != 0;

    if (timing_) record(0);
    TBLAEQ_CUDA(cudaMemsetAsync(z, 0, zeroBytes_, stream_));
    const FrontierBufs& r0 = f_[0];
    launchRootFrontier(r0.q.as<uint32_t>(), r0.cbeg.as<uint32_t>(), r0.cpre.as<uint32_t>(), r0.x.as<double>(),
                       r0.tileStart.as<uint32_t>(), hdrPtr(0), nq, static_cast<uint32_t>(di_.meshCount[0]), D, tile_,
                       stream_);
    float* boxFi = boxF_.as<float>() + static_cast<size_t>(qcap_) * 2 * D;
    if (mode == kModeExact) launchRoundBoxes(dBoxes, nq, D, boxF_.as<float>(), boxFi, stream_);
    if (timing_) record(1);
    // Node-major levels (the variant the autotuner may choose per inner level) need their buffers at
    // the current capacities (sized by the synchronous batch that must precede asynchronous ones);
    // without them every level runs entry-major. Once a level ran node-major, the frontiers below it
    // are in no particular query order, and the results are grouped by query at the end.
    const bool nmReady = useNodeMajor(mode) && nmEntryCap_ >= caps_.entries && nmResultCap_ >= caps_.results &&
                         (!(flags & kWantVals) || nmVals_);
    bool nodeMajor = false;
    int buf = 0;
    // The finest exact level decides points from their float copies (not with the staged variant),
    // and, unless per-level counts are wanted (they count the points of every surviving cluster),
    // tests the clusters' point groups first: the last inner level then hands on (query, cluster)
    // entries whose children are the cluster's groups, a group level keeps the groups whose box
    // meets the query's, and the point level tests only their points.
    const bool floatPath = mode == kModeExact && floatPoints_ && di_.pointsF.bytes() &&
                           floatPointsSupported(di_.D) && variants_[H - 1] != kVariantStaged;
    groupsThisBatch_ = floatPath && pointGroups_ && !wantLevels && di_.groupRec.bytes() && H >= 2;
    for (int m = 0; m < H; ++m) {
        if (nmReady && m < H - 1 && variants_[m] == kVariantNodeMajor) {
            nodeMajor = true;
            enqueueNodeMajorLevel(m, buf, dBoxes, nq, wantLevels);
            buf = 1 - buf;
            if (timing_) record(2 + m);
            continue;
        }
        ExpandArgs a{};
        a.in = inView(buf, hdrPtr(m));
        a.child.rows = (m == 0) ? di_.coarseVals.as<double>() : di_.rows[m - 1];
        a.child.rowsOnHost = (m == 0) ? 0 : di_.rowsOnHost[m - 1];
        a.query.boxes = dBoxes;
        a.query.boxesF = (mode == kModeExact) ? boxF_.as<float>() : nullptr;
        a.scratch.desc = desc + static_cast<size_t>(m) * tileCap_;
        a.scratch.ticket = tickets + m;
        a.scratch.status = status;
        a.scratch.levelItems = (wantLevels && m > 0) ? levels + static_cast<size_t>(m - 1) * nq : nullptr;
        a.D = D;
        a.useFma = 1;
        a.variant = variants_[m];
        a.gridPercent = grids_[m];
        if (m < H - 1) {
            a.child.nodes = (mode == kModeExact) ? innerRecords(m) : di_.nodeRef[m].as<NodeRec>();
            a.child.aabb = (mode == kModeExact) ? di_.aabb[m].as<float>() : nullptr;
            a.fout = outView(1 - buf, hdrPtr(m + 1));
            launchExpand(a, kPredRangeRadius, false, 0, stream_);
            buf = 1 - buf;
        } else {
            if (groupsThisBatch_) {
                ExpandArgs g{};
                g.in = inView(buf, hdrPtr(H - 1));
                g.child.rows = nullptr;  // a group entry keeps its cluster's coordinates
                g.child.nodes = di_.groupRec.as<NodeRec>();
                g.child.aabb = di_.groupBox.as<float>();
                g.query.boxes = dBoxes;
                g.query.boxesF = boxF_.as<float>();
                g.scratch.desc = desc + static_cast<size_t>(H) * tileCap_;
                g.scratch.ticket = tickets + H;
                g.scratch.status = status;
                g.D = D;
                g.useFma = 1;
                g.variant = kVariantDirect;
                g.gridPercent = 100;
                g.fout = outView(1 - buf, hdrPtr(H + 3));
                launchExpand(g, kPredGroupBox, false, 0, stream_);
                buf = 1 - buf;
                a.in = inView(buf, hdrPtr(H + 3));
            }
            a.child.outMap = di_.mapPtr[H - 1];
            int finestPred = (mode == kModeExact) ? kPredRangeBox : kPredAll;
            if (floatPath) {
                a.child.rowsF = di_.pointsF.as<float>();
                a.child.perm = di_.pointPerm.as<uint32_t>();
                a.query.boxesFi = boxFi;
                finestPred = kPredRangeBoxF;
            }
            a.rout.qcount = qcount;
            a.rout.hdr = hdrPtr(H);
            a.rout.cap = static_cast<uint32_t>(caps_.results);
            if (nodeMajor) {
                // The frontier is in no particular query order: results go out raw, with their query,
                // and are grouped by query below.
                a.rout.ids = rawIds_.as<uint64_t>();
                a.rout.q = rawQ_.as<uint32_t>();
                a.rout.vals = (flags & kWantVals) ? rawVals_.as<double>() : nullptr;
            } else {
                a.rout.ids = resIds_.as<uint64_t>();
                a.rout.vals = (flags & kWantVals) ? resVals_.as<double>() : nullptr;
            }
            launchExpand(a, finestPred, true, 0, stream_);
        }
        if (timing_) record(2 + m);
    }
    launchExclusiveScan(qcount, offsets_.as<uint64_t>(), nq, stream_);
    if (nodeMajor)
        launchGroupResults(rawIds_.as<uint64_t>(), rawQ_.as<uint32_t>(),
                           (flags & kWantVals) ? rawVals_.as<double>() : nullptr, hdrPtr(H),
                           static_cast<uint32_t>(caps_.results), D, offsets_.as<uint64_t>(),
                           reinterpret_cast<uint32_t*>(z + offRcursor_), resIds_.as<uint64_t>(),
                           (flags & kWantVals) ? resVals_.as<double>() : nullptr, stream_);
    if (timing_) record(2 + H);
}

std::vector<uint64_t> BatchEngine::groupCounts() {
    std::vector<uint64_t> out(3, 0);
    if (lastKnn_ || !groupsThisBatch_ || !zeroBlock_.bytes()) return out;
    const int H = static_cast<int>(di_.height);
    uint32_t a[2] = {0, 0}, b[2] = {0, 0};
    TBLAEQ_CUDA(cudaMemcpyAsync(a, hdrPtr(H - 1), 8, cudaMemcpyDeviceToHost, stream_));
    TBLAEQ_CUDA(cudaMemcpyAsync(b, hdrPtr(H + 3), 8, cudaMemcpyDeviceToHost, stream_));
    TBLAEQ_CUDA(cudaStreamSynchronize(stream_));
    out[0] = a[1];
    out[1] = b[0];
    out[2] = b[1];
    return out;
}

uint32_t BatchEngine::status() {
    uint32_t st = 0;
    TBLAEQ_CUDA(cudaMemcpyAsync(&st, zeroBlock_.as<char>() + offStatus_, 4, cudaMemcpyDeviceToHost, stream_));
    TBLAEQ_CUDA(cudaStreamSynchronize(stream_));
    return st;
}

void BatchEngine::checkSplitLimit() {
    const int H = static_cast<int>(di_.height);
    std::vector<uint32_t> h((H + 2) * 2);
    TBLAEQ_CUDA(cudaMemcpyAsync(h.data(), hdrPtr(0), h.size() * 4, cudaMemcpyDeviceToHost, stream_));
    TBLAEQ_CUDA(cudaStreamSynchronize(stream_));
    for (int lv = 1; lv < H; ++lv)
        if (h[2 * lv] > splitLimit_ || h[2 * lv + 1] > splitLimit_)
            throw SplitBatch("level " + std::to_string(lv) + " exceeds the traversal limit; split the batch");
}

void BatchEngine::growFromHeaders() {
    const int H = static_cast<int>(di_.height);
    std::vector<uint32_t> h((H + 4) * 2);
    TBLAEQ_CUDA(cudaMemcpyAsync(h.data(), hdrPtr(0), h.size() * 4, cudaMemcpyDeviceToHost, stream_));
    TBLAEQ_CUDA(cudaStreamSynchronize(stream_));
    EngineCaps want = caps_;
    bool grew = false;
    for (int lv = 1; lv <= H + 3; ++lv) {
        if (lv >= H && lv < H + 3) continue;  // result and KNN slots: below
        const uint64_t cnt = h[2 * lv], items = h[2 * lv + 1];
        if (cnt > splitLimit_ || items > splitLimit_)
            throw SplitBatch("level " + std::to_string(lv) + " exceeds the traversal limit; split the batch");
        if (cnt > caps_.entries) {
            want.entries = std::max<uint64_t>(want.entries, cnt + cnt / 4 + 1024);
            grew = true;
        }
        if (items > caps_.items) {
            want.items = std::max<uint64_t>(want.items, items + items / 4 + 4096);
            grew = true;
        }
    }
    // Results: slot H holds the one-pass (or wave-1) results, slot H+1 the wave-2 results of a
    // two-wave KNN batch (whose buffer follows the same capacity).
    // (After a node-major completion slot H+1 only counts its candidates, whose buffers follow
    // their own capacity: growKnnMajor.)
    const uint64_t res = lastCompletion_ ? h[2 * H] : std::max<uint64_t>(h[2 * H], h[2 * (H + 1)]);
    if (res > caps_.results) {
        want.results = std::max<uint64_t>(want.results, res + res / 4 + 4096);
        grew = true;
    }
    if (!grew) {
        // Every capacity is tracked by a header above; an overflow none of them shows is not
        // expected. Entry and result buffers double (cheap); item capacity is exact from the sums.
        want.entries *= 2;
        want.results *= 2;
    }
    try {
        reserve(want, qcap_, haveVals_ ? kWantVals : 0);
    } catch (const SplitBatch& e) {
        std::string msg = std::string(e.what()) + " (status " + std::to_string(status()) + "; level entries/items:";
        for (int lv = 0; lv < H + 2; ++lv) msg += " " + std::to_string(h[2 * lv]) + "/" + std::to_string(h[2 * lv + 1]);
        msg += ")";
        throw SplitBatch(msg);
    }
}

BatchOutput BatchEngine::output(uint32_t nq, unsigned flags) const {
    BatchOutput o;
    o.nq = nq;
    if (lastKnn_) {
        o.offsets = knnOff_.as<uint64_t>();
        o.ids = knnIds_.as<uint64_t>();
        o.dist2 = knnD2_.as<double>();
        o.levelItems = (flags & kWantLevels)
                           ? reinterpret_cast<const uint32_t*>(zeroBlock_.as<char>() + offLevels_)
                           : nullptr;
        return o;
    }
    o.offsets = offsets_.as<uint64_t>();
    o.ids = resIds_.as<uint64_t>();
    o.vals = (flags & kWantVals) ? resVals_.as<double>() : nullptr;
    o.levelItems = (flags & kWantLevels) ? reinterpret_cast<const uint32_t*>(zeroBlock_.as<char>() + offLevels_)
                                         : nullptr;
    return o;
}

BatchOutput BatchEngine::runRange(const double* dBoxes, uint32_t nq, int mode, unsigned flags) {
    WorkspaceGuard guard(*this);
    reserve(caps_, nq, flags);
    for (int attempt = 0; attempt < 16; ++attempt) {
        lastRuns_ = static_cast<uint32_t>(attempt + 1);
        if (useNodeMajor(mode)) reserveNodeMajor(flags);
        enqueueRange(dBoxes, nq, mode, flags);
        // The status word and the result total come back together: one host synchronisation.
        uint32_t st = 0;
        uint64_t total = 0;
        TBLAEQ_CUDA(cudaMemcpyAsync(&st, zeroBlock_.as<char>() + offStatus_, 4, cudaMemcpyDeviceToHost, stream_));
        TBLAEQ_CUDA(cudaMemcpyAsync(&total, offsets_.as<uint64_t>() + nq, 8, cudaMemcpyDeviceToHost, stream_));
        TBLAEQ_CUDA(cudaStreamSynchronize(stream_));
        // A 32-bit prefix overflow leaves the next frontier's item mapping meaningless, so the
        // launches after it may report window overflows and look-back timeouts of their own: those
        // count as failures only when no overflow explains them.
        const uint32_t over = st & (kStatusOverflowEntries | kStatusOverflowItems | kStatusOverflowSum);
        if ((st & (kStatusLookbackTimeout | kStatusWindowOverflow)) && !over) {
            throw CudaError(cudaErrorLaunchTimeout, "traversal kernel reported status " + std::to_string(st));
        }
        if (st & kStatusOverflowSum)
            throw SplitBatch("a level generates more than 2^32 items; split the batch");
        if (st == 0) {
            BatchOutput o = output(nq, flags);
            o.total = total;
            return o;
        }
        growFromHeaders();
    }
    throw CudaError(cudaErrorMemoryAllocation, "traversal workspace did not converge after 16 growth steps");
}

}  // namespace tblaeq

namespace tblaeq {

uint64_t BatchEngine::runGridLevel(int l, const uint64_t* dIds, const double* dVals, uint64_t p, bool range,
                                   const double* dQuery, const uint8_t* dMask, uint64_t* outIds, double* outVals,
                                   uint64_t outCap) {
    WorkspaceGuard guard(*this);
    if (p == 0) return 0;
    if (p > 0xffffffffull || outCap > 0xffffffffull) throw std::invalid_argument("grid too large for one level");
    const int D = static_cast<int>(di_.D);
    EngineCaps want = caps_;
    want.entries = std::max<uint64_t>(want.entries, 1);
    want.items = std::max<uint64_t>(want.items, p);
    reserve(want, 1, 0);
    // The grid's own tile starts cover p items; the survivors' children are bounded by outCap.
    if (outCap > caps_.items) {
        want.items = outCap;
        reserve(want, 1, 0);
    }
    if (p > caps_.entries) {
        want.entries = p;
        reserve(want, 1, 0);
    }
    char* z = zeroBlock_.as<char>();
    auto* desc = reinterpret_cast<unsigned long long*>(z + offDesc_);
    auto* tickets = reinterpret_cast<uint32_t*>(z + offTickets_);
    auto* statusPtr = reinterpret_cast<uint32_t*>(z + offStatus_);
    for (int attempt = 0; attempt < 2; ++attempt) {
        TBLAEQ_CUDA(cudaMemsetAsync(z, 0, zeroBytes_, stream_));
        const FrontierBufs& r0 = f_[0];
        launchRootFrontier(r0.q.as<uint32_t>(), r0.cbeg.as<uint32_t>(), r0.cpre.as<uint32_t>(), r0.x.as<double>(),
                           r0.tileStart.as<uint32_t>(), hdrPtr(0), 1, static_cast<uint32_t>(p), D, tile_, stream_);
        ExpandArgs a{};
        a.in = inView(0, hdrPtr(0));
        a.child.rows = dVals;
        a.child.keys = dIds;
        a.child.nodes = di_.nodeOrig[l].as<NodeRec>();
        a.child.mask = dMask;
        a.query.boxes = dQuery;
        a.fout = outView(1, hdrPtr(1));
        a.scratch.desc = desc;
        a.scratch.ticket = tickets;
        a.scratch.status = statusPtr;
        a.D = D;
        a.useFma = 1;
        launchExpand(a, range ? kPredRangeRadius : kPredMask, false, 0, stream_);

        ExpandArgs b{};
        b.in = inView(1, hdrPtr(1));
        b.child.rows = di_.rows[l];
        b.child.rowsOnHost = di_.rowsOnHost[l];
        b.child.outMap = di_.mapPtr[l + 1];
        b.rout.ids = outIds;
        b.rout.vals = outVals;
        b.rout.hdr = hdrPtr(2);
        b.rout.cap = static_cast<uint32_t>(outCap);
        b.scratch.desc = desc + tileCap_;
        b.scratch.ticket = tickets + 1;
        b.scratch.status = statusPtr;
        b.D = D;
        b.useFma = 1;
        launchExpand(b, kPredAll, true, 0, stream_);

        const uint32_t st = status();
        if (st & (kStatusLookbackTimeout | kStatusWindowOverflow))
            throw CudaError(cudaErrorLaunchTimeout, "traversal kernel reported status " + std::to_string(st));
        uint32_t h[6];
        TBLAEQ_CUDA(cudaMemcpyAsync(h, hdrPtr(0), sizeof(h), cudaMemcpyDeviceToHost, stream_));
        TBLAEQ_CUDA(cudaStreamSynchronize(stream_));
        if (st == 0) return h[4];
        if (st & kStatusOverflowEntries && h[4] > outCap)
            throw CudaError(cudaErrorMemoryAllocation, "level output exceeds its buffer");
        want.entries = std::max<uint64_t>(caps_.entries, h[2] + 1);
        want.items = std::max<uint64_t>(caps_.items, static_cast<uint64_t>(h[3]) + 1);
        reserve(want, 1, 0);
    }
    throw CudaError(cudaErrorMemoryAllocation, "per-level workspace did not converge");
}

}  // namespace tblaeq

namespace tblaeq {

BatchEngine::FrontierView BatchEngine::lastKnnFrontier() const {
    const int H = static_cast<int>(di_.height);
    FrontierView v;
    v.in = inView(lastKnnBuf_, hdrPtr(H - 1));
    v.node = f_[lastKnnBuf_].node.as<uint32_t>();
    v.cap = static_cast<uint32_t>(caps_.entries);
    v.offsets = twoWave_ ? offF_.as<uint64_t>() : nullptr;
    return v;
}

std::vector<uint64_t> BatchEngine::knnCounters() {
    const int H = static_cast<int>(di_.height);
    std::vector<uint32_t> h((H + 2) * 2);
    unsigned long long work[2] = {0, 0};
    TBLAEQ_CUDA(cudaMemcpyAsync(h.data(), hdrPtr(0), h.size() * 4, cudaMemcpyDeviceToHost, stream_));
    TBLAEQ_CUDA(cudaMemcpyAsync(work, zeroBlock_.as<char>() + offWork_, 16, cudaMemcpyDeviceToHost, stream_));
    TBLAEQ_CUDA(cudaStreamSynchronize(stream_));
    // One-pass traversal loads every child row of the final frontier: its item count.
    const uint64_t rows1 = twoWave_ ? work[0] : h[2 * (H - 1) + 1];
    return {h[2 * (H - 1)], h[2 * H], h[2 * (H + 1)], rows1, twoWave_ ? work[1] : 0};
}

void BatchEngine::reserveKnn(uint32_t nq) {
    if (knnQcap_ < std::max<uint32_t>(nq, 1)) {
        knnQcap_ = std::max<uint32_t>(nq, 1);
        tau_.alloc(knnQcap_ * 8ull);
        knnCount_.alloc(knnQcap_ * 4ull);
        candOff_.alloc((knnQcap_ + 1ull) * 8);
        knnOff_.alloc((knnQcap_ + 1ull) * 8);
        offF_.alloc((knnQcap_ + 1ull) * 8);
        waveM_.alloc(knnQcap_ * 4ull);
        selCount_.alloc(knnQcap_ * 4ull);
        selOff_.alloc((knnQcap_ + 1ull) * 8);
        selIds_.alloc(knnQcap_ * 32ull * 8);
        selD2_.alloc(knnQcap_ * 32ull * 8);
        candOffB_.alloc((knnQcap_ + 1ull) * 8);
        candOffS_.alloc((knnQcap_ + 1ull) * 8);
    }
    if (entryCap_ < caps_.entries) {
        entryCap_ = caps_.entries;
        const uint64_t seg = compactSegments(entryCap_);
        cmpCnt_.alloc(seg * 4);
        cmpKids_.alloc(seg * 4);
        cmpEntryOff_.alloc((seg + 1) * 8);
        cmpKidOff_.alloc((seg + 1) * 8);
        lbE_.alloc(entryCap_ * 8);
        scoreE_.alloc(entryCap_ * 8);
        sel_.alloc(entryCap_);
    }
    if (resCapB_ < caps_.results) {
        resCapB_ = caps_.results;
        resIdsB_.alloc(resCapB_ * 8);
        resQB_.alloc(resCapB_ * 4);
        resDistB_.alloc(resCapB_ * 8);
    }
}

void BatchEngine::enqueueKnn(const double* dPoints, uint32_t nq, const uint32_t* dK, unsigned flags) {
    lastKnn_ = true;
    const int H = static_cast<int>(di_.height);
    const int D = static_cast<int>(di_.D);
    char* z = zeroBlock_.as<char>();
    auto* desc = reinterpret_cast<unsigned long long*>(z + offDesc_);
    auto* tickets = reinterpret_cast<uint32_t*>(z + offTickets_);
    auto* status = reinterpret_cast<uint32_t*>(z + offStatus_);
    auto* qcount = reinterpret_cast<uint32_t*>(z + offQcount_);
    auto* qcountF = reinterpret_cast<uint32_t*>(z + offQcountF_);
    auto* qcountB = reinterpret_cast<uint32_t*>(z + offQcountB_);
    auto* levels = reinterpret_cast<uint32_t*>(z + offLevels_);
    const bool wantLevels = (flags & kWantLevels) != 0;
    double* tau = tau_.as<double>();

    if (timing_) record(0);
    TBLAEQ_CUDA(cudaMemsetAsync(z, 0, zeroBytes_, stream_));
    launchFillDouble(tau, std::numeric_limits<double>::infinity(), nq, stream_);
    const FrontierBufs& r0 = f_[0];
    launchRootFrontier(r0.q.as<uint32_t>(), r0.cbeg.as<uint32_t>(), r0.cpre.as<uint32_t>(), r0.x.as<double>(),
                       r0.tileStart.as<uint32_t>(), hdrPtr(0), nq, static_cast<uint32_t>(di_.meshCount[0]), D, tile_,
                       stream_);
    if (timing_) record(1);
    auto base = [&](int m, int buf) {
        ExpandArgs a{};
        a.in = inView(buf, hdrPtr(m));
        a.child.rows = (m == 0) ? di_.coarseVals.as<double>() : di_.rows[m - 1];
        a.child.rowsOnHost = (m == 0) ? 0 : di_.rowsOnHost[m - 1];
        a.query.points = dPoints;
        a.query.tau = tau;
        a.query.k = dK;
        a.scratch.desc = desc + static_cast<size_t>(m) * tileCap_;
        a.scratch.ticket = tickets + m;
        a.scratch.status = status;
        a.scratch.levelItems = (wantLevels && m > 0) ? levels + static_cast<size_t>(m - 1) * nq : nullptr;
        a.D = D;
        a.useFma = 1;
        a.variant = kVariantDirect;
        return a;
    };
    // The beam leaves clusters out of the last frontier, so only the completion that walks the
    // hierarchy again from the root (not the query-major wave 2 over that frontier) may follow it.
    // A batch of fewer queries than one node-major unit holds gains nothing from that walk (each
    // unit would carry a few lanes) and pays its launches and passes in latency: it runs the
    // query-major wave 2.
    const bool completion = twoWave_ && knnNodeMajor_ && nq >= kCompletionMinQueries;
    const bool probe = completion && probeBeam_ > 0;
    auto* qcountP = reinterpret_cast<uint32_t*>(z + offQcountP_);
    if (probe) launchFillU32(probeK_.as<uint32_t>(), probeBeam_, nq, stream_);
    int buf = 0;
    for (int m = 0; m < H - 1; ++m) {
        ExpandArgs a = base(m, buf);
        a.child.nodes = di_.nodeSub[m].as<NodeRec>();
        a.child.aabb = di_.aabb[m].as<float>();
        a.child.leaf = di_.leaf[m].as<uint32_t>();
        a.fout = outView(1 - buf, hdrPtr(m + 1));
        a.fout.qcount = (m == H - 2) ? qcountF : (probe ? qcountP + static_cast<size_t>(m) * qcap_ : nullptr);
        launchExpand(a, kPredKnnBound, false, 0, stream_);
        buf = 1 - buf;
        if (probe && m < H - 2) {
            // The probe's beam: every query keeps its probeBeam_ entries of smallest lower bound
            // (order kept), so the levels below and wave 1 see only the clusters under them.
            const FrontierIn Fm = inView(buf, hdrPtr(m + 1));
            const uint32_t cap = static_cast<uint32_t>(caps_.entries);
            launchExclusiveScan(qcountP + static_cast<size_t>(m) * qcap_, offF_.as<uint64_t>(), nq, stream_);
            launchEntryBounds(Fm.q, f_[buf].node.as<uint32_t>(), Fm.x, Fm.hdr, cap, D, dPoints,
                              di_.nodeSub[m].as<NodeRec>(), di_.aabb[m].as<float>(), lbE_.as<double>(),
                              scoreE_.as<double>(), stream_);
            launchClampCounts(offF_.as<uint64_t>(), probeK_.as<uint32_t>(), nq, selCount_.as<uint32_t>(), stream_);
            launchExclusiveScan(selCount_.as<uint32_t>(), selOff_.as<uint64_t>(), nq, stream_);
            launchTopK(offF_.as<uint64_t>(), nullptr, lbE_.as<double>(), cap, nullptr, nullptr, nullptr, 0,
                       probeK_.as<uint32_t>(), nq, selOff_.as<uint64_t>(), selIds_.as<uint64_t>(),
                       selD2_.as<double>(), selCount_.as<uint32_t>(), status, stream_);
            TBLAEQ_CUDA(cudaMemsetAsync(sel_.get(), 0, entryCap_, stream_));
            launchScatterSel(selIds_.as<uint64_t>(), selOff_.as<uint64_t>(), nq, cap, sel_.as<uint8_t>(), stream_);
            launchCompactFrontier(Fm, cap, 1, sel_.as<uint8_t>(), lbE_.as<double>(), tau, D, cmpCnt_.as<uint32_t>(),
                                  cmpKids_.as<uint32_t>(), cmpEntryOff_.as<uint64_t>(), cmpKidOff_.as<uint64_t>(),
                                  outView(1 - buf, hdrPtr(m + 1)), stream_);
            buf = 1 - buf;
        }
        if (timing_) record(2 + m);
    }
    // `buf` now holds the last frontier F: the surviving finest clusters, query-major.
    lastKnnBuf_ = buf;
    ExpandArgs fin = base(H - 1, buf);
    fin.child.outMap = di_.mapPtr[H - 1];
    fin.rout.ids = resIds_.as<uint64_t>();
    fin.rout.q = resQ_.as<uint32_t>();
    fin.rout.dist2 = resDist_.as<double>();
    fin.rout.qcount = qcount;
    fin.rout.hdr = hdrPtr(H);
    fin.rout.cap = static_cast<uint32_t>(caps_.results);
    lastCompletion_ = completion;
    if (!twoWave_) {
        launchExpand(fin, kPredKnnPoint, true, 0, stream_);
        if (timing_) record(1 + H);
        launchExclusiveScan(qcount, candOff_.as<uint64_t>(), nq, stream_);
        launchClampCounts(candOff_.as<uint64_t>(), dK, nq, knnCount_.as<uint32_t>(), stream_);
        launchExclusiveScan(knnCount_.as<uint32_t>(), knnOff_.as<uint64_t>(), nq, stream_);
        launchTopK(candOff_.as<uint64_t>(), resIds_.as<uint64_t>(), resDist_.as<double>(), caps_.results, nullptr,
                   nullptr, nullptr, 0, dK, nq, knnOff_.as<uint64_t>(), knnIds_.as<uint64_t>(), knnD2_.as<double>(),
                   knnCount_.as<uint32_t>(), status, stream_);
        if (timing_) record(2 + H);
        return;
    }
    const FrontierIn F = inView(buf, hdrPtr(H - 1));
    const FrontierBufs& fb = f_[buf];
    const uint32_t fcap = static_cast<uint32_t>(caps_.entries);
    // Rank F's entries per query (lower bound, or the learned score) and select the best few.
    launchExclusiveScan(qcountF, offF_.as<uint64_t>(), nq, stream_);
    launchEntryBounds(F.q, fb.node.as<uint32_t>(), F.x, F.hdr, fcap, D, dPoints, di_.nodeSub[H - 2].as<NodeRec>(),
                      di_.aabb[H - 2].as<float>(), lbE_.as<double>(), scoreE_.as<double>(), stream_);
    if (scorer_) scorer_(scorerCtx_, F, fb.node.as<uint32_t>(), fcap, dPoints, scoreE_.as<double>(), stream_);
    const double avgLeaf = static_cast<double>(di_.meshCount[H - 1]) / static_cast<double>(di_.meshCount[H - 2]);
    launchWaveWidth(dK, nq, waveScale_ / avgLeaf, waveM_.as<uint32_t>(), stream_);
    launchClampCounts(offF_.as<uint64_t>(), waveM_.as<uint32_t>(), nq, selCount_.as<uint32_t>(), stream_);
    launchExclusiveScan(selCount_.as<uint32_t>(), selOff_.as<uint64_t>(), nq, stream_);
    launchTopK(offF_.as<uint64_t>(), nullptr, scoreE_.as<double>(), fcap, nullptr, nullptr, nullptr, 0,
               waveM_.as<uint32_t>(), nq, selOff_.as<uint64_t>(), selIds_.as<uint64_t>(), selD2_.as<double>(),
               selCount_.as<uint32_t>(), status, stream_);
    TBLAEQ_CUDA(cudaMemsetAsync(sel_.get(), 0, entryCap_, stream_));
    launchScatterSel(selIds_.as<uint64_t>(), selOff_.as<uint64_t>(), nq, fcap, sel_.as<uint8_t>(), stream_);
    // Each wave expands a compacted copy of its own entries (in the other frontier buffer), so no
    // item of a skipped cluster is visited.
    const int cbuf = 1 - buf;
    auto compact = [&](int mode) {
        launchCompactFrontier(F, fcap, mode, sel_.as<uint8_t>(), lbE_.as<double>(), tau, D, cmpCnt_.as<uint32_t>(),
                              cmpKids_.as<uint32_t>(), cmpEntryOff_.as<uint64_t>(), cmpKidOff_.as<uint64_t>(),
                              outView(cbuf, hdrPtr(H + 2)), stream_);
    };
    // Wave 1: every point of the selected clusters; their K-th distance bounds tau.
    compact(1);
    fin.in = inView(cbuf, hdrPtr(H + 2));
    fin.child.entrySel = nullptr;
    fin.child.entryLb = nullptr;
    fin.wave = 1;
    fin.scratch.work = reinterpret_cast<unsigned long long*>(z + offWork_);
    launchExpand(fin, kPredKnnPoint, true, 0, stream_);
    launchExclusiveScan(qcount, candOff_.as<uint64_t>(), nq, stream_);
    launchClampCounts(candOff_.as<uint64_t>(), dK, nq, knnCount_.as<uint32_t>(), stream_);
    launchExclusiveScan(knnCount_.as<uint32_t>(), knnOff_.as<uint64_t>(), nq, stream_);
    launchTopK(candOff_.as<uint64_t>(), resIds_.as<uint64_t>(), resDist_.as<double>(), caps_.results, nullptr, nullptr,
               nullptr, 0, dK, nq, knnOff_.as<uint64_t>(), knnIds_.as<uint64_t>(), knnD2_.as<double>(),
               knnCount_.as<uint32_t>(), status, stream_);
    launchTauFromTopK(knnOff_.as<uint64_t>(), knnD2_.as<double>(), dK, nq, tau, stream_);
    if (completion) {
        // Every point within tau, outside the clusters wave 1 read: the hierarchy again from the
        // root, node-major, then the clusters' points, each read once per 32 of its queries.
        auto* tick = reinterpret_cast<uint32_t*>(z + offKnnTick_);
        uint32_t* pairCnt = tick + (H + 1);
        uint32_t* candCnt = pairCnt + H;
        launchWaveOneClusters(selIds_.as<uint64_t>(), selOff_.as<uint64_t>(), selCount_.as<uint32_t>(),
                              fb.node.as<uint32_t>(), fcap, nq, 32, excl_.as<uint32_t>(), stream_);
        const uint32_t pcap = static_cast<uint32_t>(pairCap_);
        int pb = 0;
        auto group = [&](int mesh, int from, const uint32_t* count = nullptr) {
            const uint32_t M = static_cast<uint32_t>(di_.meshCount[mesh]);
            auto* nodeCnt = reinterpret_cast<uint32_t*>(z + offKnnNodeCnt_[mesh]);
            launchNodeTranspose(pairNode_[from].as<uint32_t>(), count ? count : pairCnt + mesh, pcap, M, nodeCnt,
                                pairNodeOff_.as<uint32_t>(), pairUnitOff_.as<uint32_t>(), nodeCnt + M,
                                pairList_.as<uint32_t>(), stream_, pairUnitNode_.as<uint32_t>(),
                                static_cast<uint32_t>(pairUnitNode_.bytes() / 4));
            return M;
        };
        for (int m = 0; m < H - 1; ++m) {
            KnnBoundLevelArgs b{};
            b.nq = nq;
            if (m == 0) {
                b.nNodes = 0;
                b.rootChildren = static_cast<uint32_t>(di_.meshCount[0]);
            } else {
                b.inQ = pairQ_[pb].as<uint32_t>();
                b.inCount = pairCnt + (m - 1);
                b.inCap = pcap;
                b.nNodes = group(m - 1, pb);
                b.list = pairList_.as<uint32_t>();
                b.nodeOff = pairNodeOff_.as<uint32_t>();
                b.unitOff = pairUnitOff_.as<uint32_t>();
                b.unitNode = pairUnitNode_.as<uint32_t>();
                b.parents = di_.nodeSub[m - 1].as<NodeRec>();
            }
            b.x = di_.nodeX[m].as<double>();
            b.aabb = di_.aabb[m].as<float>();
            b.nodes = di_.nodeSub[m].as<NodeRec>();
            b.points = dPoints;
            b.tau = tau;
            b.outQ = pairQ_[1 - pb].as<uint32_t>();
            b.outNode = pairNode_[1 - pb].as<uint32_t>();
            b.outCap = pcap;
            b.outCount = pairCnt + m;
            b.ticket = tick + m;
            b.status = status;
            b.D = D;
            launchKnnBoundLevel(b, stream_);
            pb = 1 - pb;
        }
        KnnClusterArgs c{};
        c.inQ = pairQ_[pb].as<uint32_t>();
        c.inCount = pairCnt + (H - 2);
        c.inCap = pcap;
        c.nNodes = group(H - 2, pb);
        c.list = pairList_.as<uint32_t>();
        c.nodeOff = pairNodeOff_.as<uint32_t>();
        c.unitOff = pairUnitOff_.as<uint32_t>();
        c.unitNode = pairUnitNode_.as<uint32_t>();
        c.clusters = di_.nodeSub[H - 2].as<NodeRec>();
        c.x = di_.nodeX[H - 2].as<double>();
        c.rows = di_.rows[H - 2];
        c.rowsOnHost = di_.rowsOnHost[H - 2];
        c.decoded = di_.pointsD.bytes() ? di_.pointsD.as<double>() : nullptr;
        if (c.decoded && di_.pointPerm.bytes()) {  // decoded points in point-group order
            c.perm = di_.pointPerm.as<uint32_t>();
            if (knnGroups_) {
                c.clusterGroups = di_.clusterGroups.as<NodeRec>();
                c.groupRec = di_.groupRec.as<NodeRec>();
                c.groupBox = di_.groupBox.as<float>();
            }
        }
        c.map = di_.mapPtr[H - 1];
        c.points = dPoints;
        c.tau = tau;
        c.excl = excl_.as<uint32_t>();
        c.exclStride = 32;
        c.outQ = candQ_.as<uint32_t>();
        c.outId = candId_.as<uint64_t>();
        c.outD2 = candD2_.as<double>();
        c.outCap = static_cast<uint32_t>(candCap_);
        c.outCount = candCnt;
        c.qcount = qcountB;
        c.work = reinterpret_cast<unsigned long long*>(z + offWork_) + 1;
        c.ticket = tick + H;
        c.status = status;
        c.D = D;
        // After each refinement stage the cluster-level pairs are filtered under the tighter bound
        // and grouped by cluster again, so the next pass's units hold live lanes only (under wave
        // 1's bound at D = 16 nearly every cluster is listed for every query, and most lanes of a
        // unit would skip).
        uint32_t* filt = candCnt + 1 + 2 * kMaxRefineStages;
        auto refilter = [&](uint32_t k) {
            const int M2 = H - 2;
            TBLAEQ_CUDA(cudaMemsetAsync(z + offKnnNodeCnt_[M2], 0, 2 * di_.meshCount[M2] * 4, stream_));
            KnnFilterArgs f{};
            f.inQ = pairQ_[pb].as<uint32_t>();
            f.inNode = pairNode_[pb].as<uint32_t>();
            f.inCount = c.inCount;
            f.inCap = pcap;
            f.clusters = di_.nodeSub[M2].as<NodeRec>();
            f.x = di_.nodeX[M2].as<double>();
            f.points = dPoints;
            f.tau = tau;
            f.excl = excl_.as<uint32_t>();
            f.exclStride = 32;
            f.outQ = pairQ_[1 - pb].as<uint32_t>();
            f.outNode = pairNode_[1 - pb].as<uint32_t>();
            f.outCap = pcap;
            f.outCount = filt + k;
            f.status = status;
            f.D = D;
            launchKnnFilterPairs(f, stream_);
            pb = 1 - pb;
            c.inQ = pairQ_[pb].as<uint32_t>();
            c.inCount = filt + k;
            c.nNodes = group(M2, pb, filt + k);
        };
        if (refineStride_ > 1) {
            // Refine the bound first, in stages of decreasing stride (refineStride_^k, ..., the
            // stride itself): each stage tests every stride-th point of the listed clusters within
            // the current bound; with wave 1's they are real points, so their K-th distance bounds
            // tau again, and the next stage (and the full pass below, which skips every cluster
            // whose sphere lies beyond it) works under the tighter bound. A coarse first stage keeps
            // the candidate lists small while the bound is still loose. The stages' candidates serve
            // only the bound (the pass below tests those points again).
            uint32_t* qcS = qcountP;           // the probe's per-level counts are free again
            uint32_t* curS = qcountP + qcap_;
            uint64_t stride = 1;
            for (uint32_t k = 0; k < refineStages_; ++k) stride *= refineStride_;
            for (uint32_t st = 0; st < refineStages_; ++st, stride /= refineStride_) {
                if (stride > 0xffffffffull) continue;
                uint32_t* sTick = candCnt + 1 + 2 * st;
                uint32_t* sCnt = candCnt + 2 + 2 * st;
                TBLAEQ_CUDA(cudaMemsetAsync(qcountP, 0, 2 * static_cast<size_t>(qcap_) * 4, stream_));
                KnnClusterArgs sc = c;
                sc.sampleStride = static_cast<uint32_t>(stride);
                sc.outCount = sCnt;
                sc.qcount = qcS;
                sc.ticket = sTick;
                launchKnnClusterPoints(sc, stream_);
                launchExclusiveScan(qcS, candOffS_.as<uint64_t>(), nq, stream_);
                launchGroupResults(candId_.as<uint64_t>(), candQ_.as<uint32_t>(), candD2_.as<double>(), sCnt,
                                   static_cast<uint32_t>(std::min<uint64_t>(candCap_, resCapB_)), 1,
                                   candOffS_.as<uint64_t>(), curS, resIdsB_.as<uint64_t>(), resDistB_.as<double>(),
                                   stream_);
                launchClampCounts2(candOff_.as<uint64_t>(), candOffS_.as<uint64_t>(), dK, nq,
                                   knnCount_.as<uint32_t>(), stream_);
                launchExclusiveScan(knnCount_.as<uint32_t>(), knnOff_.as<uint64_t>(), nq, stream_);
                launchTopK(candOff_.as<uint64_t>(), resIds_.as<uint64_t>(), resDist_.as<double>(), caps_.results,
                           candOffS_.as<uint64_t>(), resIdsB_.as<uint64_t>(), resDistB_.as<double>(), resCapB_, dK,
                           nq, knnOff_.as<uint64_t>(), knnIds_.as<uint64_t>(), knnD2_.as<double>(),
                           knnCount_.as<uint32_t>(), status, stream_);
                launchTauFromTopK(knnOff_.as<uint64_t>(), knnD2_.as<double>(), dK, nq, tau, stream_);
                refilter(st);
            }
        }
        launchKnnClusterPoints(c, stream_);
        if (timing_) record(1 + H);
        launchExclusiveScan(qcountB, candOffB_.as<uint64_t>(), nq, stream_);
        launchGroupResults(candId_.as<uint64_t>(), candQ_.as<uint32_t>(), candD2_.as<double>(), candCnt,
                           static_cast<uint32_t>(std::min<uint64_t>(candCap_, resCapB_)), 1, candOffB_.as<uint64_t>(),
                           reinterpret_cast<uint32_t*>(z + offCandCursor_), resIdsB_.as<uint64_t>(),
                           resDistB_.as<double>(), stream_);
        launchOneItemHeader(candCnt, hdrPtr(H + 1), stream_);  // the wave-2 candidate count (counters)
        launchClampCounts2(candOff_.as<uint64_t>(), candOffB_.as<uint64_t>(), dK, nq, knnCount_.as<uint32_t>(),
                           stream_);
        launchExclusiveScan(knnCount_.as<uint32_t>(), knnOff_.as<uint64_t>(), nq, stream_);
        launchTopK(candOff_.as<uint64_t>(), resIds_.as<uint64_t>(), resDist_.as<double>(), caps_.results,
                   candOffB_.as<uint64_t>(), resIdsB_.as<uint64_t>(), resDistB_.as<double>(), resCapB_, dK, nq,
                   knnOff_.as<uint64_t>(), knnIds_.as<uint64_t>(), knnD2_.as<double>(), knnCount_.as<uint32_t>(),
                   status, stream_);
        if (timing_) record(2 + H);
        return;
    }
    // Wave 2: the other clusters whose lower bound tau cannot exclude, points within tau.
    compact(2);
    ExpandArgs w2 = fin;
    w2.scratch.desc = desc + static_cast<size_t>(H) * tileCap_;
    w2.scratch.ticket = tickets + H;
    w2.scratch.levelItems = nullptr;
    w2.rout.ids = resIdsB_.as<uint64_t>();
    w2.rout.q = resQB_.as<uint32_t>();
    w2.rout.dist2 = resDistB_.as<double>();
    w2.rout.qcount = qcountB;
    w2.rout.hdr = hdrPtr(H + 1);
    w2.rout.cap = static_cast<uint32_t>(resCapB_);
    w2.wave = 2;
    w2.scratch.work = reinterpret_cast<unsigned long long*>(z + offWork_) + 1;
    launchExpand(w2, kPredKnnPoint, true, 0, stream_);
    if (timing_) record(1 + H);
    launchExclusiveScan(qcountB, candOffB_.as<uint64_t>(), nq, stream_);
    launchClampCounts2(candOff_.as<uint64_t>(), candOffB_.as<uint64_t>(), dK, nq, knnCount_.as<uint32_t>(), stream_);
    launchExclusiveScan(knnCount_.as<uint32_t>(), knnOff_.as<uint64_t>(), nq, stream_);
    launchTopK(candOff_.as<uint64_t>(), resIds_.as<uint64_t>(), resDist_.as<double>(), caps_.results,
               candOffB_.as<uint64_t>(), resIdsB_.as<uint64_t>(), resDistB_.as<double>(), resCapB_, dK, nq,
               knnOff_.as<uint64_t>(), knnIds_.as<uint64_t>(), knnD2_.as<double>(), knnCount_.as<uint32_t>(), status,
               stream_);
    if (timing_) record(2 + H);
}

void BatchEngine::reserveKnnMajor(uint32_t nq) {
    const size_t q1 = std::max<uint32_t>(nq, 1);
    if (excl_.bytes() < q1 * 32 * 4) {
        excl_.alloc(q1 * 32 * 4);
        probeK_.alloc(q1 * 4);
    }
    if (pairCap_ == 0) {
        pairCap_ = std::max<uint64_t>(caps_.entries, 1u << 20);
        uint64_t maxM = 1;
        for (uint64_t m = 0; m + 1 < di_.height; ++m) maxM = std::max<uint64_t>(maxM, di_.meshCount[m]);
        pairNodeOff_.alloc((maxM + 1) * 4);
        pairUnitOff_.alloc((maxM + 1) * 4);
    }
    if (pairQ_[0].bytes() < pairCap_ * 4) {
        for (int b = 0; b < 2; ++b) {
            pairQ_[b].alloc(pairCap_ * 4);
            pairNode_[b].alloc(pairCap_ * 4);
        }
        pairList_.alloc(pairCap_ * 4);
        uint64_t maxM = 1;
        for (uint64_t m = 0; m + 1 < di_.height; ++m) maxM = std::max<uint64_t>(maxM, di_.meshCount[m]);
        pairUnitNode_.alloc((pairCap_ / 32 + maxM + 2) * 4);  // units <= pairs / 32 + nodes
    }
    if (candCap_ == 0) candCap_ = std::max<uint64_t>(caps_.results, 1u << 20);
    if (candQ_.bytes() < candCap_ * 4) {
        candQ_.alloc(candCap_ * 4);
        candId_.alloc(candCap_ * 8);
        candD2_.alloc(candCap_ * 8);
    }
    if (resCapB_ < candCap_) {
        resCapB_ = candCap_;
        resIdsB_.alloc(resCapB_ * 8);
        resQB_.alloc(resCapB_ * 4);
        resDistB_.alloc(resCapB_ * 8);
    }
}

bool BatchEngine::growKnnMajor() {
    const int H = static_cast<int>(di_.height);
    // pair counts, candidates, then (ticket, candidates) per refine stage
    std::vector<uint32_t> c(H + 1 + 2 * kMaxRefineStages, 0);
    TBLAEQ_CUDA(cudaMemcpyAsync(c.data(), zeroBlock_.as<char>() + offKnnTick_ + (H + 1) * 4, c.size() * 4,
                                cudaMemcpyDeviceToHost, stream_));
    TBLAEQ_CUDA(cudaStreamSynchronize(stream_));
    bool grew = false;
    for (int m = 0; m + 1 < H; ++m) {
        if (c[m] > pairCap_) {
            pairCap_ = static_cast<uint64_t>(c[m]) + c[m] / 4 + 4096;
            grew = true;
        }
    }
    uint32_t cand = c[H];
    for (uint32_t st = 0; st < kMaxRefineStages; ++st) cand = std::max(cand, c[H + 2 + 2 * st]);
    if (cand > candCap_) {
        candCap_ = static_cast<uint64_t>(cand) + cand / 4 + 4096;
        grew = true;
    }
    if (pairCap_ >= 0x80000000ull || candCap_ >= 0x80000000ull)
        throw SplitBatch("node-major KNN pairs exceed 2^31; split the batch");
    return grew;
}

BatchOutput BatchEngine::runKnn(const double* dPoints, uint32_t nq, const uint32_t* dK, uint64_t sumK,
                                unsigned flags) {
    WorkspaceGuard guard(*this);
    reserve(caps_, nq, flags);
    reserveKnn(nq);
    if (knnCap_ < std::max<uint64_t>(sumK, 1)) {
        knnCap_ = std::max<uint64_t>(sumK, 1);
        knnIds_.alloc(knnCap_ * 8);
        knnD2_.alloc(knnCap_ * 8);
    }
    bool sumSeen = false;
    for (int attempt = 0; attempt < 16; ++attempt) {
        lastRuns_ = static_cast<uint32_t>(attempt + 1);
        reserveKnnMajor(nq);
        enqueueKnn(dPoints, nq, dK, flags);
        const uint32_t st = status();
        // Window overflows and look-back timeouts that follow an overflow are its consequences (see
        // runRange); alone they are failures.
        const uint32_t over = st & (kStatusOverflowEntries | kStatusOverflowItems | kStatusOverflowSum);
        if ((st & (kStatusLookbackTimeout | kStatusWindowOverflow)) && !over)
            throw CudaError(cudaErrorLaunchTimeout, "traversal kernel reported status " + std::to_string(st));
        // A count past the 32-bit space calls for a split unless a capacity upstream overflowed in
        // the same run (wave 1's results, a pair list: bounds left unset make every stage after it
        // see far more than the batch holds); then the engine grows once and decides on the rerun.
        if (st & kStatusOverflowSum) {
            if (sumSeen || !(st & (kStatusOverflowEntries | kStatusOverflowItems)))
                throw SplitBatch("a level generates more than 2^32 items; split the batch");
            sumSeen = true;
        }
        if (st == 0) {
            if (splitLimit_ < 0xffffffffull) checkSplitLimit();
            BatchOutput o = output(nq, flags);
            o.total = lastTotal(nq);
            return o;
        }
        const bool grewMajor = lastCompletion_ ? growKnnMajor() : false;
        if (!grewMajor) growFromHeaders();
        reserveKnn(nq);
    }
    throw CudaError(cudaErrorMemoryAllocation, "KNN workspace did not converge after 16 growth steps");
}

}  // namespace tblaeq
