// Batched traversal engine: runs many queries through the hierarchy together, one `expand`
// launch per mesh, with all intermediate state on the device.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <memory>
#include <vector>

#include "device_index.hpp"
#include "traverse.cuh"

namespace tblaeq {

enum QueryMode : int {
    kModeRefParity = 0,  // the reference's candidate sets (child radii, STEP, no final filter)
    kModeExact = 1,      // subtree radii + exact final filter / top-K
};

enum BatchFlags : unsigned {
    kWantVals = 1u << 0,    // also return decoded coordinates of every result
    kWantLevels = 1u << 1,  // per-query generated-children count per level
    kUseGraph = 1u << 2,    // replay the batch's launches from a captured CUDA graph
};

struct BatchOutput {
    uint32_t nq = 0;
    uint64_t total = 0;              // number of results
    const uint64_t* offsets = nullptr;  // device, nq + 1
    const uint64_t* ids = nullptr;      // device, total
    const double* vals = nullptr;       // device, total * D (kWantVals)
    const double* dist2 = nullptr;      // device, total (KNN)
    const uint32_t* levelItems = nullptr;  // device, intervals * nq (kWantLevels), [l * nq + q]
};

struct EngineCaps {
    uint64_t entries = 1u << 16;  // frontier entries per level
    uint64_t items = 1u << 22;    // work items per level (children of one frontier)
    uint64_t results = 1u << 20;  // final results per batch
};

// Most stages of the KNN completion's bound refinement.
constexpr uint32_t kMaxRefineStages = 4;
// Smallest KNN batch that runs the node-major completion (smaller ones: the query-major wave 2).
constexpr uint32_t kCompletionMinQueries = 32;

class BatchEngine {
public:
    BatchEngine(const DeviceIndex& di, cudaStream_t stream);
    ~BatchEngine();
    BatchEngine(const BatchEngine&) = delete;
    BatchEngine& operator=(const BatchEngine&) = delete;

    // Range batch: dBoxes = nq rows of lo[D] then hi[D] (device). Blocks until done.
    BatchOutput runRange(const double* dBoxes, uint32_t nq, int mode, unsigned flags);

    // Exact KNN batch: dPoints = nq rows of D coordinates, dK = neighbours per query (device),
    // sumK = sum of K over the batch (host). Results: per-query offsets, ids and squared distances,
    // ascending by (distance, id). Blocks until done.
    BatchOutput runKnn(const double* dPoints, uint32_t nq, const uint32_t* dK, uint64_t sumK, unsigned flags);
    void enqueueKnn(const double* dPoints, uint32_t nq, const uint32_t* dK, unsigned flags);
    // Two-wave final level (default on): rank the last frontier's clusters, expand the best few per
    // query to bound the K-th distance by real points, then expand only the clusters that bound
    // cannot exclude. Off: one pass over every surviving cluster.
    void setTwoWave(bool on) { twoWave_ = on; }
    // Wave 1 of a two-wave KNN batch reads the ceil(scale * K / leaf) + 1 best-ranked clusters of
    // each query (2..32; leaf = points per finest cluster on average); default scale 16.
    void setWaveScale(double scale) { waveScale_ = scale > 0 ? scale : 16.0; }
    // Node-major completion: before its point pass, passes over every stride^k-th, ..., stride-th
    // point of the listed clusters (`stages` of them) tighten each query's bound (stride 0 or 1:
    // off; default 16 in two stages, 256 then 16).
    void setKnnRefine(uint32_t stride, uint32_t stages = 2) {
        refineStride_ = stride;
        refineStages_ = stages < 1 ? 1 : (stages > kMaxRefineStages ? kMaxRefineStages : stages);
    }
    // Node-major completion's point pass: walk each cluster's point groups, skipping a group whose
    // box lies beyond the query's bound (default on; with the range path's point groups).
    void setKnnGroups(bool on) { knnGroups_ = on; }
    uint32_t knnRefine() const { return refineStride_; }
    uint32_t knnRefineStages() const { return refineStages_; }
    double waveScale() const { return waveScale_; }
    // Exact KNN with the two-wave finest level: beam width of the probe (each query keeps its
    // probeBeam entries of smallest lower bound at every level above the clusters, so wave 1 ranks
    // only the clusters under them; 0: no beam, every surviving cluster is ranked), and whether the
    // completion after wave 1 walks the hierarchy node-major (default) or expands every remaining
    // frontier entry query by query (the beam then stays off: that wave only covers the frontier).
    void setKnnProbe(uint32_t beam, bool nodeMajorCompletion) {
        if (beam > 32) throw std::invalid_argument("probe beam must be at most 32");
        probeBeam_ = beam;
        knnNodeMajor_ = nodeMajorCompletion;
    }
    uint32_t probeBeam() const { return probeBeam_; }
    bool knnNodeMajor() const { return knnNodeMajor_; }
    // Largest entry / item capacity a batch may use before it must be split (tests lower it).
    void setSplitLimit(uint64_t limit) { splitLimit_ = limit; }
    // Exact range batches may run inner levels node-major (see NodeMajorArgs) where the level's
    // variant is kVariantNodeMajor (the autotuner's choice): same results, each query's ids in no
    // particular order. Off: those levels run entry-major.
    void setNodeMajor(bool on) {
        if (on != nodeMajor_) dropGraph();
        nodeMajor_ = on;
    }
    bool nodeMajor() const { return nodeMajor_; }
    // Finest exact range level: decide points from their float copies first (default on; the
    // results are the same either way).
    void setFloatPoints(bool on) {
        if (on != floatPoints_) dropGraph();
        floatPoints_ = on;
    }
    // Finest exact range level with float points: test the clusters' point groups first (default
    // on; same results). groupCounts: of the last range batch, the groups tested, the (query,
    // group) pairs kept and the points tested, or zeros when it tested no groups.
    void setPointGroups(bool on) {
        if (on != pointGroups_) dropGraph();
        pointGroups_ = on;
    }
    std::vector<uint64_t> groupCounts();
    // Enqueues of the last synchronous batch: 1, plus one rerun per workspace growth.
    uint32_t lastRuns() const { return lastRuns_; }
    // Kernel nodes and all nodes of the captured range graph (0, 0 when none is held).
    uint64_t graphKernels() const { return graphExec_ ? graphKernels_ : 0; }
    uint64_t graphNodes() const { return graphExec_ ? graphNodes_ : 0; }
    bool twoWave() const { return twoWave_; }
    // Optional device scorer of the last frontier's entries (higher = expand earlier); when unset
    // the entries are ranked by their lower bound. Called with (frontier, hdr, cap, points, out scores).
    using EntryScorer = void (*)(void* ctx, const FrontierIn& f, const uint32_t* node, uint32_t cap,
                                 const double* points, double* score, cudaStream_t s);
    // The last KNN batch's final frontier (surviving finest clusters, query-major): view, node
    // positions and capacity; valid until the next batch.
    struct FrontierView {
        FrontierIn in;
        const uint32_t* node;
        uint32_t cap;
        const uint64_t* offsets;  // per-query entry offsets (nq + 1), two-wave batches only
    };
    FrontierView lastKnnFrontier() const;
    // Counters of the last KNN batch: [0] final-frontier entries, [1] wave-1 candidates,
    // [2] wave-2 candidates, [3] point rows loaded by wave 1 (by the single pass when two-wave is
    // off), [4] point rows loaded by wave 2. [3] + [4] is the finest-level work the ranking saves.
    std::vector<uint64_t> knnCounters();
    void setScorer(EntryScorer fn, void* ctx) {
        scorer_ = fn;
        scorerCtx_ = ctx;
    }

    // Enqueue a range batch without synchronising (capacities must already suffice; used for
    // CUDA-graph capture and timing). check() afterwards reports overflow / timeouts.
    void enqueueRange(const double* dBoxes, uint32_t nq, int mode, unsigned flags);
    // Returns the device status bits of the last enqueued batch (synchronises the stream).
    uint32_t status();
    // Total results of the last batch (synchronises the stream).
    uint64_t lastTotal(uint32_t nq);

    // Kernel variant (Variant) per expand launch m = 0..height-1; default direct everywhere.
    void setVariants(const std::vector<int>& v);
    const std::vector<int>& variants() const { return variants_; }
    // Launch shape per expand launch: the variant and the persistent grid as a percentage of full
    // occupancy (gridPercent of ExpandArgs; 100 = every CTA the SMs hold).
    void setLaunchShapes(const std::vector<int>& variants, const std::vector<int>& gridPercent);
    const std::vector<int>& gridPercents() const { return grids_; }
    // Searches the launch shapes on this batch: every combination of variant {direct, staged} and
    // grid {100, 75, 50, 25}% is timed (median of `reps` runs after a warm-up) and each level keeps
    // its fastest. Returns the per-level median milliseconds of the choice.
    std::vector<float> autotuneRange(const double* dBoxes, uint32_t nq, int mode, unsigned flags, int reps);

    // (entries, items) of every frontier header of the last batch, and the result count.
    void levelCounts(std::vector<uint64_t>& entries, std::vector<uint64_t>& items, uint64_t& results);

    // Per-stage event timing of every batch (memset+root, one stage per expand, scan).
    void setTiming(bool on);
    // Elapsed milliseconds of each stage of the last batch; requires setTiming(true).
    std::vector<float> stageTimes();
    BatchOutput output(uint32_t nq, unsigned flags) const;

    // Per-level plugin step (reference semantics for one query at interval l): keep the grid entries
    // whose pruning predicate holds (range: box distance vs the reference radius; KNN: dMask), then
    // expand the survivors through P_l and Map_{l+1} into outIds/outVals (capacity outCap).
    // Returns the number of output entries. dQuery is the device box (lo|hi) for range queries.
    uint64_t runGridLevel(int l, const uint64_t* dIds, const double* dVals, uint64_t p, bool range,
                          const double* dQuery, const uint8_t* dMask, uint64_t* outIds, double* outVals,
                          uint64_t outCap);

    // Reserve workspace for at least these capacities and this many queries.
    void reserve(const EngineCaps& caps, uint32_t nq, unsigned flags);
    // Releases every workspace buffer and forgets every capacity, so the next batch allocates
    // afresh. A batch that throws (an allocation that failed part-way through a growth, a split,
    // a timeout) calls it on the way out: no later launch can see a capacity whose buffer is gone.
    void resetWorkspace() noexcept;
    const EngineCaps& caps() const { return caps_; }
    size_t workspaceBytes() const;
    int launchesPerBatch() const { return static_cast<int>(di_.height) + 2; }
    cudaStream_t stream() const { return stream_; }

private:
    struct FrontierBufs {
        DeviceMem q, node, cbeg, cpre, x, tileStart;
    };
    const DeviceIndex& di_;
    cudaStream_t stream_;
    int tile_;
    EngineCaps caps_{};
    uint32_t qcap_ = 0;
    bool haveVals_ = false;
    FrontierBufs f_[2];
    // Node-major range levels: the node grouping of the input frontier, and the raw (frontier-order)
    // results before they are grouped by query.
    bool nodeMajor_ = true;
    bool floatPoints_ = true;
    bool pointGroups_ = true;
    bool groupsThisBatch_ = false;
    const NodeRec* innerRecords(int m) const;
    DeviceMem nmNodeOff_, nmUnitOff_, nmUnitNode_, nmList_, rawIds_, rawQ_, rawVals_;
    uint64_t nmEntryCap_ = 0, nmResultCap_ = 0;
    bool nmVals_ = false;
    size_t offNm_ = 0, offRcursor_ = 0;
    std::vector<size_t> offNodeCnt_;  // per level m: nodeCnt then cursor (meshCount[m-1] each), in zeroBlock_
    void reserveNodeMajor(unsigned flags);
    bool useNodeMajor(int mode) const;
    void enqueueNodeMajorLevel(int m, int buf, const double* dBoxes, uint32_t nq, bool wantLevels);
    // Node-major KNN completion: pair lists (query, node) per level, their grouping by node, the raw
    // candidates of the point level and the clusters wave 1 read per query.
    uint32_t probeBeam_ = 32;
    bool knnNodeMajor_ = true;
    DeviceMem pairQ_[2], pairNode_[2], pairList_, pairNodeOff_, pairUnitOff_, pairUnitNode_;
    DeviceMem candQ_, candId_, candD2_, excl_, probeK_;
    uint64_t pairCap_ = 0, candCap_ = 0;
    size_t offKnnTick_ = 0, offQcountP_ = 0, offCandCursor_ = 0;
    std::vector<size_t> offKnnNodeCnt_;  // per mesh m <= height-2: nodeCnt then cursor, in zeroBlock_
    void reserveKnnMajor(uint32_t nq);
    bool growKnnMajor();                 // after an overflow: true when a capacity grew
    DeviceMem resIds_, resVals_, resQ_, resDist_;
    DeviceMem zeroBlock_;  // desc | tickets | status | hdrs | qcount | levelItems
    uint64_t splitLimit_ = 0xffffffffull;
    DeviceMem cmpCnt_, cmpKids_, cmpEntryOff_, cmpKidOff_;  // frontier compaction scratch (per query)
    DeviceMem offsets_;
    DeviceMem boxF_;  // exact range batches: the query boxes as outward-rounded floats
    DeviceMem tau_, candOff_, knnCount_, knnOff_, knnIds_, knnD2_;
    uint64_t knnCap_ = 0;
    bool lastKnn_ = false;
    bool lastCompletion_ = false;  // the last KNN batch ran the node-major completion
    // Two-wave final level of exact KNN (see enqueueKnn).
    DeviceMem lbE_, scoreE_, sel_, offF_, waveM_, selCount_, selOff_, selIds_, selD2_, candOffB_;
    DeviceMem resIdsB_, resQB_, resDistB_;
    uint64_t entryCap_ = 0, resCapB_ = 0;
    uint32_t knnQcap_ = 0;
    size_t offQcountF_ = 0, offQcountB_ = 0, offWork_ = 0;
    int lastKnnBuf_ = 0;
    uint32_t lastRuns_ = 0;  // enqueues of the last synchronous batch (1 + growth reruns)
    void reserveKnn(uint32_t nq);
    size_t zeroBytes_ = 0;
    // offsets into zeroBlock_
    size_t offDesc_ = 0, offTickets_ = 0, offStatus_ = 0, offHdr_ = 0, offQcount_ = 0, offLevels_ = 0;
    uint64_t tileCap_ = 0;

    void growFromHeaders();
    void checkSplitLimit();  // throws SplitBatch when the last batch's levels exceed splitLimit_
    void enqueueLaunches(const double* dBoxes, uint32_t nq, int mode, unsigned flags);
    void dropGraph();
    bool timing_ = false;
    bool capturing_ = false;
    bool twoWave_ = true;
    double waveScale_ = 16.0;
    uint32_t refineStride_ = 16;
    uint32_t refineStages_ = 2;
    bool knnGroups_ = true;
    DeviceMem candOffS_;
    EntryScorer scorer_ = nullptr;
    void* scorerCtx_ = nullptr;
    std::vector<int> variants_;
    std::vector<int> grids_;
    void record(int i);
    std::vector<cudaEvent_t> events_;
    cudaGraphExec_t graphExec_ = nullptr;
    uint64_t graphKernels_ = 0, graphNodes_ = 0;
    struct GraphKey {
        const double* boxes = nullptr;
        uint32_t nq = 0;
        int mode = -1;
        unsigned flags = 0;
        bool timing = false;
        bool operator==(const GraphKey& o) const {
            return boxes == o.boxes && nq == o.nq && mode == o.mode && flags == o.flags && timing == o.timing;
        }
    } graphKey_;
    FrontierIn inView(int buf, uint32_t* hdr) const;
    FrontierOut outView(int buf, uint32_t* hdr) const;
    uint32_t* hdrPtr(int level) const;
};

}  // namespace tblaeq
