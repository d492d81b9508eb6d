// KNN building blocks on the device:
//   * the reference's per-centroid lower bound (src/Query/KNN.cu:9-24) for the per-level plugin;
//   * a sort of (key, label) pairs: bitonic 2048-element tiles in shared memory, then merge-path
//     passes (the reference sorts 512-element tiles on the device and merges them on the host,
//     src/MergeSort/MergeSort.cuh:240-313,628-696);
//   * STEP selection (src/core/strategies/L0Strategy.cu:133-154) as a scan, a max-reduction and a
//     search over the sorted bounds instead of a sequential host loop;
//   * per-query top-K selection of candidate points for exact KNN.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "traverse.cuh"

namespace tblaeq {

// Orderable 64-bit key of a double (total order equal to the numeric order for non-NaN values).
__host__ __device__ inline uint64_t orderKey(double v) {
    uint64_t b;
    memcpy(&b, &v, 8);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

// keys[i] = orderKey(sqrt_rd(|q - vals[i]|^2) - rad(ids[i])), labels[i] = i, cnt[i] / rr[i] = the
// node's child count and lb + 2 * radius (the STEP inputs), for the p entries of a grid.
void launchKnnLowerBound(const uint64_t* ids, const double* vals, uint64_t p, int D, const double* dPoint,
                         const NodeRec* nodes, uint64_t* keys, uint32_t* labels, uint32_t* cnt, double* rr,
                         cudaStream_t s);

// Sorts n (key, label) pairs ascending by (key, label). Uses (keys2, labels2) as scratch of the
// same size; the result ends in (keys, labels).
void sortPairs(uint64_t* keys, uint32_t* labels, uint64_t* keys2, uint32_t* labels2, uint64_t n, cudaStream_t s);

// STEP over sorted pairs: mask[label] = 1 for every selected entry (mask zeroed by the caller).
void launchStep(const uint64_t* keys, const uint32_t* labels, const uint32_t* cnt, const double* rr, uint64_t n,
                uint64_t K, uint8_t* mask, cudaStream_t s);

// Per-query exact top-K: candidates of query q are the concatenation of
// [offA[q], offA[q+1]) in (idsA, d2A) and [offB[q], offB[q+1]) in (idsB, d2B) (B may be null).
// Writes the K[q] (or fewer) smallest by (dist2, id), ascending, to outIds/outD2 starting at
// outOff[q]; outCount[q] receives how many. Status bit kStatusOverflowEntries when a query has
// more candidates than the selection can stage.
// capA / capB are the capacities of the candidate arrays: a query whose candidates lie beyond them
// (the producer overflowed and the host will rerun the batch) is skipped and flagged.
void launchTopK(const uint64_t* offA, const uint64_t* idsA, const double* d2A, uint64_t capA, const uint64_t* offB,
                const uint64_t* idsB, const double* d2B, uint64_t capB, const uint32_t* K, uint32_t nq,
                const uint64_t* outOff, uint64_t* outIds, double* outD2, uint32_t* outCount, uint32_t* status,
                cudaStream_t s);

// Lower bound and ranking score of every entry of the last KNN frontier: lb = max(centre distance -
// subtree radius, distance to the entry's box) (conservative), score = lb.
void launchEntryBounds(const uint32_t* q, const uint32_t* node, const double* x, const uint32_t* hdr, uint32_t cap,
                       int D, const double* points, const NodeRec* nodes, const float* aabb, double* lb, double* score,
                       cudaStream_t s);

// Wave-1 width per query: clamp(ceil(factor * K[q]) + 1, 2, 32) entries.
void launchWaveWidth(const uint32_t* K, uint32_t nq, double factor, uint32_t* M, cudaStream_t s);

// Compacts the last KNN frontier F (query-major) into `out`: mode 1 keeps the selected entries
// (sel), mode 2 the others whose lower bound is within their query's tau. Order is kept; the child
// prefix, tile starts and header (count, children) of `out` are rebuilt, so a wave expands only
// its own entries. Blocks work on fixed segments of F's capacity `cap`; scratch: cnt, kids
// (compactSegments(cap)), entryOff, kidOff (compactSegments(cap) + 1).
void launchCompactFrontier(const FrontierIn& F, uint32_t cap, int mode, const uint8_t* sel, const double* lb,
                           const double* tau, int D, uint32_t* cnt, uint32_t* kids, uint64_t* entryOff,
                           uint64_t* kidOff, const FrontierOut& out, cudaStream_t s);
uint32_t compactSegments(uint64_t cap);

// sel[ids[i]] = 1 for every selected entry position in [0, off[nq]) below cap (positions at or
// above cap come from slots a skipped query never wrote).
void launchScatterSel(const uint64_t* ids, const uint64_t* off, uint32_t nq, uint64_t cap, uint8_t* sel,
                      cudaStream_t s);

// tau[q] = min(tau[q], sqrt(d2 of the K[q]-th candidate) * (1 + 1e-12)) when a query has K[q] of them.
void launchTauFromTopK(const uint64_t* off, const double* d2, const uint32_t* K, uint32_t nq, double* tau,
                       cudaStream_t s);

// out[q] = min(K[q], (offA[q+1] - offA[q]) + (offB[q+1] - offB[q])).
void launchClampCounts2(const uint64_t* offA, const uint64_t* offB, const uint32_t* K, uint32_t nq, uint32_t* out,
                        cudaStream_t s);

// v[i] = value for i < n.
void launchFillDouble(double* v, double value, uint32_t n, cudaStream_t s);

// out[q] = min(K[q], off[q+1] - off[q]).
void launchClampCounts(const uint64_t* off, const uint32_t* K, uint32_t nq, uint32_t* out, cudaStream_t s);

}  // namespace tblaeq

namespace tblaeq {

// ---- Exact KNN completion, node-major (see BatchEngine::enqueueKnn) --------------------------------
// Once wave 1 has bounded every query's K-th distance by tau, every point within tau lies in a
// cluster whose lower bound is within tau, below ancestors whose bounds are within tau too. The
// hierarchy is walked again node-major: a warp takes one node and 32 of the queries holding it
// (query points and tau in registers, every child's decoded centre, box and record read once per
// warp), and the surviving (query, child) pairs form the next level's input. At the cluster level
// a warp loads each of a cluster's points once for 32 queries and keeps the points within tau, so
// a cluster's rows are read once per batch per 32 of its queries instead of once per query.

// One bound level (children of mesh m). Input pairs (query, node of mesh m-1) grouped by node
// through list / nodeOff / unitOff (nNodes = 0: the root level, every query with the virtual root).
struct KnnBoundLevelArgs {
    const uint32_t* inQ;
    const uint32_t* inCount;
    uint32_t inCap;
    uint32_t nq;
    const uint32_t* list;
    const uint32_t* nodeOff;
    const uint32_t* unitOff;
    const uint32_t* unitNode;    // optional: the node of every unit (from the transpose)
    uint32_t nNodes;
    const NodeRec* parents;
    uint32_t rootChildren;
    const double* x;           // decoded centres of the children (mesh m)
    const float* aabb;         // their point boxes
    const NodeRec* nodes;      // their subtree radius and child counts
    const double* points;
    const double* tau;
    uint32_t* outQ;            // surviving pairs
    uint32_t* outNode;
    uint32_t outCap;
    uint32_t* outCount;
    uint32_t* ticket;
    uint32_t* status;
    int D;
};
void launchKnnBoundLevel(const KnnBoundLevelArgs& a, cudaStream_t s);

// The point level: pairs (query, cluster) grouped by cluster; every point of the cluster within
// tau of the query (squared FP64 distance <= tau^2 (1 + 1e-9), accumulated like the expand kernel's
// point test) becomes a candidate (query, id, squared distance), except in the clusters wave 1
// already read for that query (excl: per query exclStride cluster positions, ~0 for none).
struct KnnClusterArgs {
    const uint32_t* inQ;
    const uint32_t* inCount;
    uint32_t inCap;
    const uint32_t* list;
    const uint32_t* nodeOff;
    const uint32_t* unitOff;
    const uint32_t* unitNode;    // optional: the node of every unit (from the transpose)
    uint32_t nNodes;
    const NodeRec* clusters;
    const double* x;
    const double* rows;
    int rowsOnHost;
    const double* decoded;  // optional: the decoded finest points (else rebuilt from rows and x)
    // With decoded: perm non-null means decoded is in point-group order (perm maps a position to
    // its row, for the output id); the groups, when given, are walked with their boxes.
    const uint32_t* perm;
    const NodeRec* clusterGroups;  // per cluster: {-, first group, groups}
    const NodeRec* groupRec;       // per group: {-, first position, points}
    const float* groupBox;         // per group: lo[D] hi[D], rounded outward
    // Test only every sampleStride-th point of each cluster (0 or 1: every point). Lanes whose
    // cluster's lower bound (centre distance - subtree radius) already exceeds the query's bound
    // skip the cluster either way.
    uint32_t sampleStride;
    const uint64_t* map;
    const double* points;
    const double* tau;
    const uint32_t* excl;
    uint32_t exclStride;
    uint32_t* outQ;
    uint64_t* outId;
    double* outD2;
    uint32_t outCap;
    uint32_t* outCount;
    uint32_t* qcount;
    unsigned long long* work;  // optional: point rows tested
    uint32_t* ticket;
    uint32_t* status;
    int D;
};
void launchKnnClusterPoints(const KnnClusterArgs& a, cudaStream_t s);

// Keeps the (query, cluster) pairs whose cluster sphere (centre distance - subtree radius, with the
// point kernel's slack) is within the query's current bound and whose cluster wave 1 did not read,
// appending them (no particular order) to outQ/outNode through outCount; the units the point
// kernel forms from them afterwards are full of live lanes again.
struct KnnFilterArgs {
    const uint32_t* inQ;
    const uint32_t* inNode;
    const uint32_t* inCount;
    uint32_t inCap;
    const NodeRec* clusters;
    const double* x;
    const double* points;
    const double* tau;
    const uint32_t* excl;
    uint32_t exclStride;
    uint32_t* outQ;
    uint32_t* outNode;
    uint32_t outCap;
    uint32_t* outCount;
    uint32_t* status;
    int D;
};
void launchKnnFilterPairs(const KnnFilterArgs& a, cudaStream_t s);

// excl[q * stride + i] = node[selIds[selOff[q] + i]] for the selCount[q] entries wave 1 read, ~0
// for the rest of the row.
void launchWaveOneClusters(const uint64_t* selIds, const uint64_t* selOff, const uint32_t* selCount,
                           const uint32_t* node, uint64_t cap, uint32_t nq, uint32_t stride, uint32_t* excl,
                           cudaStream_t s);

// v[i] = value for i < n.
void launchFillU32(uint32_t* v, uint32_t value, uint32_t n, cudaStream_t s);

}  // namespace tblaeq
