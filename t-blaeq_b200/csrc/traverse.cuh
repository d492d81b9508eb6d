// Level-synchronous traversal kernels for the T-BLAEQ hierarchy on sm_100a.
//
// One kernel, `expand`, does the whole per-level pipeline of the reference
// (prune -> compact -> SpTSpM -> refactor, src/core/strategies/L0Strategy.cu:50-191) for every
// query of a batch at once:
//
//   * work items are (frontier entry, child) pairs, laid out as a flat index space whose prefix
//     over entries (`cpre`) was produced by the previous level; a tile of kTile items finds its
//     entries through `tileStart` (also written by the producer), so no global search is needed;
//   * each item rebuilds its child's coordinates y = P[j] (*) x_parent exactly like
//     SpMSpVKernelAOS_v2 (src/Kernel/SpMSpV.cuh:47-67: one rounded multiply per dimension);
//   * the item is kept or dropped by the predicate of the child's level (range box vs radius,
//     a precomputed mask, or the exact final filter);
//   * kept items are compacted in order (warp ballot / shuffle scans inside the tile, a
//     single-pass decoupled look-back across tiles) and written either as the next frontier
//     (with the next level's child prefix and tile starts) or as final result ids (Map applied,
//     src/Query/Refactor.cu:10-16).
//
// Each warp works alone on a tile of kWarpTile consecutive items (no block-wide barriers): it maps
// items to entries with a ballot and an OR-reduction over the 32 entries that can overlap a 32-item
// round, tests every item in a first pass that keeps one bit per item, publishes its counts through
// the look-back, and only then rebuilds and writes the kept items (a small fraction at every level).
// A tile that kept nothing publishes its empty counts and moves on without waiting for its
// predecessors. Rounds whose 32 items lie in one entry read their consecutive rows (or child boxes)
// as one coalesced block, a 16-byte piece per lane, and combine the pieces' tests by ballot.
// Tiles are claimed through an atomic ticket by a persistent grid, so every tile a look-back waits
// on belongs to a warp that is already running; every spin is bounded and reports a status bit
// instead of hanging.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace tblaeq {

constexpr int kThreads = 256;
constexpr int kWarpTile = 256;  // work items per warp tile (8 rounds of 32)

// Packed per-node record of a child level: pruning radius, first grandchild row and grandchild
// count, read with one 16-byte load per item.
struct __align__(16) NodeRec {
    double rad;
    uint32_t cbeg;
    uint32_t cnt;
};

// Frontier in structure-of-arrays layout.
struct FrontierIn {
    const uint32_t* q;          // query slot of each entry
    const uint32_t* cbeg;       // first child (row index into the child level)
    const uint32_t* cpre;       // exclusive prefix of child counts over the frontier
    const double* x;            // decoded coordinates, count * D
    const uint32_t* tileStart;  // entry holding work item b * kTile
    const uint32_t* hdr;        // [0] = entry count, [1] = total children
    uint32_t cap;               // entry capacity of the arrays above
    uint32_t tileCap;           // tileStart capacity
};

struct FrontierOut {
    uint32_t* q;
    uint32_t* node;             // child key (row index or original id) of the kept entry
    uint32_t* cbeg;
    uint32_t* cpre;
    double* x;
    uint32_t* tileStart;
    uint32_t* hdr;              // written by the tile holding the last item
    uint32_t cap;               // entry capacity
    uint32_t tileCap;           // tileStart capacity
    uint32_t* qcount;           // optional per-query kept-entry counts (atomic)
};

struct ResultOut {
    uint64_t* ids;              // output ids (Map applied)
    double* vals;               // optional decoded coordinates (count * D)
    uint32_t* q;                // optional query slot per result
    double* dist2;              // optional squared distance per result (KNN)
    uint32_t* qcount;           // optional per-query result counts (atomic)
    uint32_t* hdr;              // [0] = total results
    uint32_t cap;
};

// The child level: rows to multiply, and the arrays of the child nodes themselves.
struct ChildLevel {
    const double* rows;         // row j: D factors (P-tensor row, or coordinates with x = 1)
    const uint64_t* keys;       // optional key of row j into the node records (null: key = j)
    const NodeRec* nodes;       // child node records (by key)
    const float* aabb;          // optional box of the points below each child (by key): lo[D] hi[D]
    const uint32_t* leaf;       // finest points below each child (by key), for the KNN bound
    // Two-wave KNN over the last frontier (by input entry): wave 1 keeps every point of the
    // selected entries; wave 2 skips selected entries and entries whose lower bound exceeds tau
    // (without loading their rows) and keeps the points within tau. Null entrySel: the input
    // frontier already holds only the wave's entries (compacted).
    const uint8_t* entrySel;
    const double* entryLb;
    const uint8_t* mask;        // keep flags (by row) for kPredMask
    const uint64_t* outMap;     // final output id of row j (null: id = key)
    // Optional, finest exact range level: the decoded point of row j (the product y above) as D
    // floats rounded to nearest. Compared with the query box rounded outward and inward, a point
    // is decided from these 4·D bytes unless a coordinate lies within float rounding of a face,
    // where the FP64 test on the row decides.
    const float* rowsF;
    // Optional with rowsF: rowsF is in point-group order, and its row j is row perm[j] of `rows` and
    // of outMap (the FP64 test, the output id and the written coordinates use perm[j]).
    const uint32_t* perm;
    int rowsOnHost;             // rows (and possibly outMap) are mapped host memory: plain loads only
};

struct QueryArgs {
    const double* boxes;        // range: per query lo[D] then hi[D]
    const float* boxesF;        // range, exact mode: the same boxes as floats rounded outward
    const float* boxesFi;       // range, exact mode: the boxes as floats rounded inward (lo up, hi down)
    const double* points;       // knn: per query point[D]
    double* tau;                // knn: per query upper bound on the K-th neighbour distance (tightened
                                //      in place with an atomic minimum)
    const uint32_t* k;          // knn: neighbours wanted per query
};

struct Scratch {
    unsigned long long* desc;   // look-back descriptors, one per tile, zeroed before launch
    uint32_t* ticket;           // tile ticket counter, zeroed before launch
    uint32_t* status;           // DeviceStatus bits
    uint32_t* levelItems;       // optional: per-query count of generated children at this level
    unsigned long long* work;   // optional: number of child rows actually loaded and tested
};

enum Pred : int {
    kPredRangeRadius = 0,       // keep child if boxdist^2 <= rad^2 and it has children
    kPredMask = 1,              // keep child if mask[row] (and it has children, frontier output)
    kPredAll = 2,               // keep every child
    kPredRangeBox = 3,          // keep point if lo <= y <= hi on every dimension
    kPredKnnBound = 4,          // keep child if dist - rad <= tau (and it has children)
    kPredKnnPoint = 5,          // keep point if dist2 <= tau^2 (records dist2)
    kPredRangeBoxF = 6,         // kPredRangeBox decided from the points' float copies (child.rowsF,
                                // query.boxesFi), with the FP64 test only near a face: same keeps
    kPredGroupBox = 7,          // keep point group if its float box meets the query's (frontier
                                // output; child.rows null: the entry's coordinates pass through)
};

// Kernel variants an autotuner chooses between per level: rows loaded straight into registers,
// or streamed through a per-warp cp.async ring in shared memory.
// A third choice exists for the inner levels of exact range batches only: kVariantNodeMajor runs the
// level node-major (nodeMajorRangeKernel + a kPredAll expand, see NodeMajorArgs); elsewhere it
// launches as kVariantDirect.
enum Variant : int { kVariantDirect = 0, kVariantStaged = 1, kVariantNodeMajor = 2 };

struct ExpandArgs {
    FrontierIn in;
    ChildLevel child;
    QueryArgs query;
    FrontierOut fout;
    ResultOut rout;
    Scratch scratch;
    int D;
    int useFma;                 // accumulate squared distances with fma (reference kernels' contraction)
    int variant;                // Variant
    int wave;                   // 0: plain; 1 / 2: two-wave KNN final level (see ChildLevel)
    // Failure-detection test hook (set by launchExpand from setLookbackTestHook for range and
    // plugin launches only): tile `withholdTile` never publishes its counts, and look-back spins
    // give up after `spinLimit` polls (0: the default limit).
    uint32_t withholdTile;
    uint32_t spinLimit;
    // Persistent grid as a percentage of the instantiation's full occupancy (resident CTAs per SM x
    // SMs); 0 means 100. An autotuner knob: fewer resident warps contend less on the tile ticket and
    // the look-back, more hide more memory latency.
    int gridPercent;
};

// Launch the expand kernel for dimension D with the given predicate; `toResult` selects the
// result output (final level) instead of the next frontier. gridBlocks <= 0 picks a persistent
// grid sized from the occupancy of the instantiation.
void launchExpand(const ExpandArgs& a, int pred, bool toResult, int gridBlocks, cudaStream_t stream);

// Failure-detection test hook: from now on, every range or per-level plugin expand launch (not
// KNN launches, whose later kernels read the frontier without the status check) leaves tile
// `withholdTile` unpublished and bounds its look-back spins at `spinLimit` polls, so the batch ends
// with kStatusLookbackTimeout instead of results. withholdTile = 0xffffffff (or spinLimit = 0)
// restores normal operation. Process-wide; launches captured in a CUDA graph keep the values they
// were captured with.
void setLookbackTestHook(uint32_t withholdTile, uint32_t spinLimit);

// Tile size (work items per tile) used by every expand instantiation.
inline int expandTile(int) { return kWarpTile; }

// ---- node-major range levels (exact mode) ----------------------------------------------------------
// A frontier level of an exact range batch tests every (query, child) pair. In a frontier the same
// node sits in many queries' entries (a mesh-1 node in about 240 of 4,096 at N = 10M, D = 8), and
// entry by entry every one of them re-reads the node's children. Node-major, a warp takes one node
// and 32 of the queries holding it: each query box stays in registers, each child's float box is
// read once per 32 queries (a broadcast load), and only children that pass it are tested in FP64
// against the radius (the same prefilter and the same radius test as the entry-major kernel, so the
// same children survive). Survivors are appended, in no particular order, to a one-item-per-entry
// frontier (query, child row, the parent's coordinates); an ordinary kPredAll expand of it rebuilds
// the children's coordinates and writes the next frontier.

struct NodeMajorArgs {
    // Input frontier, grouped by node: entry list[nodeOff[n] .. nodeOff[n+1]) hold node n, in units
    // of 32 entries (unitOff[n] = first unit of node n, unitOff[nNodes] = all units). nNodes = 0: the
    // root level (every entry holds the virtual root, whose children are rows 0 .. rootChildren-1).
    const uint32_t* inQ;
    const double* inX;
    const uint32_t* inHdr;
    uint32_t inCap;
    const uint32_t* list;
    const uint32_t* nodeOff;
    const uint32_t* unitOff;
    const uint32_t* unitNode;   // optional: the node of every unit (from the transpose)
    uint32_t nNodes;
    const NodeRec* parents;     // records of the input level's nodes (first child row, child count)
    uint32_t rootChildren;
    // Root level: children per unit (0: all). A root unit is 32 entries and one chunk of the root's
    // children, so that a small batch still spreads over the whole GPU.
    uint32_t rootChunk;
    // The children: rows, float boxes and records (by row).
    const double* rows;
    const float* aabb;
    const NodeRec* children;
    int rowsOnHost;
    // Query boxes: double lo|hi, and as floats rounded outward.
    const double* boxes;
    const float* boxesF;
    // Survivors: the next frontier itself (entries in no particular query order). Each warp appends
    // a batch of survivors through one 64-bit atomic on `counter` (entries in the low half, their
    // children in the high half), so entry positions and child prefixes stay in the same order;
    // out.hdr is written from the counter afterwards (launchFrontierHeader).
    FrontierOut out;
    unsigned long long* counter;  // zeroed before launch
    uint32_t* ticket;           // unit ticket, zeroed before launch
    uint32_t* status;
    uint32_t* levelItems;       // optional per-query generated-children counts
    int D;
};

// Groups the entries of a frontier by node (node keys < nNodes): nodeCnt and cursor (nNodes each)
// must be zero; writes nodeOff / unitOff (nNodes + 1) and list (entries).
// unitNode (optional, unitCap words >= cap / 32 + nNodes): the node of every unit, so a unit's
// node is one load instead of a binary search over unitOff.
void launchNodeTranspose(const uint32_t* node, const uint32_t* hdr, uint32_t cap, uint32_t nNodes, uint32_t* nodeCnt,
                         uint32_t* nodeOff, uint32_t* unitOff, uint32_t* cursor, uint32_t* list, cudaStream_t s,
                         uint32_t* unitNode = nullptr, uint32_t unitCap = 0);
// The node-major test of one level (persistent grid; gridPercent as for the expand kernel).
void launchNodeMajorRange(const NodeMajorArgs& a, int gridPercent, cudaStream_t s);
// hdr[0] / hdr[1] = the entries and children a node-major level appended (its packed counter);
// sets the overflow bits of `status` when they exceed the frontier's capacities.
void launchFrontierHeader(const unsigned long long* counter, uint32_t* hdr, uint32_t cap, uint32_t tileCap,
                          uint32_t* status, cudaStream_t s);
// hdr[0] = hdr[1] = *count: the header of a one-item-per-entry frontier.
void launchOneItemHeader(const uint32_t* count, uint32_t* hdr, cudaStream_t s);
// Moves results written in frontier order (rawIds/rawQ/rawVals, count = *hdr) to their query's slot
// offsets[q] + k (cursor: nq zeros), so every query's results are contiguous.
void launchGroupResults(const uint64_t* rawIds, const uint32_t* rawQ, const double* rawVals, const uint32_t* hdr,
                        uint32_t cap, int D, const uint64_t* offsets, uint32_t* cursor, uint64_t* ids, double* vals,
                        cudaStream_t s);

// Builds a root frontier of `nq` entries, each with `nChildren` children starting at row 0 and
// x = 1 (so the first expand reproduces the coarsest coordinates exactly). Capacities must hold
// nq entries and ceil(nq*nChildren / tile) tile starts.
void launchRootFrontier(uint32_t* q, uint32_t* cbeg, uint32_t* cpre, double* x, uint32_t* tileStart, uint32_t* hdr,
                        uint32_t nq, uint32_t nChildren, int D, int tile, cudaStream_t stream);

// boxesF = the nq query boxes (lo[D] hi[D]) as floats, lower corners rounded down and upper
// corners rounded up; boxesFi (optional) = the same rounded inward (lower up, upper down).
void launchRoundBoxes(const double* boxes, uint32_t nq, int D, float* boxesF, float* boxesFi, cudaStream_t stream);

// Whether the finest range level decides points from their float copies (rowsF) at dimension D.
constexpr bool floatPointsSupported(uint64_t D) { return D == 4 || D == 8 || D == 16; }

// offsets[q] = exclusive scan of counts[0..n), offsets[n] = total (single CTA).
void launchExclusiveScan(const uint32_t* counts, uint64_t* offsets, uint32_t n, cudaStream_t stream);

}  // namespace tblaeq
