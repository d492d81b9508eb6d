// Level-synchronous traversal kernels (see traverse.cuh for the design).
#include "traverse.cuh"

#include <cuda/atomic>

#include <algorithm>
#include <atomic>

namespace tblaeq {

namespace {

constexpr uint32_t kFlagAggregate = 1;
constexpr uint32_t kFlagPrefix = 2;
constexpr uint32_t kMaxCount30 = (1u << 30) - 1;
constexpr uint32_t kSpinLimit = 1u << 21;  // ~0.2-2 s of polling before giving up

__device__ __forceinline__ unsigned long long packDesc(uint32_t flag, uint32_t cnt, uint32_t sum) {
    return (static_cast<unsigned long long>(flag) << 62) |
           (static_cast<unsigned long long>(cnt & kMaxCount30) << 32) | sum;
}

__device__ __forceinline__ unsigned long long loadDesc(unsigned long long* p) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*p);
    return r.load(cuda::memory_order_relaxed);
}

__device__ __forceinline__ void storeDesc(unsigned long long* p, unsigned long long v) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*p);
    r.store(v, cuda::memory_order_relaxed);
}

// Warp 0 of the tile: publish the tile aggregate, look back over predecessors and publish the
// inclusive prefix. Returns the exclusive prefix (count, child sum) in lanes of warp 0.
__device__ void lookback(unsigned long long* desc, uint32_t tile, uint32_t aggCnt, uint32_t aggSum,
                         uint32_t* status, uint32_t spinLimit, unsigned long long& exCnt, unsigned long long& exSum) {
    const int lane = threadIdx.x & 31;
    exCnt = 0;
    exSum = 0;
    if (tile == 0) {
        if (lane == 0) storeDesc(&desc[0], packDesc(kFlagPrefix, aggCnt, aggSum));
        return;
    }
    if (lane == 0) storeDesc(&desc[tile], packDesc(kFlagAggregate, aggCnt, aggSum));
    long long pred = static_cast<long long>(tile) - 1;
    uint32_t spins = 0;
    while (true) {
        const long long idx = pred - lane;
        const unsigned long long v = (idx >= 0) ? loadDesc(&desc[idx]) : packDesc(kFlagPrefix, 0, 0);
        const uint32_t flag = static_cast<uint32_t>(v >> 62);
        const uint32_t pmask = __ballot_sync(0xffffffffu, flag == kFlagPrefix);
        const uint32_t xmask = __ballot_sync(0xffffffffu, flag == 0);
        const uint32_t needed = pmask ? ((pmask & (~pmask + 1)) << 1) - 1 : 0xffffffffu;  // lanes <= first P
        if (xmask & needed) {
            if (++spins > spinLimit) {
                if (lane == 0) atomicOr(status, kStatusLookbackTimeout);
                break;
            }
            __nanosleep(64);
            continue;
        }
        unsigned long long c = (needed >> lane) & 1u ? (v >> 32) & kMaxCount30 : 0;
        unsigned long long s = (needed >> lane) & 1u ? (v & 0xffffffffull) : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            c += __shfl_xor_sync(0xffffffffu, c, o);
            s += __shfl_xor_sync(0xffffffffu, s, o);
        }
        exCnt += c;
        exSum += s;
        if (pmask) break;
        pred -= 32;
    }
    const unsigned long long incCnt = exCnt + aggCnt;
    const unsigned long long incSum = exSum + aggSum;
    if (lane == 0) {
        if (incCnt > kMaxCount30) atomicOr(status, kStatusOverflowEntries);
        if (incSum > 0xffffffffull) atomicOr(status, kStatusOverflowSum);
        storeDesc(&desc[tile], packDesc(kFlagPrefix, static_cast<uint32_t>(incCnt),
                                        static_cast<uint32_t>(incSum)));
    }
}

// Items are evaluated chunk by chunk: child rows, parent coordinates, query boxes and points are
// read 2 or 4 doubles at a time (16-byte loads; every such row starts on a 16-byte boundary when D
// is even) and consumed at once, so no per-item D-vector stays live in registers.
template <int D>
constexpr int chunkOf() {
    return (D > 0 && D % 4 == 0) ? 4 : ((D > 0 && D % 2 == 0) ? 2 : 1);
}

// v[0..C) = p[0..C); SMEM selects a plain (shared-memory) load over the read-only global path.
template <int C, bool SMEM>
__device__ __forceinline__ void ldChunk(const double* p, double (&v)[C]) {
    if constexpr (C == 1) {
        v[0] = SMEM ? *p : __ldg(p);
    } else {
#pragma unroll
        for (int i = 0; i < C; i += 2) {
            const double2 t = SMEM ? *reinterpret_cast<const double2*>(p + i)
                                   : __ldg(reinterpret_cast<const double2*>(p + i));
            v[i] = t.x;
            v[i + 1] = t.y;
        }
    }
}

template <int C>
__device__ __forceinline__ void ldChunkF(const float* p, float (&v)[C]) {
    if constexpr (C == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    } else if constexpr (C == 2) {
        const float2 t = __ldg(reinterpret_cast<const float2*>(p));
        v[0] = t.x;
        v[1] = t.y;
    } else {
        v[0] = __ldg(p);
    }
}

template <int C>
__device__ __forceinline__ void stChunk(double* p, const double (&v)[C]) {
    if constexpr (C == 1) {
        *p = v[0];
    } else {
#pragma unroll
        for (int i = 0; i < C; i += 2) *reinterpret_cast<double2*>(p + i) = make_double2(v[i], v[i + 1]);
    }
}

// One dimension of the squared distance from y to the box [l, h], accumulated like the
// reference (RangePruning.cu:7-20; nvcc contracts `dist += diff * diff` into an fma by default).
__device__ __forceinline__ double boxGapAcc(double y, double l, double h, double dist, int useFma) {
    double diff = 0.0;
    if (y < l) {
        diff = l - y;
    } else if (y > h) {
        diff = y - h;
    }
    return useFma ? __fma_rn(diff, diff, dist) : __dadd_rn(dist, __dmul_rn(diff, diff));
}

// Rebuilds item (entry e, row j) chunk by chunk, y = rows[j] (*) x_e with one rounded multiply
// per dimension (SpMSpV.cuh:47-67), and hands each chunk to sink(d, y).
template <int D, int DM, typename Sink>
__device__ __forceinline__ void rebuildChunks(const ExpandArgs& a, int dim, uint32_t e, uint32_t j, Sink&& sink) {
    constexpr int C = chunkOf<D>();
    const double* xp = a.in.x + static_cast<size_t>(e) * dim;
    const double* rp = a.child.rows ? a.child.rows + static_cast<size_t>(j) * dim : nullptr;
#pragma unroll
    for (int d = 0; d < DM; d += C) {
        if (D > 0 || d < dim) {
            double r[C], x[C], y[C];
            ldChunk<C, false>(xp + d, x);
            if (rp) {  // warp-uniform; no rows: the child takes its parent's coordinates (point groups)
                ldChunk<C, false>(rp + d, r);
#pragma unroll
                for (int i = 0; i < C; ++i) y[i] = __dmul_rn(r[i], x[i]);
            } else {
#pragma unroll
                for (int i = 0; i < C; ++i) y[i] = x[i];
            }
            sink(d, y);
        }
    }
}

// Shared-memory staging of child rows: every lane copies its own row with cp.async into a
// per-warp ring of kStages rounds, so several rounds of loads are in flight per warp without
// holding them in registers. Rows of even D move in 16-byte chunks with a padded stride (an odd
// number of 16-byte chunks, so the eight lanes of a 128-bit shared-memory phase hit distinct
// banks); rows of odd D move in 8-byte chunks (their 8*D-byte stride is already conflict-free).
template <int D, bool STAGED>
struct Staging {
    static constexpr bool kOn = STAGED && D > 0;
    static constexpr int kChunk = (D % 2 == 0) ? 16 : 8;
    static constexpr int kChunks = kOn ? (8 * D) / kChunk : 0;
    static constexpr int kStride = !kOn ? 0 : ((kChunk == 16 && (kChunks % 2) == 0) ? 8 * D + 16 : 8 * D);
    static constexpr int kStages = 4;
    static constexpr int kRounds = kWarpTile / 32;
    static constexpr int kRowBytes = kOn ? kStages * 32 * kStride : 0;
    static constexpr int kNodeBytes = kOn ? kStages * 32 * 16 : 0;
    static constexpr int kCacheBytes = kRounds * 32 * (4 + 2);  // per item: row (u32), window slot (u16)
    static constexpr int kWindow = kWarpTile + 1;  // most entries a tile can overlap
    static constexpr int kWindowBytes = 3 * kWindow * 4 + 4;
    static constexpr int kWarpBytes = kRowBytes + kNodeBytes + kCacheBytes + ((kWindowBytes + 15) / 16) * 16;
    // Range frontier levels only (kept out of the others' shared memory, which would shrink their
    // L1): the tile's prefilter survivors (item indices) and their keep bits.
    static constexpr int kDeferBytes = kWarpTile * 2 + kRounds * 4;
};

template <int D, bool STAGED, int PRED>
constexpr int warpSmemBytes() {
    return Staging<D, STAGED>::kWarpBytes + (PRED == kPredRangeRadius ? Staging<D, STAGED>::kDeferBytes : 0);
}

// Launch shape of the expand kernels (independent warps per CTA and the register bound). These are
// build-time tuning knobs; the defaults are the fastest measured on B200 for the benchmark index.
#ifndef TBLAEQ_EXPAND_THREADS
#define TBLAEQ_EXPAND_THREADS 128
#endif
#ifndef TBLAEQ_EXPAND_MIN_BLOCKS
#define TBLAEQ_EXPAND_MIN_BLOCKS 10
#endif
#ifndef TBLAEQ_EXPAND_MIN_BLOCKS_BOUND
#define TBLAEQ_EXPAND_MIN_BLOCKS_BOUND 8
#endif
// Unroll factors of the per-round loops of the range levels (build-time knobs, like the launch
// shape): the item test of levels that output a frontier, and pass 2 of every range level.
// Measured on B200: fully unrolled, the range frontier levels stall on instruction fetch (their
// loop body holds the box prefilter, the radius test, the node loads and the frontier writes);
// with the test unrolled twice and pass 2 rolled, the mesh-2 range level went from 0.65 to 0.45 ms;
// a rolled pass 2 also frees registers at the finest range level. The KNN levels stay fully
// unrolled: their pass 2 is hot (wave 1 writes every point of its clusters) and the batched KNN
// step measured about 8% slower rolled. The test loop of point levels and the item-to-entry
// mapping stay fully unrolled everywhere.
#ifndef TBLAEQ_UNROLL_FRONTIER_TEST
#define TBLAEQ_UNROLL_FRONTIER_TEST 2
#endif
#ifndef TBLAEQ_UNROLL_PASS2
#define TBLAEQ_UNROLL_PASS2 1
#endif
// The finest exact range level with float points (kPredRangeBoxF).
#ifndef TBLAEQ_UNROLL_FLOAT_TEST
#define TBLAEQ_UNROLL_FLOAT_TEST 2
#endif
constexpr int kExpandThreads = TBLAEQ_EXPAND_THREADS;

// Resident CTAs per SM the register allocation is sized for (128 threads: 10 CTAs = 51 registers,
// 8 CTAs = 64). Levels that prune inner nodes (range radius + box, KNN sphere + box bounds) keep
// more state live and get the larger budget; point levels and plain expansions the smaller one.
#ifndef TBLAEQ_EXPAND_MIN_BLOCKS_BOX
#define TBLAEQ_EXPAND_MIN_BLOCKS_BOX 10
#endif
template <int PRED>
constexpr int expandMinBlocks() {
    return (PRED == kPredKnnBound || PRED == kPredRangeRadius) ? TBLAEQ_EXPAND_MIN_BLOCKS_BOUND
           : (PRED == kPredRangeBox || PRED == kPredRangeBoxF) ? TBLAEQ_EXPAND_MIN_BLOCKS_BOX
                                                               : TBLAEQ_EXPAND_MIN_BLOCKS;
}

template <int D, bool STAGED, int PRED>
constexpr size_t expandSmemBytes() {
    return static_cast<size_t>(warpSmemBytes<D, STAGED, PRED>()) * (kExpandThreads / 32);
}

__device__ __forceinline__ void cpAsync16(void* dst, const void* src) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cpAsync8(void* dst, const void* src) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpAsyncWait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Bulk L2 prefetch of a contiguous byte range (16-byte aligned start, size a multiple of 16).
__device__ __forceinline__ void bulkPrefetchL2(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}

// Whether a level's kernel prefetches its tile's rows: predicates that read every child row, for
// row sizes that keep every row on a 16-byte boundary.
template <int D, int PRED>
constexpr bool prefetchesRows() {
    return D > 0 && (8 * D) % 16 == 0 &&
           (PRED == kPredRangeBox || PRED == kPredRangeBoxF || PRED == kPredKnnPoint || PRED == kPredKnnBound ||
            PRED == kPredRangeRadius);
}

// Prefetches into L2 the child rows of tile `t`: one contiguous run per frontier entry that the
// tile overlaps, one bulk prefetch per run (lanes take entries in turn). Levels that decide most
// children without loading their rows (the box prefilter, two-wave KNN) prefetch nothing.
template <int D, int PRED>
__device__ __forceinline__ void prefetchTileRows(const ExpandArgs& a, uint32_t t, uint32_t nTiles, uint32_t entries,
                                                 uint32_t total, int lane, bool floatRows) {
    if (t >= nTiles) return;
    if (a.child.rowsOnHost && !floatRows) return;  // bulk prefetches are for device memory
    if (PRED == kPredRangeRadius && a.child.aabb) return;
    if (PRED == kPredKnnPoint && a.wave != 0 && a.child.entrySel) return;
    const uint32_t t0 = t * kWarpTile;
    const uint32_t itemEnd = min(t0 + static_cast<uint32_t>(kWarpTile), total);
    const uint32_t eLo = a.in.tileStart[t];
    uint32_t eHi = (t + 1 < nTiles) ? a.in.tileStart[t + 1] : entries - 1;
    if (eHi >= entries) eHi = entries - 1;
    // The finest exact range level with float points reads those (4·D bytes a row) instead.
    const bool f = floatRows;
    const unsigned char* base = f ? reinterpret_cast<const unsigned char*>(a.child.rowsF)
                                  : reinterpret_cast<const unsigned char*>(a.child.rows);
    const uint32_t rowBytes = f ? 4u * D : 8u * D;
    for (uint32_t e = eLo + lane; e <= eHi; e += 32) {
        const uint32_t cpi = a.in.cpre[e];
        const uint32_t from = max(t0, cpi);
        const uint32_t to = (e + 1 < entries) ? min(itemEnd, a.in.cpre[e + 1]) : itemEnd;
        if (to > from) {
            const unsigned char* src = base + (static_cast<size_t>(a.in.cbeg[e]) + (from - cpi)) * rowBytes;
            bulkPrefetchL2(src, (to - from) * rowBytes);
        }
    }
}

template <int PRED, bool TO_RESULT>
constexpr bool needsNode() {
    return PRED == kPredRangeRadius || PRED == kPredKnnBound || PRED == kPredGroupBox ||
           (!TO_RESULT && (PRED == kPredMask || PRED == kPredAll));
}

// Exact-mode prefilter of range levels: whether the query box meets the box of the points below
// child kk. Both boxes are floats rounded outward (the child's when the index is loaded, the
// query's once per batch), so the test never rejects a child whose points meet the query box. It
// reads 2*D floats of the child and 2*D of the query (one address per warp, mostly) instead of the
// child's row, the parent's coordinates and the double query box, and rejects most children.
template <int D, int DM>
__device__ __forceinline__ bool aabbMeets(const ExpandArgs& a, int dim, uint32_t kk, uint32_t q) {
    constexpr int C = chunkOf<D>();
    const float* b = a.child.aabb + static_cast<size_t>(kk) * 2 * dim;
    const float* f = a.query.boxesF + static_cast<size_t>(q) * 2 * dim;
    bool meets = true;
#pragma unroll
    for (int d = 0; d < DM; d += C) {
        if (D > 0 || d < dim) {
            float bl[C], bh[C], ql[C], qh[C];
            ldChunkF<C>(b + d, bl);
            ldChunkF<C>(b + dim + d, bh);
            ldChunkF<C>(f + d, ql);
            ldChunkF<C>(f + dim + d, qh);
#pragma unroll
            for (int i = 0; i < C; ++i) meets = meets && bl[i] <= qh[i] && bh[i] >= ql[i];
        }
    }
    return meets;
}

// Pass-1 test of one item: entry coordinates xp, child row j (read from `rowp`: global memory, or
// the shared-memory staging ring when SMEM) and child key kk, for query q. Rebuilds the child's
// coordinates chunk by chunk and applies the level predicate; cc receives the child's own child
// count when the output is a frontier.
template <int D, int DM, int PRED, bool TO_RESULT, bool SMEM>
__device__ __forceinline__ bool evalItem(const ExpandArgs& a, int dim, const double* rowp, const double* xp,
                                         uint32_t q, uint32_t j, uint32_t kk, const NodeRec& nr, uint32_t& cc) {
    constexpr int C = chunkOf<D>();
    cc = 0;
    if constexpr (PRED == kPredMask) {
        bool keep = a.child.mask[j] != 0;
        if constexpr (!TO_RESULT) {
            cc = nr.cnt;
            keep = keep && cc > 0;
        }
        return keep;
    } else if constexpr (PRED == kPredGroupBox) {
        cc = nr.cnt;
        return cc > 0 && aabbMeets<D, DM>(a, dim, kk, q);
    } else if constexpr (PRED == kPredAll) {
        if constexpr (!TO_RESULT) {
            cc = nr.cnt;
            return cc > 0;
        }
        return true;
    } else if constexpr (PRED == kPredRangeRadius || PRED == kPredRangeBox || PRED == kPredRangeBoxF) {
        const double* box = a.query.boxes + static_cast<size_t>(q) * 2 * dim;
        double dist = 0.0;
        bool in = true;
#pragma unroll
        for (int d = 0; d < DM; d += C) {
            if (D > 0 || d < dim) {
                double r[C], x[C], l[C], h[C];
                ldChunk<C, SMEM>(rowp + d, r);
                ldChunk<C, false>(xp + d, x);
                ldChunk<C, false>(box + d, l);
                ldChunk<C, false>(box + dim + d, h);
#pragma unroll
                for (int i = 0; i < C; ++i) {
                    const double y = __dmul_rn(r[i], x[i]);
                    if constexpr (PRED == kPredRangeRadius) {
                        dist = boxGapAcc(y, l[i], h[i], dist, a.useFma);
                    } else {
                        in = in && (l[i] <= y) && (y <= h[i]);
                    }
                }
            }
        }
        if constexpr (PRED == kPredRangeRadius) {
            cc = nr.cnt;
            return (cc > 0) && (dist <= __dmul_rn(nr.rad, nr.rad));
        } else {
            return in;
        }
    } else if constexpr (PRED == kPredKnnBound) {
        // Distance bounds of the points below the child: sphere (centre distance -/+ subtree radius)
        // and, when present, its box (outward-rounded, so slightly widened bounds stay conservative).
        const double* p = a.query.points + static_cast<size_t>(q) * dim;
        const float* b = a.child.aabb ? a.child.aabb + static_cast<size_t>(kk) * 2 * dim : nullptr;
        double dist = 0.0, gapSum = 0.0, farSum = 0.0;
#pragma unroll
        for (int d = 0; d < DM; d += C) {
            if (D > 0 || d < dim) {
                double r[C], x[C], pp[C];
                float bl[C], bh[C];
                ldChunk<C, SMEM>(rowp + d, r);
                ldChunk<C, false>(xp + d, x);
                ldChunk<C, false>(p + d, pp);
                if (b) {
                    ldChunkF<C>(b + d, bl);
                    ldChunkF<C>(b + dim + d, bh);
                }
#pragma unroll
                for (int i = 0; i < C; ++i) {
                    const double diff = pp[i] - __dmul_rn(r[i], x[i]);
                    dist = __fma_rn(diff, diff, dist);
                    if (b) {
                        const double l = static_cast<double>(bl[i]), h = static_cast<double>(bh[i]);
                        const double g = fmax(fmax(l - pp[i], pp[i] - h), 0.0);
                        const double f = fmax(pp[i] - l, h - pp[i]);
                        gapSum = __fma_rn(g, g, gapSum);
                        farSum = __fma_rn(f, f, farSum);
                    }
                }
            }
        }
        const double dd = sqrt(dist);
        double lb = dd - nr.rad, ub = dd + nr.rad;
        if (b) {
            lb = fmax(lb, sqrt(gapSum) * (1.0 - 1e-12));
            ub = fmin(ub, sqrt(farSum) * (1.0 + 1e-12));
        }
        cc = nr.cnt;
        double tau = __ldcg(a.query.tau + q);
        // Any child with K points below it bounds the K-th neighbour distance by its far distance.
        if (ub < tau && __ldg(a.child.leaf + kk) >= __ldg(a.query.k + q)) {
            atomicMin(reinterpret_cast<unsigned long long*>(a.query.tau + q), __double_as_longlong(ub));
            tau = ub;
        }
        return (cc > 0) && (lb <= tau);
    } else {  // kPredKnnPoint
        if (a.wave == 1) return true;  // every point of a selected entry
        const double* p = a.query.points + static_cast<size_t>(q) * dim;
        double dist = 0.0;
#pragma unroll
        for (int d = 0; d < DM; d += C) {
            if (D > 0 || d < dim) {
                double r[C], x[C], pp[C];
                ldChunk<C, SMEM>(rowp + d, r);
                ldChunk<C, false>(xp + d, x);
                ldChunk<C, false>(p + d, pp);
#pragma unroll
                for (int i = 0; i < C; ++i) {
                    const double diff = pp[i] - __dmul_rn(r[i], x[i]);
                    dist = __fma_rn(diff, diff, dist);
                }
            }
        }
        const double t = __ldcg(a.query.tau + q);
        return dist <= t * t * (1.0 + 1e-9);
    }
}

// Row pieces each lane keeps in flight in singleEntryRangeBox. Measured on B200 (finest range
// level, D = 8): 2 pieces 0.322 ms, all 4 pieces of the round 0.303 ms, although the latter spills
// 72 bytes (outside the fast path) at the point levels' 48-register bound.
#ifndef TBLAEQ_FAST_PIECES
#define TBLAEQ_FAST_PIECES 4
#endif
// Finest range level, a round whose 32 items all belong to one frontier entry: the items' rows
// are 32 consecutive P rows, so the warp reads them as one contiguous block, each lane taking one
// 16-byte piece (two dimensions) of a row per load, and tests its piece against the same two
// dimensions of the entry's coordinates and query box (constant over the round). A ballot per
// load collects the pieces; an item is kept when all D/2 pieces of its row are inside the box.
// Same products and comparisons as evalItem, so the kept set is identical. Returns whether the
// calling lane's own item (item `lane` of the round) is kept.
template <int D>
constexpr bool coalescedBox() {
    return D >= 4 && D % 2 == 0 && 32 % (D >= 2 ? D / 2 : 1) == 0;
}
template <int D>
__device__ __forceinline__ bool singleEntryRangeBox(const ExpandArgs& a, uint32_t j0, uint32_t e, uint32_t q,
                                                    int lane) {
    constexpr int L = D / 2;   // lanes (16-byte pieces) per row
    constexpr int G = 32 / L;  // rows per load
    constexpr uint32_t kAll = (1u << L) - 1u;
    const int c = lane % L;
    const double2* rows2 = reinterpret_cast<const double2*>(a.child.rows + static_cast<size_t>(j0) * D);
    const double2 xv = __ldg(reinterpret_cast<const double2*>(a.in.x + static_cast<size_t>(e) * D) + c);
    const double* box = a.query.boxes + static_cast<size_t>(q) * 2 * D;
    const double2 lo = __ldg(reinterpret_cast<const double2*>(box) + c);
    const double2 hi = __ldg(reinterpret_cast<const double2*>(box + D) + c);
    // Loads in flight per lane (TBLAEQ_FAST_PIECES).
    constexpr int P = L >= TBLAEQ_FAST_PIECES ? TBLAEQ_FAST_PIECES : L;
    uint32_t mine = 0;
#pragma unroll 1
    for (int s0 = 0; s0 < L; s0 += P) {
        double2 rv[P];
        // Mapped host rows (a streamed interval) take plain loads; the block is just as contiguous,
        // so each load instruction still moves whole lines across the host link.
#pragma unroll
        for (int i = 0; i < P; ++i)
            rv[i] = a.child.rowsOnHost ? rows2[(s0 + i) * 32 + lane] : __ldg(rows2 + (s0 + i) * 32 + lane);
#pragma unroll
        for (int i = 0; i < P; ++i) {
            const double y0 = __dmul_rn(rv[i].x, xv.x), y1 = __dmul_rn(rv[i].y, xv.y);
            const bool pass = (lo.x <= y0) & (y0 <= hi.x) & (lo.y <= y1) & (y1 <= hi.y);
            const uint32_t b = __ballot_sync(0xffffffffu, pass);
            if (s0 + i == lane / G) mine = b;
        }
    }
    return ((mine >> ((lane % G) * L)) & kAll) == kAll;
}

// The FP64 test of one finest point (row j below entry e) against query q's box: the products and
// comparisons of evalItem's kPredRangeBox branch. Out of line: it is rare, and inlined its registers
// would count against the float test around it.
template <int D>
__device__ __noinline__ bool exactPointInBoxRow(const double* r, const double* x, const double* box) {
    bool in = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const double y = __dmul_rn(__ldg(r + d), __ldg(x + d));
        in = in && (__ldg(box + d) <= y) && (y <= __ldg(box + D + d));
    }
    return in;
}
template <int D>
__device__ __forceinline__ bool exactPointInBox(const ExpandArgs& a, uint32_t j, uint32_t e, uint32_t q) {
    const uint32_t jr = a.child.perm ? __ldg(a.child.perm + j) : j;
    return exactPointInBoxRow<D>(a.child.rows + static_cast<size_t>(jr) * D, a.in.x + static_cast<size_t>(e) * D,
                                 a.query.boxes + static_cast<size_t>(q) * 2 * D);
}

// Float decisions of one 4-dimension piece of a point: `in` when every coordinate lies strictly
// inside the inward-rounded box (then the exact coordinate lies inside the box), `out` when one
// lies outside the outward-rounded box (then the exact one lies outside). Rounding to nearest is
// monotone, which gives both implications; a piece that is neither is undecided.
__device__ __forceinline__ void pieceF(const float4 v, const float4 lo, const float4 hi, const float4 li,
                                       const float4 hiI, bool& in, bool& out) {
    in = (v.x > li.x) & (v.y > li.y) & (v.z > li.z) & (v.w > li.w) & (v.x < hiI.x) & (v.y < hiI.y) &
         (v.z < hiI.z) & (v.w < hiI.w);
    out = (v.x < lo.x) | (v.y < lo.y) | (v.z < lo.z) | (v.w < lo.w) | (v.x > hi.x) | (v.y > hi.y) |
          (v.z > hi.z) | (v.w > hi.w);
}

// Finest exact range level, one item tested from its float point (any round): kept when every
// piece is inside, dropped when one is outside, else the FP64 test.
template <int D>
__device__ __forceinline__ bool pointInBoxF(const ExpandArgs& a, uint32_t j, uint32_t e, uint32_t q) {
    constexpr int L = D / 4;
    const float4* p = reinterpret_cast<const float4*>(a.child.rowsF + static_cast<size_t>(j) * D);
    const float4* fo = reinterpret_cast<const float4*>(a.query.boxesF + static_cast<size_t>(q) * 2 * D);
    const float4* fi = reinterpret_cast<const float4*>(a.query.boxesFi + static_cast<size_t>(q) * 2 * D);
    bool allIn = true, anyOut = false;
#pragma unroll
    for (int c = 0; c < L; ++c) {
        bool in, out;
        pieceF(__ldcs(p + c), __ldg(fo + c), __ldg(fo + L + c), __ldg(fi + c), __ldg(fi + L + c), in, out);
        allIn = allIn && in;
        anyOut = anyOut || out;
    }
    if (allIn) return true;
    if (anyOut) return false;
    return exactPointInBox<D>(a, j, e, q);
}

// Finest exact range level, a round whose 32 items all belong to one frontier entry, from the
// float points: the items' float rows are one contiguous block of 32·4·D bytes, each lane loads
// one 16-byte piece (four coordinates) per load and a ballot per load collects the pieces'
// decisions. Half the bytes of singleEntryRangeBox; identical outcome (pointInBoxF's rule).
template <int D>
constexpr bool coalescedBoxF() {
    return floatPointsSupported(D);
}
template <int D>
__device__ __forceinline__ bool singleEntryRangeBoxF(const ExpandArgs& a, uint32_t j0, uint32_t e, uint32_t q,
                                                     int lane) {
    constexpr int L = D / 4;   // pieces per point
    constexpr int G = 32 / L;  // points per load
    constexpr uint32_t kAll = (1u << L) - 1u;
    const int c = lane % L;
    const float4* rows4 = reinterpret_cast<const float4*>(a.child.rowsF + static_cast<size_t>(j0) * D);
    const float4* fo = reinterpret_cast<const float4*>(a.query.boxesF + static_cast<size_t>(q) * 2 * D);
    const float4* fi = reinterpret_cast<const float4*>(a.query.boxesFi + static_cast<size_t>(q) * 2 * D);
    const float4 lo = __ldg(fo + c), hi = __ldg(fo + L + c), li = __ldg(fi + c), hiI = __ldg(fi + L + c);
    float4 v[L];
#pragma unroll
    for (int i = 0; i < L; ++i) v[i] = __ldcs(rows4 + i * 32 + lane);
    uint32_t inMine = 0, outMine = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        bool in, out;
        pieceF(v[i], lo, hi, li, hiI, in, out);
        const uint32_t bi = __ballot_sync(0xffffffffu, in), bo = __ballot_sync(0xffffffffu, out);
        if (i == lane / G) {
            inMine = bi;
            outMine = bo;
        }
    }
    const int sh = (lane % G) * L;
    if (((inMine >> sh) & kAll) == kAll) return true;
    if (((outMine >> sh) & kAll) != 0) return false;
    return exactPointInBox<D>(a, j0 + lane, e, q);
}

// Exact range frontier levels, a round whose 32 children all belong to one frontier entry: the
// children are consecutive nodes, so their float boxes (lo[D] then hi[D], 8·D bytes each) form one
// contiguous block. Each lane takes one 16-byte piece (four lower or four upper bounds) of a box
// per load and tests it against the matching four upper or lower bounds of the query's box; a
// ballot per load collects the pieces. Same comparisons as aabbMeets, so the outcome is identical.
// Returns the prefilter outcome of the calling lane's own child (item `lane` of the round).
template <int D>
constexpr bool coalescedAabb() {
    return D >= 4 && D % 4 == 0 && 32 % (D >= 2 ? D / 2 : 1) == 0;
}
template <int D>
__device__ __forceinline__ bool singleEntryAabb(const ExpandArgs& a, uint32_t kk0, uint32_t q, int lane) {
    constexpr int L = D / 2;   // pieces per box
    constexpr int G = 32 / L;  // boxes per load
    constexpr int LO = D / 4;  // pieces holding lower bounds
    constexpr int P = L < 4 ? L : 4;
    constexpr uint32_t kAll = (1u << L) - 1u;
    const int c = lane % L;
    const bool lower = c < LO;
    const float4* cb = reinterpret_cast<const float4*>(a.child.aabb + static_cast<size_t>(kk0) * 2 * D);
    const float* qb = a.query.boxesF + static_cast<size_t>(q) * 2 * D;
    // A lower-bound piece is tested against the query's upper bounds, and the other way round.
    const float4 qv = __ldg(reinterpret_cast<const float4*>(lower ? qb + D + 4 * c : qb + 4 * (c - LO)));
    uint32_t mine = 0;
#pragma unroll
    for (int s0 = 0; s0 < L; s0 += P) {
        float4 bv[P];
#pragma unroll
        for (int i = 0; i < P; ++i) bv[i] = __ldg(cb + (s0 + i) * 32 + lane);
#pragma unroll
        for (int i = 0; i < P; ++i) {
            const float4 v = bv[i];
            const bool pass = lower ? (v.x <= qv.x) & (v.y <= qv.y) & (v.z <= qv.z) & (v.w <= qv.w)
                                    : (v.x >= qv.x) & (v.y >= qv.y) & (v.z >= qv.z) & (v.w >= qv.w);
            const uint32_t b = __ballot_sync(0xffffffffu, pass);
            if (s0 + i == lane / G) mine = b;
        }
    }
    return ((mine >> ((lane % G) * L)) & kAll) == kAll;
}

template <int D, int PRED, bool TO_RESULT, bool STAGED>
__global__ void __launch_bounds__(kExpandThreads, expandMinBlocks<PRED>()) expandKernel(ExpandArgs a) {
    using S = Staging<D, STAGED>;
    constexpr int R = S::kRounds;
    constexpr int DM = (D > 0) ? D : 32;
    constexpr bool NODE = needsNode<PRED, TO_RESULT>();
    // Code size (see TBLAEQ_UNROLL_FRONTIER_TEST); the KNN levels unroll every loop.
    constexpr bool kKnn = PRED == kPredKnnBound || PRED == kPredKnnPoint;
    constexpr int kUnrollTest = (PRED == kPredRangeBoxF) ? TBLAEQ_UNROLL_FLOAT_TEST
                                : (TO_RESULT || kKnn)     ? R
                                                          : TBLAEQ_UNROLL_FRONTIER_TEST;
    constexpr int kUnrollPass2 = kKnn ? R : TBLAEQ_UNROLL_PASS2;
    constexpr bool kFastBox = PRED == kPredRangeBox && TO_RESULT && !STAGED && coalescedBox<D>();
    // Finest exact range level with float points (a.child.rowsF): every round tests them first.
    constexpr bool kFloatPts = PRED == kPredRangeBoxF && TO_RESULT && !STAGED && coalescedBoxF<D>();
    constexpr bool kFastAabb = PRED == kPredRangeRadius && coalescedAabb<D>();
    // Exact range frontier levels test children that pass the box prefilter after the rounds,
    // 32 at a time, so the FP64 radius test runs on full warps instead of in every round that
    // holds one survivor.
    constexpr bool kDefer = PRED == kPredRangeRadius;
    constexpr uint32_t FULL = 0xffffffffu;
    extern __shared__ __align__(16) unsigned char smem[];
    const int dim = (D > 0) ? D : a.D;
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint32_t lanesLe = (2u << lane) - 1u;  // lanes 0..lane (wraps to all lanes for lane 31)
    const uint32_t lanesLt = (1u << lane) - 1u;
    unsigned char* warpSmem = smem + static_cast<size_t>(w) * warpSmemBytes<D, STAGED, PRED>();
    unsigned char* rowBuf = warpSmem;                                    // [kStages][32][kStride]
    NodeRec* nodeBuf = reinterpret_cast<NodeRec*>(warpSmem + S::kRowBytes);  // [kStages][32]
    uint32_t* sRow = reinterpret_cast<uint32_t*>(warpSmem + S::kRowBytes + S::kNodeBytes);  // [R][32]
    uint16_t* sWin = reinterpret_cast<uint16_t*>(sRow + R * 32);  // item -> window slot of its entry
    uint32_t* wCp = reinterpret_cast<uint32_t*>(sWin + R * 32);  // window of the tile's entries: prefix, first child, query
    uint32_t* wCb = wCp + S::kWindow;
    uint32_t* wQ = wCb + S::kWindow;
    uint16_t* sList = reinterpret_cast<uint16_t*>(warpSmem + S::kRowBytes + S::kNodeBytes + S::kCacheBytes +
                                                  ((S::kWindowBytes + 15) / 16) * 16);  // deferred items
    uint32_t* sKeep = reinterpret_cast<uint32_t*>(sList + kWarpTile);                   // [R] keep words

    // A look-back that gave up earlier in this batch, or a child prefix that passed 32 bits, left
    // the frontiers after it inconsistent: never read them; the host reports the status.
    if (*a.scratch.status & kStatusInconsistent) return;
    const uint32_t entries = a.in.hdr[0];
    const uint32_t total = a.in.hdr[1];
    const uint32_t nTiles = (total + kWarpTile - 1) / kWarpTile;
    if (entries == 0 || total == 0) return;
    // A producer that overflowed its capacities left this frontier incomplete: never read past
    // the arrays (the host sees the status bit, grows the workspace and reruns the batch).
    if (entries > a.in.cap || nTiles > a.in.tileCap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(a.scratch.status, kStatusOverflowEntries);
        return;
    }

    unsigned long long warpRows = 0;  // child rows this warp loaded (two-wave work counter)
    while (true) {
        uint32_t tile = 0;
        if (lane == 0) tile = atomicAdd(a.scratch.ticket, 1u);
        tile = __shfl_sync(FULL, tile, 0);
        if (tile >= nTiles) {
            if (a.scratch.work && lane == 0 && warpRows) atomicAdd(a.scratch.work, warpRows);
            break;
        }
        // The tile's rows are one contiguous run per entry: the TMA unit brings each run into L2
        // now (one instruction per run, no registers), ahead of the per-round row loads.
        if constexpr (prefetchesRows<D, PRED>())
            prefetchTileRows<D, PRED>(a, tile, nTiles, entries, total, lane, kFloatPts);
        const uint32_t t0 = tile * kWarpTile;

        // ---- phase A: stage the tile's entries in shared memory (one round of parallel loads),
        // then map every item of the tile to its entry and child row.
        const uint32_t eLo = a.in.tileStart[tile];
        uint32_t eHi = (tile + 1 < nTiles) ? a.in.tileStart[tile + 1] : entries - 1;
        if (eHi >= entries) eHi = entries - 1;
        // A tile start outside the frontier means an inconsistent input (an overflowed producer):
        // the tile is processed as empty, so it still publishes its (zero) counts to the look-back.
        const bool tileOk = eLo <= eHi;
        if (!tileOk && lane == 0) atomicOr(a.scratch.status, kStatusOverflowEntries);
        uint32_t W = tileOk ? eHi - eLo + 1 : 0u;
        if (W > S::kWindow) {
            if (lane == 0) atomicOr(a.scratch.status, kStatusWindowOverflow);
            W = S::kWindow;
        }
        for (uint32_t i = lane; i < W; i += 32) {
            wCp[i] = a.in.cpre[eLo + i];
            wCb[i] = a.in.cbeg[eLo + i];
            wQ[i] = a.in.q[eLo + i];
        }
        __syncwarp();
        uint32_t validBits = 0;
        uint32_t cur = 0;  // window index of the entry holding the round's first item
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const uint32_t rs = t0 + r * 32;
            if (rs >= total || W == 0) continue;  // warp-uniform
            const uint32_t k = rs + lane;
            const bool valid = k < total;
            // Every entry overlapping a 32-item round lies within the 32 window slots from `cur`:
            // `cur` holds the round's first item and every other entry starts at a distinct item.
            const uint32_t ce = cur + lane;
            const uint32_t cp = ce < W ? wCp[ce] : 0xffffffffu;
            const uint32_t base = __popc(__ballot_sync(FULL, cp <= rs)) - 1u;
            const uint32_t off = cp - rs;
            const uint32_t starts = __reduce_or_sync(FULL, (cp > rs && off < 32u) ? (1u << off) : 0u);
            const uint32_t my = cur + base + __popc(starts & lanesLe);
            const uint32_t e = my < W ? my : W - 1;
            sRow[r * 32 + lane] = wCb[e] + (k - wCp[e]);
            sWin[r * 32 + lane] = static_cast<uint16_t>(e);
            validBits |= (valid ? 1u : 0u) << r;
            // The next round's first item (rs + 32) lies in the entry holding this round's last item,
            // or in the next entry when that one starts exactly there.
            const uint32_t last = __shfl_sync(FULL, e, 31);
            cur = (last + 1 < W && wCp[last + 1] == rs + 32) ? last + 1 : last;
        }
        __syncwarp();

        // ---- phase B: stream the rows (and node records) through the cp.async ring and test.
        auto issue = [&](int r) {
            if constexpr (S::kOn) {
                if (W == 0) return;  // an empty (inconsistent) tile has no rows to stage
                // The round's rows move as 32 * kChunks chunk copies spread over the warp so that
                // consecutive lanes copy consecutive chunks: rows of one entry are consecutive in
                // the P-tensor, so each copy instruction reads whole sectors (a lane copying its own
                // row would touch a different sector per lane). Each row still lands in its own
                // lane's padded slot, and the lane later reads it back whole.
                const int slot = r % S::kStages;
                const uint32_t rs = t0 + r * 32;
#pragma unroll
                for (int i = 0; i < S::kChunks; ++i) {
                    const uint32_t t = static_cast<uint32_t>(i) * 32u + lane;
                    const uint32_t it = t / S::kChunks, c = t % S::kChunks;
                    if (rs + it < total) {
                        const uint32_t j = sRow[r * 32 + it];
                        const unsigned char* src = reinterpret_cast<const unsigned char*>(a.child.rows) +
                                                   static_cast<size_t>(j) * (8 * D) + c * S::kChunk;
                        unsigned char* dst = rowBuf + (slot * 32 + it) * S::kStride + c * S::kChunk;
                        if constexpr (S::kChunk == 16) {
                            cpAsync16(dst, src);
                        } else {
                            cpAsync8(dst, src);
                        }
                    }
                }
                if constexpr (NODE) {
                    if ((validBits >> r) & 1u) {
                        const uint32_t j = sRow[r * 32 + lane];
                        const uint32_t kk = a.child.keys ? static_cast<uint32_t>(a.child.keys[j]) : j;
                        cpAsync16(&nodeBuf[slot * 32 + lane], &a.child.nodes[kk]);
                    }
                }
            }
        };
        if constexpr (S::kOn) {
            __syncwarp();
#pragma unroll
            for (int r = 0; r < S::kStages - 1; ++r) {
                if (r < R) issue(r);
                cpAsyncCommit();
            }
        }
        uint32_t keepBits = 0, aggCnt = 0, aggSum = 0;
        uint32_t listLen = 0;  // deferred prefilter survivors of this tile (kDefer)
        const bool deferOn = kDefer && a.child.aabb != nullptr && a.query.boxesF != nullptr;
        if constexpr (kDefer) {
            if (lane < R) sKeep[lane] = 0u;
            __syncwarp();
        }
#pragma unroll kUnrollTest
        for (int r = 0; r < R; ++r) {
            if constexpr (S::kOn) {
                // Lanes copy each other's rows: the slot being refilled must be read out by every
                // lane first, and a landed round is visible to the warp only after its barrier.
                __syncwarp();
                if (r + S::kStages - 1 < R) issue(r + S::kStages - 1);
                cpAsyncCommit();
                cpAsyncWait<S::kStages - 1>();
                __syncwarp();
            }
            if (t0 + r * 32 >= total) continue;  // warp-uniform
            const bool valid = (validBits >> r) & 1u;
            bool keep = false, defer = false;
            uint32_t cc = 0;
            bool work = valid;
            if (PRED == kPredKnnPoint && valid && a.wave != 0 && a.child.entrySel) {
                // Two-wave KNN: decide from the entry alone before touching the child's row.
                const uint32_t e = eLo + sWin[r * 32 + lane];
                const bool sel = __ldg(a.child.entrySel + e) != 0;
                if (a.wave == 1) {
                    work = sel;
                } else {
                    work = !sel && __ldg(a.child.entryLb + e) <= __ldcg(a.query.tau + wQ[sWin[r * 32 + lane]]);
                }
            }
            bool done = false;
            if constexpr (kFastBox) {
                // Warp-uniform: a full round inside one entry (its first and last item share it).
                const uint32_t w0 = sWin[r * 32], w31 = sWin[r * 32 + 31];
                if (W != 0 && t0 + r * 32 + 32 <= total && w0 == w31) {
                    keep = singleEntryRangeBox<D>(a, sRow[r * 32], eLo + w0, wQ[w0], lane);
                    done = true;
                }
            }
            if constexpr (kFloatPts) {
                const uint32_t w0 = sWin[r * 32], w31 = sWin[r * 32 + 31];
                if (W != 0 && t0 + r * 32 + 32 <= total && w0 == w31) {
                    keep = singleEntryRangeBoxF<D>(a, sRow[r * 32], eLo + w0, wQ[w0], lane);
                    done = true;
                }
            }
            bool preKnown = false, preFast = true;
            if constexpr (kFastAabb) {
                // Warp-uniform: a full round inside one entry, children keyed by their rows.
                const uint32_t w0 = sWin[r * 32], w31 = sWin[r * 32 + 31];
                if (W != 0 && t0 + r * 32 + 32 <= total && w0 == w31 && a.child.aabb && a.query.boxesF &&
                    !a.child.keys) {
                    preFast = singleEntryAabb<D>(a, sRow[r * 32], wQ[w0], lane);
                    preKnown = true;
                }
            }
            if (work && !done) {
                const uint32_t j = sRow[r * 32 + lane];
                const uint32_t w = sWin[r * 32 + lane];
                const uint32_t e = eLo + w;
                const uint32_t q = wQ[w];
                const uint32_t kk = a.child.keys ? static_cast<uint32_t>(a.child.keys[j]) : j;
                bool pre = true;
                if constexpr (PRED == kPredRangeRadius) {
                    if (preKnown)
                        pre = preFast;
                    else if (a.child.aabb && a.query.boxesF)
                        pre = aabbMeets<D, DM>(a, dim, kk, q);
                }
                if (pre && deferOn) {
                    defer = true;  // radius test after the rounds
                } else if (pre) {
                    NodeRec nr{0.0, 0u, 0u};
                    const double* xp = a.in.x + static_cast<size_t>(e) * dim;
                    if constexpr (S::kOn) {
                        const int slot = r % S::kStages;
                        const double* rowp = reinterpret_cast<const double*>(rowBuf + (slot * 32 + lane) * S::kStride);
                        if constexpr (NODE) nr = nodeBuf[slot * 32 + lane];
                        keep = evalItem<D, DM, PRED, TO_RESULT, true>(a, dim, rowp, xp, q, j, kk, nr, cc);
                    } else if constexpr (kFloatPts) {
                        keep = pointInBoxF<D>(a, j, e, q);
                    } else {
                        if constexpr (NODE) nr = a.child.nodes[kk];
                        keep = evalItem<D, DM, PRED, TO_RESULT, false>(a, dim, a.child.rows + static_cast<size_t>(j) * dim,
                                                                       xp, q, j, kk, nr, cc);
                    }
                }
            }
            if constexpr (kDefer) {
                const uint32_t dm = __ballot_sync(FULL, defer);
                if (dm) {  // warp-uniform
                    if (defer) sList[listLen + __popc(dm & lanesLt)] = static_cast<uint16_t>(r * 32 + lane);
                    listLen += __popc(dm);
                }
            }
            if (a.scratch.work) warpRows += __popc(__ballot_sync(FULL, work));
            // Per-query generated-children counts (the reference's levelFineMeshSize).
            if (a.scratch.levelItems) {
                const uint32_t vm = __ballot_sync(FULL, valid);
                if (valid) {
                    const uint32_t q = wQ[sWin[r * 32 + lane]];
                    const uint32_t peers = __match_any_sync(vm, q);
                    if (lane == __ffs(peers) - 1) atomicAdd(&a.scratch.levelItems[q], __popc(peers));
                }
            }
            const uint32_t kb = __ballot_sync(FULL, keep);
            if (kb) {  // warp-uniform
                keepBits |= (keep ? 1u : 0u) << r;
                aggCnt += __popc(kb);
                if constexpr (!TO_RESULT) {
                    uint32_t s = keep ? cc : 0u;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
                    aggSum += s;
                }
            }
        }

        // ---- deferred radius tests (kDefer): the prefilter survivors of every round, 32 at a time.
        if constexpr (kDefer) {
            if (listLen) {  // warp-uniform
                __syncwarp();
                for (uint32_t b0 = 0; b0 < listLen; b0 += 32) {
                    const uint32_t t = b0 + lane;
                    bool k2 = false;
                    uint32_t cc2 = 0, idx = 0;
                    if (t < listLen) {
                        idx = sList[t];
                        const uint32_t j = sRow[idx];
                        const uint32_t w = sWin[idx];
                        const uint32_t q = wQ[w];
                        const uint32_t kk = a.child.keys ? static_cast<uint32_t>(a.child.keys[j]) : j;
                        const NodeRec nr = a.child.nodes[kk];
                        k2 = evalItem<D, DM, PRED, TO_RESULT, false>(a, dim, a.child.rows + static_cast<size_t>(j) * dim,
                                                                     a.in.x + static_cast<size_t>(eLo + w) * dim, q, j,
                                                                     kk, nr, cc2);
                        if (k2) atomicOr(&sKeep[idx >> 5], 1u << (idx & 31u));
                    }
                    const uint32_t kb2 = __ballot_sync(FULL, k2);
                    aggCnt += __popc(kb2);
                    uint32_t s2 = k2 ? cc2 : 0u;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(FULL, s2, o);
                    aggSum += s2;
                }
                __syncwarp();
#pragma unroll
                for (int r = 0; r < R; ++r) keepBits |= ((sKeep[r] >> lane) & 1u) << r;
            }
        }

        // ---- publish the tile's counts and learn where its output starts. A tile that kept
        // nothing writes nothing, so it needs no output position: it publishes its empty
        // aggregate and moves on without waiting for its predecessors (most tiles of the finest
        // levels); successors sum through it. The last tile still resolves the totals.
        if (tile == a.withholdTile) continue;  // test hook: this tile never publishes
        if (aggCnt == 0 && aggSum == 0 && tile != nTiles - 1) {
            if (lane == 0) storeDesc(&a.scratch.desc[tile], packDesc(tile == 0 ? kFlagPrefix : kFlagAggregate, 0, 0));
            continue;
        }
        unsigned long long exCnt, exSum;
        lookback(a.scratch.desc, tile, aggCnt, aggSum, a.scratch.status, a.spinLimit ? a.spinLimit : kSpinLimit,
                 exCnt, exSum);
        if (tile == nTiles - 1 && lane == 0) {
            const unsigned long long totC = exCnt + aggCnt;
            const unsigned long long totS = exSum + aggSum;
            if constexpr (TO_RESULT) {
                a.rout.hdr[0] = static_cast<uint32_t>(min(totC, 0xffffffffull));
                if (totC > a.rout.cap) atomicOr(a.scratch.status, kStatusOverflowEntries);
            } else {
                a.fout.hdr[0] = static_cast<uint32_t>(min(totC, 0xffffffffull));
                a.fout.hdr[1] = static_cast<uint32_t>(min(totS, 0xffffffffull));
                if (totC > a.fout.cap) atomicOr(a.scratch.status, kStatusOverflowEntries);
                if (totS > 0xffffffffull) atomicOr(a.scratch.status, kStatusOverflowSum);
                const unsigned long long tilesNeeded = (totS + kWarpTile - 1) / kWarpTile;
                if (tilesNeeded > a.fout.tileCap) atomicOr(a.scratch.status, kStatusOverflowItems);
            }
        }

        // ---- pass 2: rebuild and write the kept items in order.
        unsigned long long runCnt = exCnt, runSum = exSum;
#pragma unroll kUnrollPass2
        for (int r = 0; r < R; ++r) {
            const bool keep = (keepBits >> r) & 1u;
            const uint32_t kb = __ballot_sync(FULL, keep);
            if (kb == 0) continue;  // warp-uniform
            const uint32_t j = sRow[r * 32 + lane];
            const uint32_t wr = sWin[r * 32 + lane];
            const uint32_t qr = wQ[wr];
            const uint32_t er = eLo + wr;
            uint32_t cc = 0, ncb = 0, kk = 0;
            if (keep) {
                kk = a.child.keys ? static_cast<uint32_t>(a.child.keys[j]) : j;
                if constexpr (!TO_RESULT) {
                    const NodeRec nr = a.child.nodes[kk];
                    cc = nr.cnt;
                    ncb = nr.cbeg;
                }
            }
            const uint32_t v = keep ? cc : 0u;
            uint32_t inc = v;
            if constexpr (!TO_RESULT) {
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(FULL, inc, o);
                    if (lane >= o) inc += t;
                }
            }
            const uint32_t roundSum = TO_RESULT ? 0u : __shfl_sync(FULL, inc, 31);
            if (keep) {
                const unsigned long long pos = runCnt + __popc(kb & lanesLt);
                if constexpr (TO_RESULT) {
                    if (pos < a.rout.cap) {
                        // Float points in point-group order: the row's place in the P tensor.
                        const uint32_t jr = (PRED == kPredRangeBoxF && a.child.perm) ? a.child.perm[j] : j;
                        a.rout.ids[pos] = a.child.outMap ? a.child.outMap[jr] : static_cast<uint64_t>(kk);
                        if (a.rout.q) a.rout.q[pos] = qr;
                        double* vals = a.rout.vals ? a.rout.vals + pos * dim : nullptr;
                        if constexpr (PRED == kPredKnnPoint) {
                            if (vals || a.rout.dist2) {
                                constexpr int C = chunkOf<D>();
                                const double* p = a.query.points + static_cast<size_t>(qr) * dim;
                                double dist = 0.0;
                                rebuildChunks<D, DM>(a, dim, er, j, [&](int d, const double (&y)[C]) {
                                    if (vals) stChunk<C>(vals + d, y);
                                    double pp[C];
                                    ldChunk<C, false>(p + d, pp);
#pragma unroll
                                    for (int i = 0; i < C; ++i) {
                                        const double diff = pp[i] - y[i];
                                        dist = __fma_rn(diff, diff, dist);
                                    }
                                });
                                if (a.rout.dist2) a.rout.dist2[pos] = dist;
                            }
                        } else if (vals) {
                            constexpr int C = chunkOf<D>();
                            rebuildChunks<D, DM>(a, dim, er, jr,
                                                 [&](int d, const double (&y)[C]) { stChunk<C>(vals + d, y); });
                        }
                    }
                } else if (pos < a.fout.cap) {
                    const unsigned long long cp = runSum + (inc - v);
                    a.fout.q[pos] = qr;
                    a.fout.node[pos] = kk;
                    a.fout.cbeg[pos] = ncb;
                    a.fout.cpre[pos] = static_cast<uint32_t>(cp);
                    {
                        constexpr int C = chunkOf<D>();
                        double* xo = a.fout.x + pos * dim;
                        rebuildChunks<D, DM>(a, dim, er, j, [&](int d, const double (&y)[C]) { stChunk<C>(xo + d, y); });
                    }
                    // Tile starts of the next level: every tile boundary inside this entry's children.
                    const unsigned long long cend = cp + cc;
                    for (unsigned long long b = (cp + kWarpTile - 1) / kWarpTile; b * kWarpTile < cend; ++b) {
                        if (b < a.fout.tileCap) a.fout.tileStart[b] = static_cast<uint32_t>(pos);
                    }
                }
            }
            {
                uint32_t* qc = TO_RESULT ? a.rout.qcount : a.fout.qcount;
                if (qc && keep) {
                    const uint32_t peers = __match_any_sync(kb, qr);
                    if (lane == __ffs(peers) - 1) atomicAdd(&qc[qr], __popc(peers));
                }
            }
            runCnt += __popc(kb);
            runSum += roundSum;
        }
    }
}

__global__ void rootFrontierKernel(uint32_t* q, uint32_t* cbeg, uint32_t* cpre, double* x, uint32_t* tileStart,
                                   uint32_t* hdr, uint32_t nq, uint32_t nChildren, int D, int tile) {
    const uint64_t total = static_cast<uint64_t>(nq) * nChildren;
    const uint64_t nTiles = (total + tile - 1) / tile;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += stride) {
        q[i] = static_cast<uint32_t>(i);
        cbeg[i] = 0;
        cpre[i] = static_cast<uint32_t>(i * nChildren);
        for (int d = 0; d < D; ++d) x[i * D + d] = 1.0;
    }
    for (uint64_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nTiles; b += stride) {
        tileStart[b] = static_cast<uint32_t>((b * tile) / nChildren);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        hdr[0] = nq;
        hdr[1] = static_cast<uint32_t>(total);
    }
}

// One block; each thread scans kScanItems consecutive counts per pass (independent loads), then the
// block scans the threads' sums.
constexpr int kScanItems = 4;
__global__ void exclusiveScanKernel(const uint32_t* counts, uint64_t* offsets, uint32_t n) {
    __shared__ unsigned long long sCarry;
    __shared__ unsigned long long sWarp[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) sCarry = 0;
    __syncthreads();
    for (uint64_t base = 0; base < n; base += static_cast<uint64_t>(blockDim.x) * kScanItems) {
        const uint64_t i0 = base + static_cast<uint64_t>(tid) * kScanItems;
        uint32_t c[kScanItems];
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) c[k] = (i0 + k < n) ? counts[i0 + k] : 0u;
        unsigned long long v = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) v += c[k];
        unsigned long long inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        if (lane == 31) sWarp[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const int nw = blockDim.x / 32;
            unsigned long long w = (lane < nw) ? sWarp[lane] : 0;
            unsigned long long wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long t = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += t;
            }
            if (lane < nw) sWarp[lane] = wi - w;
        }
        __syncthreads();
        const unsigned long long carry = sCarry;
        unsigned long long run = carry + sWarp[warp] + inc - v;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            if (i0 + k < n) offsets[i0 + k] = run;
            run += c[k];
        }
        __syncthreads();
        if (tid == blockDim.x - 1) sCarry = carry + sWarp[warp] + inc;
        __syncthreads();
    }
    if (tid == 0) offsets[n] = sCarry;
}

template <int D, int PRED, bool TO_RESULT, bool STAGED>
void launchOne(const ExpandArgs& a, int gridBlocks, cudaStream_t s) {
    auto kern = expandKernel<D, PRED, TO_RESULT, STAGED>;
    constexpr size_t smemBytes = expandSmemBytes<D, STAGED, PRED>();
    static int cached = 0;
    if (cached == 0) {
        int dev = 0, sms = 0, perSm = 0;
        TBLAEQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smemBytes)));
        TBLAEQ_CUDA(cudaGetDevice(&dev));
        TBLAEQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        TBLAEQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kExpandThreads, smemBytes));
        cached = std::max(1, sms * std::max(1, perSm));
    }
    if (gridBlocks <= 0) {
        const int pct = (a.gridPercent > 0 && a.gridPercent < 100) ? a.gridPercent : 100;
        gridBlocks = std::max(1, static_cast<int>((static_cast<long long>(cached) * pct + 99) / 100));
    }
    kern<<<gridBlocks, kExpandThreads, smemBytes, s>>>(a);
    TBLAEQ_LAUNCHED();
}

template <int D, bool ST>
void dispatchPred(const ExpandArgs& a, int pred, bool toResult, int g, cudaStream_t s) {
    if (toResult) {
        switch (pred) {
            case kPredAll: return launchOne<D, kPredAll, true, ST>(a, g, s);
            case kPredRangeBox: return launchOne<D, kPredRangeBox, true, ST>(a, g, s);
            case kPredRangeBoxF: return launchOne<D, kPredRangeBoxF, true, ST>(a, g, s);
            case kPredMask: return launchOne<D, kPredMask, true, ST>(a, g, s);
            case kPredKnnPoint: return launchOne<D, kPredKnnPoint, true, ST>(a, g, s);
            default: break;
        }
    } else {
        switch (pred) {
            case kPredRangeRadius: return launchOne<D, kPredRangeRadius, false, ST>(a, g, s);
            case kPredMask: return launchOne<D, kPredMask, false, ST>(a, g, s);
            case kPredAll: return launchOne<D, kPredAll, false, ST>(a, g, s);
            case kPredGroupBox: return launchOne<D, kPredGroupBox, false, false>(a, g, s);
            case kPredKnnBound: return launchOne<D, kPredKnnBound, false, ST>(a, g, s);
            default: break;
        }
    }
    throw std::invalid_argument("expand: unsupported predicate/output combination");
}

template <int D>
void dispatchStaged(const ExpandArgs& a, int pred, bool toResult, int g, cudaStream_t s) {
    // Rows in mapped host memory are read with plain loads only (no cp.async staging).
    if (a.variant == kVariantStaged && !a.child.rowsOnHost) return dispatchPred<D, true>(a, pred, toResult, g, s);
    return dispatchPred<D, false>(a, pred, toResult, g, s);
}

}  // namespace

namespace {
std::atomic<uint32_t> gHookWithhold{0xffffffffu};
std::atomic<uint32_t> gHookSpins{0};
}  // namespace

void setLookbackTestHook(uint32_t withholdTile, uint32_t spinLimit) {
    const bool off = withholdTile == 0xffffffffu || spinLimit == 0;
    gHookWithhold.store(off ? 0xffffffffu : withholdTile);
    gHookSpins.store(off ? 0u : spinLimit);
}

void launchExpand(const ExpandArgs& in, int pred, bool toResult, int gridBlocks, cudaStream_t stream) {
    ExpandArgs a = in;
    a.withholdTile = 0xffffffffu;
    a.spinLimit = 0;
    if (pred != kPredKnnBound && pred != kPredKnnPoint) {
        a.withholdTile = gHookWithhold.load();
        a.spinLimit = gHookSpins.load();
    }
    switch (a.D) {
        case 2: return dispatchStaged<2>(a, pred, toResult, gridBlocks, stream);
        case 3: return dispatchStaged<3>(a, pred, toResult, gridBlocks, stream);
        case 4: return dispatchStaged<4>(a, pred, toResult, gridBlocks, stream);
        case 5: return dispatchStaged<5>(a, pred, toResult, gridBlocks, stream);
        case 8: return dispatchStaged<8>(a, pred, toResult, gridBlocks, stream);
        case 16: return dispatchStaged<16>(a, pred, toResult, gridBlocks, stream);
        default:
            if (a.D < 1 || a.D > 32) throw std::invalid_argument("expand: D must be in [1, 32]");
            return dispatchPred<0, false>(a, pred, toResult, gridBlocks, stream);
    }
}

void launchRootFrontier(uint32_t* q, uint32_t* cbeg, uint32_t* cpre, double* x, uint32_t* tileStart, uint32_t* hdr,
                        uint32_t nq, uint32_t nChildren, int D, int tile, cudaStream_t stream) {
    const uint64_t total = static_cast<uint64_t>(nq) * nChildren;
    const uint64_t nTiles = (total + tile - 1) / tile;
    const uint64_t work = std::max<uint64_t>(nq, nTiles);
    const int blocks = static_cast<int>(std::min<uint64_t>(1024, (work + 255) / 256 + 1));
    rootFrontierKernel<<<blocks, 256, 0, stream>>>(q, cbeg, cpre, x, tileStart, hdr, nq, nChildren, D, tile);
    TBLAEQ_LAUNCHED();
}

__global__ void roundBoxesKernel(const double* boxes, uint32_t nq, int D, float* boxesF, float* boxesFi) {
    const uint64_t n = static_cast<uint64_t>(nq) * 2 * D;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const bool upper = (i % (2 * D)) >= static_cast<uint64_t>(D);
        boxesF[i] = upper ? __double2float_ru(boxes[i]) : __double2float_rd(boxes[i]);
        if (boxesFi) boxesFi[i] = upper ? __double2float_rd(boxes[i]) : __double2float_ru(boxes[i]);
    }
}

void launchRoundBoxes(const double* boxes, uint32_t nq, int D, float* boxesF, float* boxesFi, cudaStream_t stream) {
    if (nq == 0) return;
    const uint64_t n = static_cast<uint64_t>(nq) * 2 * D;
    const int blocks = static_cast<int>(std::min<uint64_t>(148 * 4, (n + 255) / 256));
    roundBoxesKernel<<<blocks, 256, 0, stream>>>(boxes, nq, D, boxesF, boxesFi);
    TBLAEQ_LAUNCHED();
}

void launchExclusiveScan(const uint32_t* counts, uint64_t* offsets, uint32_t n, cudaStream_t stream) {
    exclusiveScanKernel<<<1, 1024, 0, stream>>>(counts, offsets, n);
    TBLAEQ_LAUNCHED();
}

// ---- node-major range levels (exact mode) -------------------------------------------------------

namespace {

// Node keys at or above M (only an inconsistent frontier has them) are skipped by the count and the
// scatter alike, so the grouping stays within its arrays.
// Entries come in runs of the same node (a unit's survivors are appended child by child), so the
// lanes of a warp holding one node add to its count (and claim its list slots) with one atomic.
__global__ void nodeCountKernel(const uint32_t* node, const uint32_t* hdr, uint32_t cap, uint32_t M,
                                uint32_t* nodeCnt) {
    const uint32_t n = min(hdr[0], cap);
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + lane;
        const uint32_t nd = i < n ? node[i] : M;
        const uint32_t peers = __match_any_sync(0xffffffffu, nd);
        if (nd < M && lane == static_cast<uint32_t>(__ffs(peers) - 1)) atomicAdd(&nodeCnt[nd], __popc(peers));
    }
}

// One CTA: nodeOff = exclusive scan of the entry counts, unitOff = exclusive scan of their units of 32.
__global__ void __launch_bounds__(1024) nodeScanKernel(const uint32_t* nodeCnt, uint32_t M, uint32_t* nodeOff,
                                                       uint32_t* unitOff) {
    __shared__ uint32_t sWarpA[32], sWarpB[32];
    __shared__ uint32_t sCarryA, sCarryB;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        sCarryA = 0;
        sCarryB = 0;
    }
    __syncthreads();
    for (uint32_t base = 0; base < M; base += blockDim.x) {
        const uint32_t i = base + tid;
        const uint32_t va = i < M ? nodeCnt[i] : 0u;
        const uint32_t vb = (va + 31u) / 32u;
        uint32_t ia = va, ib = vb;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t ta = __shfl_up_sync(0xffffffffu, ia, o), tb = __shfl_up_sync(0xffffffffu, ib, o);
            if (lane >= o) {
                ia += ta;
                ib += tb;
            }
        }
        if (lane == 31) {
            sWarpA[warp] = ia;
            sWarpB[warp] = ib;
        }
        __syncthreads();
        if (warp == 0) {
            const int nw = blockDim.x / 32;
            uint32_t wa = lane < nw ? sWarpA[lane] : 0u, wb = lane < nw ? sWarpB[lane] : 0u;
            uint32_t xa = wa, xb = wb;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t ta = __shfl_up_sync(0xffffffffu, xa, o), tb = __shfl_up_sync(0xffffffffu, xb, o);
                if (lane >= o) {
                    xa += ta;
                    xb += tb;
                }
            }
            if (lane < nw) {
                sWarpA[lane] = xa - wa;
                sWarpB[lane] = xb - wb;
            }
        }
        __syncthreads();
        const uint32_t ca = sCarryA, cb = sCarryB;
        if (i < M) {
            nodeOff[i] = ca + sWarpA[warp] + ia - va;
            unitOff[i] = cb + sWarpB[warp] + ib - vb;
        }
        __syncthreads();
        if (tid == static_cast<int>(blockDim.x) - 1) {
            sCarryA = ca + sWarpA[warp] + ia;
            sCarryB = cb + sWarpB[warp] + ib;
        }
        __syncthreads();
    }
    if (tid == 0) {
        nodeOff[M] = sCarryA;
        unitOff[M] = sCarryB;
    }
}

// Levels with few nodes (the upper meshes: hundreds to thousands of nodes, each in thousands of
// entries) count and place entries through a per-block shared-memory histogram instead: one global
// atomic per (block, node) and shared-memory atomics for the rest. The scatter block takes a
// contiguous slice of the entries, counts it, claims a range per node, then places the slice.
constexpr uint32_t kSmemNodes = 6144;

__global__ void nodeCountSmemKernel(const uint32_t* node, const uint32_t* hdr, uint32_t cap, uint32_t M,
                                    uint32_t* nodeCnt) {
    __shared__ uint32_t hist[kSmemNodes];
    for (uint32_t i = threadIdx.x; i < M; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const uint32_t n = min(hdr[0], cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t nd = node[i];
        if (nd < M) atomicAdd(&hist[nd], 1u);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < M; i += blockDim.x)
        if (hist[i]) atomicAdd(&nodeCnt[i], hist[i]);
}

__global__ void nodeScatterSmemKernel(const uint32_t* node, const uint32_t* hdr, uint32_t cap, uint32_t M,
                                      const uint32_t* nodeOff, uint32_t* cursor, uint32_t* list) {
    __shared__ uint32_t slot[kSmemNodes];
    for (uint32_t i = threadIdx.x; i < M; i += blockDim.x) slot[i] = 0;
    __syncthreads();
    const uint64_t n = min(hdr[0], cap);
    const uint64_t per = (n + gridDim.x - 1) / gridDim.x;
    const uint64_t lo = blockIdx.x * per < n ? blockIdx.x * per : n;
    const uint64_t hi = lo + per < n ? lo + per : n;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint32_t nd = node[i];
        if (nd < M) atomicAdd(&slot[nd], 1u);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < M; i += blockDim.x) {
        const uint32_t c = slot[i];
        slot[i] = c ? nodeOff[i] + atomicAdd(&cursor[i], c) : 0u;
    }
    __syncthreads();
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint32_t nd = node[i];
        if (nd < M) list[atomicAdd(&slot[nd], 1u)] = static_cast<uint32_t>(i);
    }
}

__global__ void nodeScatterKernel(const uint32_t* node, const uint32_t* hdr, uint32_t cap, uint32_t M,
                                  const uint32_t* nodeOff, uint32_t* cursor, uint32_t* list) {
    const uint32_t n = min(hdr[0], cap);
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + lane;
        const uint32_t nd = i < n ? node[i] : M;
        const uint32_t peers = __match_any_sync(0xffffffffu, nd);
        const int leader = __ffs(peers) - 1;
        uint32_t b = 0;
        if (nd < M && static_cast<int>(lane) == leader) b = atomicAdd(&cursor[nd], __popc(peers));
        b = __shfl_sync(0xffffffffu, b, leader);
        if (nd < M) list[nodeOff[nd] + b + __popc(peers & ((1u << lane) - 1u))] = i;
    }
}

constexpr int kNodeMajorThreads = 128;
constexpr int kNodeMajorStage = 128;  // survivors a warp stages in shared memory between appends
constexpr int kNodeMajorChunk = 64;   // children whose float boxes a warp stages in shared memory at once

// One warp per unit (a node and up to 32 of the entries holding it), claimed through a ticket.
// Lanes hold one query's float box each. The loop runs over the node's children with a
// warp-uniform trip count; the children's float boxes are staged in shared memory a chunk at a
// time, so each box is read from memory once per 32 queries. Survivors are staged per warp in
// shared memory and appended with one atomic per flush (at most kNodeMajorStage of them, and at
// the end of the unit), not one per child.
template <int D>
__global__ void __launch_bounds__(kNodeMajorThreads) nodeMajorRangeKernel(NodeMajorArgs a) {
    constexpr uint32_t FULL = 0xffffffffu;
    constexpr int DM = D > 0 ? D : 32;
    __shared__ uint32_t sQ[kNodeMajorThreads / 32][kNodeMajorStage];
    __shared__ uint32_t sJ[kNodeMajorThreads / 32][kNodeMajorStage];
    // (lane, child) pairs whose float boxes meet: the FP64 radius test runs on them 32 at a time,
    // one pair per lane, instead of once per child with the few lanes that passed.
    __shared__ uint32_t sCandJ[kNodeMajorThreads / 32][64];
    __shared__ uint8_t sCandL[kNodeMajorThreads / 32][64];
    // The float boxes of up to kNodeMajorChunk children of the unit's node, copied in with coalesced
    // 16-byte loads by the whole warp (one round of loads instead of one dependent load per child).
    constexpr int kBoxFloats = 2 * (D > 0 ? D : 16);
    constexpr bool kStageBoxes = D > 0 && D % 2 == 0 && D <= 16;
    __shared__ __align__(16) float sBox[kStageBoxes ? kNodeMajorThreads / 32 : 1][kStageBoxes ? kNodeMajorChunk * kBoxFloats : 1];
    if (*a.status & kStatusInconsistent) return;
    const int dim = D > 0 ? D : a.D;
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint32_t lanesLt = (1u << lane) - 1u;
    if (a.inHdr[0] > a.inCap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(a.status, kStatusOverflowEntries);
        return;
    }
    const uint32_t entries = a.inHdr[0];
    const bool root = a.nNodes == 0;
    const uint32_t rootChunk = (a.rootChunk && a.rootChunk < a.rootChildren) ? a.rootChunk : max(1u, a.rootChildren);
    const uint32_t rootChunks = (a.rootChildren + rootChunk - 1) / rootChunk;
    const uint32_t units = root ? (entries + 31u) / 32u * rootChunks : a.unitOff[a.nNodes];
    uint32_t staged = 0;  // warp-uniform
    const double* xp = nullptr;
    // Appends the staged survivors of the current unit (all children of one node, so they share the
    // node's coordinates xp) to the next frontier: one packed atomic claims their entry positions and
    // their children's item range together, a warp scan gives each survivor its child prefix, and
    // each writes its entry (query, node, first child, prefix, coordinates rebuilt as y = P[j] * x)
    // and the tile starts of the next level that fall inside its children.
    auto flush = [&]() {
        if (staged == 0) return;
        __syncwarp();
        uint32_t sum = 0;
        for (uint32_t i = lane; i < staged; i += 32) sum += __ldg(&a.children[sJ[w][i]].cnt);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(FULL, sum, o);
        unsigned long long old = 0;
        if (lane == 0) old = atomicAdd(a.counter, (static_cast<unsigned long long>(sum) << 32) | staged);
        old = __shfl_sync(FULL, old, 0);
        const uint32_t ePos = static_cast<uint32_t>(old);
        const unsigned long long iPos = old >> 32;
        if (lane == 0 && iPos + sum > 0xffffffffull) atomicOr(a.status, kStatusOverflowSum);
        unsigned long long run = iPos;
        for (uint32_t i0 = 0; i0 < staged; i0 += 32) {  // warp-uniform
            const uint32_t i = i0 + lane;
            const bool v = i < staged;
            const uint32_t j = v ? sJ[w][i] : 0u;
            const NodeRec nr = v ? a.children[j] : NodeRec{0.0, 0u, 0u};
            const uint32_t c = v ? nr.cnt : 0u;
            uint32_t inc = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(FULL, inc, o);
                if (lane >= o) inc += t;
            }
            const unsigned long long cp = run + (inc - c);
            run += __shfl_sync(FULL, inc, 31);
            if (!v) continue;
            const uint32_t pos = ePos + i;
            if (pos >= a.out.cap) continue;  // the header kernel reports the overflow
            a.out.q[pos] = sQ[w][i];
            a.out.node[pos] = j;
            a.out.cbeg[pos] = nr.cbeg;
            a.out.cpre[pos] = static_cast<uint32_t>(cp);
            const double* row = a.rows + static_cast<size_t>(j) * dim;
            double* xo = a.out.x + static_cast<size_t>(pos) * dim;
#pragma unroll
            for (int d = 0; d < DM; ++d)
                if (D > 0 || d < dim) xo[d] = __dmul_rn(a.rowsOnHost ? row[d] : __ldg(row + d), __ldg(xp + d));
            for (unsigned long long b = (cp + kWarpTile - 1) / kWarpTile; b * kWarpTile < cp + c; ++b)
                if (b < a.out.tileCap) a.out.tileStart[b] = pos;
        }
        __syncwarp();
        staged = 0;
    };
    while (true) {
        uint32_t u = 0;
        if (lane == 0) u = atomicAdd(a.ticket, 1u);
        u = __shfl_sync(FULL, u, 0);
        if (u >= units) break;
        uint32_t base, count, cbeg, cnt;
        if (root) {
            const uint32_t qu = u / rootChunks;
            base = qu * 32u;
            count = min(32u, entries - base);
            cbeg = (u - qu * rootChunks) * rootChunk;
            cnt = min(rootChunk, a.rootChildren - cbeg);
        } else {
            uint32_t lo = 0, hi = a.nNodes - 1;  // the node whose units hold u: last unitOff[n] <= u
            if (a.unitNode) {
                lo = min(__ldg(a.unitNode + u), a.nNodes - 1);
            } else {
                while (lo < hi) {
                    const uint32_t mid = (lo + hi + 1) >> 1;
                    if (__ldg(a.unitOff + mid) <= u) lo = mid; else hi = mid - 1;
                }
            }
            base = __ldg(a.nodeOff + lo) + (u - __ldg(a.unitOff + lo)) * 32u;
            count = min(32u, __ldg(a.nodeOff + lo + 1) - base);
            const NodeRec pr = a.parents[lo];
            cbeg = pr.cbeg;
            cnt = pr.cnt;
        }
        const bool active = static_cast<uint32_t>(lane) < count;
        uint32_t e = 0, q = 0;
        if (active) {
            e = root ? base + lane : __ldg(a.list + base + lane);
            q = __ldg(a.inQ + e);
            if (a.levelItems) atomicAdd(&a.levelItems[q], cnt);
        }
        // Every entry of the node carries the node's coordinates: take the first one's.
        xp = a.inX + static_cast<size_t>(__shfl_sync(FULL, e, 0)) * dim;
        float ql[DM], qh[DM];
        {
            const float* f = a.boxesF + static_cast<size_t>(q) * 2 * dim;
#pragma unroll
            for (int d = 0; d < DM; ++d) {
                if (D > 0 || d < dim) {
                    ql[d] = active ? __ldg(f + d) : 0.f;
                    qh[d] = active ? __ldg(f + dim + d) : -1.f;
                }
            }
        }
        // The entry-major kernel's radius test (kPredRangeRadius) on the first n queued pairs, one
        // per lane: the child's coordinates rebuilt with one rounded multiply per dimension, the box
        // gap accumulated with fma in dimension order, against the child's subtree radius. Kept
        // pairs are staged for the next frontier.
        uint32_t nCand = 0;  // warp-uniform
        auto testCandidates = [&](uint32_t n) {
            __syncwarp();
            const bool v = static_cast<uint32_t>(lane) < n;
            const uint32_t j = v ? sCandJ[w][lane] : 0u;
            const uint32_t cq = __shfl_sync(FULL, q, v ? sCandL[w][lane] : 0);
            bool keep = false;
            if (v) {
                const NodeRec nr = a.children[j];
                const double* row = a.rows + static_cast<size_t>(j) * dim;
                const double* box = a.boxes + static_cast<size_t>(cq) * 2 * dim;
                double dist = 0.0;
#pragma unroll
                for (int d = 0; d < DM; ++d) {
                    if (D > 0 || d < dim) {
                        const double r = a.rowsOnHost ? row[d] : __ldg(row + d);
                        const double y = __dmul_rn(r, __ldg(xp + d));
                        dist = boxGapAcc(y, __ldg(box + d), __ldg(box + dim + d), dist, 1);
                    }
                }
                keep = nr.cnt > 0 && dist <= __dmul_rn(nr.rad, nr.rad);
            }
            const uint32_t kb = __ballot_sync(FULL, keep);
            if (keep) {
                const uint32_t slot = staged + __popc(kb & lanesLt);
                sQ[w][slot] = cq;
                sJ[w][slot] = j;
            }
            staged += __popc(kb);
            if (staged + 32 > static_cast<uint32_t>(kNodeMajorStage)) flush();
            // Move the pairs past the first n to the front of the queue.
            const uint32_t rest = nCand - n;
            uint32_t tj = 0, tl = 0;
            if (static_cast<uint32_t>(lane) < rest) {
                tj = sCandJ[w][n + lane];
                tl = sCandL[w][n + lane];
            }
            __syncwarp();
            if (static_cast<uint32_t>(lane) < rest) {
                sCandJ[w][lane] = tj;
                sCandL[w][lane] = static_cast<uint8_t>(tl);
            }
            nCand = rest;
        };
        for (uint32_t c = 0; c < cnt; ++c) {
            const uint32_t j = cbeg + c;
            const float* b = a.aabb + static_cast<size_t>(j) * 2 * dim;
            if constexpr (kStageBoxes) {
                if (c % kNodeMajorChunk == 0) {  // warp-uniform: stage the next chunk of boxes
                    const uint32_t n = min(static_cast<uint32_t>(kNodeMajorChunk), cnt - c);
                    const float4* src = reinterpret_cast<const float4*>(b);
                    float4* dst = reinterpret_cast<float4*>(sBox[w]);
                    __syncwarp();
                    for (uint32_t i = lane; i < n * (kBoxFloats / 4); i += 32) dst[i] = __ldg(src + i);
                    __syncwarp();
                }
                b = sBox[w] + (c % kNodeMajorChunk) * kBoxFloats;
            }
            bool pass = active;
            constexpr int C = chunkOf<D>();
#pragma unroll
            for (int d = 0; d < DM; d += C) {
                if (D > 0 || d < dim) {
                    float cl[C], ch[C];
                    if constexpr (kStageBoxes) {
#pragma unroll
                        for (int i = 0; i < C; ++i) {
                            cl[i] = b[d + i];
                            ch[i] = b[dim + d + i];
                        }
                    } else {
                        ldChunkF<C>(b + d, cl);
                        ldChunkF<C>(b + dim + d, ch);
                    }
#pragma unroll
                    for (int i = 0; i < C; ++i) pass = pass && cl[i] <= qh[d + i] && ch[i] >= ql[d + i];
                }
            }
            const uint32_t pb = __ballot_sync(FULL, pass);
            if (pb == 0) continue;
            if (pass) {
                const uint32_t slot = nCand + __popc(pb & lanesLt);
                sCandJ[w][slot] = j;
                sCandL[w][slot] = static_cast<uint8_t>(lane);
            }
            nCand += __popc(pb);  // at most 31 + 32 < 64
            if (nCand >= 32) testCandidates(32);
        }
        if (nCand) testCandidates(nCand);
        flush();
    }
}

__global__ void frontierHeaderKernel(const unsigned long long* counter, uint32_t* hdr, uint32_t cap, uint32_t tileCap,
                                     uint32_t* status) {
    const unsigned long long c = *counter;
    const uint32_t entries = static_cast<uint32_t>(c), items = static_cast<uint32_t>(c >> 32);
    hdr[0] = entries;
    hdr[1] = items;
    if (entries > cap) atomicOr(status, kStatusOverflowEntries);
    if ((static_cast<unsigned long long>(items) + kWarpTile - 1) / kWarpTile > tileCap)
        atomicOr(status, kStatusOverflowItems);
}

__global__ void oneItemHeaderKernel(const uint32_t* count, uint32_t* hdr) {
    const uint32_t c = *count;
    hdr[0] = c;
    hdr[1] = c;
}

__global__ void groupResultsKernel(const uint64_t* rawIds, const uint32_t* rawQ, const double* rawVals,
                                   const uint32_t* hdr, uint32_t cap, int D, const uint64_t* offsets, uint32_t* cursor,
                                   uint64_t* ids, double* vals) {
    const uint32_t n = min(hdr[0], cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t q = rawQ[i];
        const uint64_t pos = offsets[q] + atomicAdd(&cursor[q], 1u);
        if (pos >= cap) continue;  // more results than the buffers hold: the batch reruns after growth
        ids[pos] = rawIds[i];
        if (vals)
            for (int d = 0; d < D; ++d) vals[pos * D + d] = rawVals[static_cast<size_t>(i) * D + d];
    }
}

int residentGrid(const void* kern, int threads, int percent) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        TBLAEQ_CUDA(cudaGetDevice(&dev));
        TBLAEQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    int perSm = 0;
    TBLAEQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, threads, 0));
    const int pct = (percent > 0 && percent < 100) ? percent : 100;
    return std::max(1, (sms * std::max(1, perSm) * pct + 99) / 100);
}

template <int D>
void launchNodeMajorD(const NodeMajorArgs& a, int gridPercent, cudaStream_t s) {
    static int full = 0;
    if (full == 0) full = residentGrid(reinterpret_cast<const void*>(nodeMajorRangeKernel<D>), kNodeMajorThreads, 100);
    const int pct = (gridPercent > 0 && gridPercent < 100) ? gridPercent : 100;
    const int grid = std::max(1, (full * pct + 99) / 100);
    nodeMajorRangeKernel<D><<<grid, kNodeMajorThreads, 0, s>>>(a);
    TBLAEQ_LAUNCHED();
}

int smallGrid(uint64_t work) { return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((work + 255) / 256, 148 * 8))); }

}  // namespace

// One warp per node; its lanes write the node's units.
__global__ void unitNodeKernel(const uint32_t* unitOff, uint32_t M, uint32_t* unitNode, uint32_t unitCap) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * blockDim.x / 32u;
    for (uint32_t n = (blockIdx.x * blockDim.x + threadIdx.x) / 32u; n < M; n += warps) {
        const uint32_t u1 = min(unitOff[n + 1], unitCap);
        for (uint32_t u = unitOff[n] + lane; u < u1; u += 32u) unitNode[u] = n;
    }
}

void launchNodeTranspose(const uint32_t* node, const uint32_t* hdr, uint32_t cap, uint32_t nNodes, uint32_t* nodeCnt,
                         uint32_t* nodeOff, uint32_t* unitOff, uint32_t* cursor, uint32_t* list, cudaStream_t s,
                         uint32_t* unitNode, uint32_t unitCap) {
    const bool smem = nNodes <= kSmemNodes;
    if (smem)
        nodeCountSmemKernel<<<smallGrid(cap), 256, 0, s>>>(node, hdr, cap, nNodes, nodeCnt);
    else
        nodeCountKernel<<<smallGrid(cap), 256, 0, s>>>(node, hdr, cap, nNodes, nodeCnt);
    TBLAEQ_LAUNCHED();
    nodeScanKernel<<<1, 1024, 0, s>>>(nodeCnt, nNodes, nodeOff, unitOff);
    TBLAEQ_LAUNCHED();
    if (unitNode) {
        unitNodeKernel<<<smallGrid(static_cast<uint64_t>(nNodes) * 32), 256, 0, s>>>(unitOff, nNodes, unitNode, unitCap);
        TBLAEQ_LAUNCHED();
    }
    if (smem)
        nodeScatterSmemKernel<<<smallGrid(cap), 256, 0, s>>>(node, hdr, cap, nNodes, nodeOff, cursor, list);
    else
        nodeScatterKernel<<<smallGrid(cap), 256, 0, s>>>(node, hdr, cap, nNodes, nodeOff, cursor, list);
    TBLAEQ_LAUNCHED();
}

void launchNodeMajorRange(const NodeMajorArgs& a, int gridPercent, cudaStream_t s) {
    switch (a.D) {
        case 2: return launchNodeMajorD<2>(a, gridPercent, s);
        case 3: return launchNodeMajorD<3>(a, gridPercent, s);
        case 4: return launchNodeMajorD<4>(a, gridPercent, s);
        case 5: return launchNodeMajorD<5>(a, gridPercent, s);
        case 8: return launchNodeMajorD<8>(a, gridPercent, s);
        case 16: return launchNodeMajorD<16>(a, gridPercent, s);
        default:
            if (a.D < 1 || a.D > 32) throw std::invalid_argument("node-major level: D must be in [1, 32]");
            return launchNodeMajorD<0>(a, gridPercent, s);
    }
}

void launchFrontierHeader(const unsigned long long* counter, uint32_t* hdr, uint32_t cap, uint32_t tileCap,
                          uint32_t* status, cudaStream_t s) {
    frontierHeaderKernel<<<1, 1, 0, s>>>(counter, hdr, cap, tileCap, status);
    TBLAEQ_LAUNCHED();
}

void launchOneItemHeader(const uint32_t* count, uint32_t* hdr, cudaStream_t s) {
    oneItemHeaderKernel<<<1, 1, 0, s>>>(count, hdr);
    TBLAEQ_LAUNCHED();
}

void launchGroupResults(const uint64_t* rawIds, const uint32_t* rawQ, const double* rawVals, const uint32_t* hdr,
                        uint32_t cap, int D, const uint64_t* offsets, uint32_t* cursor, uint64_t* ids, double* vals,
                        cudaStream_t s) {
    groupResultsKernel<<<smallGrid(cap), 256, 0, s>>>(rawIds, rawQ, rawVals, hdr, cap, D, offsets, cursor, ids, vals);
    TBLAEQ_LAUNCHED();
}

}  // namespace tblaeq
