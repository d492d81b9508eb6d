// Level-synchronous traversal kernels (see traverse.cuh for the design).
#include "traverse.cuh"

#include <cuda/atomic>

#include <algorithm>

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
                         uint32_t* status, unsigned long long& exCnt, unsigned long long& exSum) {
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
            if (++spins > kSpinLimit) {
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

// Squared distance from y to the box [lo, hi] with the reference's accumulation
// (RangePruning.cu:7-20; nvcc contracts `dist += diff * diff` into an fma by default).
template <int DM>
__device__ __forceinline__ double boxDist2(const double* y, const double* lo, const double* hi, int D, int useFma) {
    double dist = 0.0;
#pragma unroll
    for (int d = 0; d < DM; ++d) {
        if (d < D) {
            const double cv = y[d];
            const double l = lo[d], h = hi[d];
            double diff = 0.0;
            if (cv < l) {
                diff = l - cv;
            } else if (cv > h) {
                diff = cv - h;
            }
            dist = useFma ? __fma_rn(diff, diff, dist) : __dadd_rn(dist, __dmul_rn(diff, diff));
        }
    }
    return dist;
}

template <int DM>
__device__ __forceinline__ double pointDist2(const double* y, const double* p, int D, int useFma) {
    double dist = 0.0;
#pragma unroll
    for (int d = 0; d < DM; ++d) {
        if (d < D) {
            const double diff = p[d] - y[d];
            dist = useFma ? __fma_rn(diff, diff, dist) : __dadd_rn(dist, __dmul_rn(diff, diff));
        }
    }
    return dist;
}

// Rebuilds item (entry e, row j): y = rows[j] (*) x_e, one rounded multiply per dimension.
template <int D, int DM>
__device__ __forceinline__ void rebuild(const ExpandArgs& a, int dim, uint32_t e, uint32_t j, double (&y)[DM]) {
    const double* xp = a.in.x + static_cast<size_t>(e) * dim;
    const double* rp = a.child.rows + static_cast<size_t>(j) * dim;
    if constexpr (D > 0 && (D % 2) == 0) {
#pragma unroll
        for (int d = 0; d < D; d += 2) {
            const double2 pv = __ldg(reinterpret_cast<const double2*>(rp + d));
            const double2 xv = __ldg(reinterpret_cast<const double2*>(xp + d));
            y[d] = __dmul_rn(pv.x, xv.x);
            y[d + 1] = __dmul_rn(pv.y, xv.y);
        }
    } else {
#pragma unroll
        for (int d = 0; d < DM; ++d) {
            if (d < dim) y[d] = __dmul_rn(__ldg(rp + d), __ldg(xp + d));
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
    static constexpr int kCacheBytes = 3 * kRounds * 32 * 4;
    static constexpr int kWindow = kWarpTile + 1;  // most entries a tile can overlap
    static constexpr int kWindowBytes = 3 * kWindow * 4 + 4;
    static constexpr int kWarpBytes = kRowBytes + kNodeBytes + kCacheBytes + ((kWindowBytes + 15) / 16) * 16;
};

// Launch shape of the expand kernels (independent warps per CTA and the register bound). These are
// build-time tuning knobs; the defaults are the fastest measured on B200 for the benchmark index.
#ifndef TBLAEQ_EXPAND_THREADS
#define TBLAEQ_EXPAND_THREADS 128
#endif
#ifndef TBLAEQ_EXPAND_MIN_BLOCKS
#define TBLAEQ_EXPAND_MIN_BLOCKS 8
#endif
#ifndef TBLAEQ_EXPAND_CACHE
#define TBLAEQ_EXPAND_CACHE 0
#endif
constexpr int kExpandThreads = TBLAEQ_EXPAND_THREADS;

template <int D, bool STAGED>
constexpr size_t expandSmemBytes() {
    return static_cast<size_t>(Staging<D, STAGED>::kWarpBytes) * (kExpandThreads / 32);
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

template <int PRED, bool TO_RESULT>
constexpr bool needsNode() {
    return PRED == kPredRangeRadius || PRED == kPredKnnBound || (!TO_RESULT && (PRED == kPredMask || PRED == kPredAll));
}

// Applies the level predicate to a rebuilt item; cc receives the item's child count when the
// output is a frontier.
// Per-lane register cache of the current query's box (range) or point (KNN) and bound, reloaded
// only when the item's query changes (queries change at entry boundaries, rarely within a warp).
template <int DM, int PRED>
struct QueryCache {
    static constexpr bool kRange = PRED == kPredRangeRadius || PRED == kPredRangeBox;
    static constexpr bool kKnn = PRED == kPredKnnBound || PRED == kPredKnnPoint;
    uint32_t q = 0xffffffffu;
    double lo[(kRange || kKnn) ? DM : 1];
    double hi[kRange ? DM : 1];
    double tau = 0.0;
    __device__ __forceinline__ void load(const ExpandArgs& a, int dim, uint32_t nq) {
        if (TBLAEQ_EXPAND_CACHE && nq == q) return;
        q = nq;
        if constexpr (kRange) {
            const double* box = a.query.boxes + static_cast<size_t>(nq) * 2 * dim;
#pragma unroll
            for (int d = 0; d < DM; ++d) {
                if (d < dim) {
                    lo[d] = __ldg(box + d);
                    hi[d] = __ldg(box + dim + d);
                }
            }
        } else if constexpr (kKnn) {
            const double* p = a.query.points + static_cast<size_t>(nq) * dim;
#pragma unroll
            for (int d = 0; d < DM; ++d)
                if (d < dim) lo[d] = __ldg(p + d);
        }
    }
};

// Per-lane register cache of the parent entry's coordinates.
template <int D, int DM>
struct ParentCache {
    uint32_t e = 0xffffffffu;
    double x[DM];
    __device__ __forceinline__ void load(const ExpandArgs& a, int dim, uint32_t ne) {
        if (TBLAEQ_EXPAND_CACHE && ne == e) return;
        e = ne;
        const double* xp = a.in.x + static_cast<size_t>(ne) * dim;
        if constexpr (D > 0 && (D % 2) == 0) {
#pragma unroll
            for (int d = 0; d < D; d += 2) {
                const double2 v = __ldg(reinterpret_cast<const double2*>(xp + d));
                x[d] = v.x;
                x[d + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int d = 0; d < DM; ++d)
                if (d < dim) x[d] = __ldg(xp + d);
        }
    }
};

template <int DM, int PRED, bool TO_RESULT>
__device__ __forceinline__ bool testItem(const ExpandArgs& a, int dim, const double (&y)[DM],
                                         const QueryCache<DM, PRED>& qc, uint32_t j, uint32_t kk, const NodeRec& nr,
                                         uint32_t& cc) {
    cc = 0;
    if constexpr (PRED == kPredRangeRadius) {
        const double dist = boxDist2<DM>(y, qc.lo, qc.hi, dim, a.useFma);
        cc = nr.cnt;
        bool keep = (cc > 0) && (dist <= __dmul_rn(nr.rad, nr.rad));
        if (keep && a.child.aabb) {
            // Exact mode only: the query box must also meet the box of the points below the child.
            const float* b = a.child.aabb + static_cast<size_t>(kk) * 2 * dim;
#pragma unroll
            for (int d = 0; d < DM; ++d) {
                if (d < dim) {
                    keep = keep && (static_cast<double>(__ldg(b + d)) <= qc.hi[d]) &&
                           (static_cast<double>(__ldg(b + dim + d)) >= qc.lo[d]);
                }
            }
        }
        return keep;
    } else if constexpr (PRED == kPredMask) {
        bool keep = a.child.mask[j] != 0;
        if constexpr (!TO_RESULT) {
            cc = nr.cnt;
            keep = keep && cc > 0;
        }
        return keep;
    } else if constexpr (PRED == kPredAll) {
        if constexpr (!TO_RESULT) {
            cc = nr.cnt;
            return cc > 0;
        }
        return true;
    } else if constexpr (PRED == kPredRangeBox) {
        bool in = true;
#pragma unroll
        for (int d = 0; d < DM; ++d) {
            if (d < dim) in = in && (qc.lo[d] <= y[d]) && (y[d] <= qc.hi[d]);
        }
        return in;
    } else if constexpr (PRED == kPredKnnBound) {
        // Distance bounds of the points below the child: sphere (centre distance -/+ subtree radius)
        // and, when present, its box (outward-rounded, so slightly widened bounds stay conservative).
        const double dd = sqrt(pointDist2<DM>(y, qc.lo, dim, 1));
        double lb = dd - nr.rad, ub = dd + nr.rad;
        if (a.child.aabb) {
            const float* b = a.child.aabb + static_cast<size_t>(kk) * 2 * dim;
            double gapSum = 0.0, farSum = 0.0;
#pragma unroll
            for (int d = 0; d < DM; ++d) {
                if (d < dim) {
                    const double l = static_cast<double>(__ldg(b + d)), h = static_cast<double>(__ldg(b + dim + d));
                    const double g = fmax(fmax(l - qc.lo[d], qc.lo[d] - h), 0.0);
                    const double f = fmax(qc.lo[d] - l, h - qc.lo[d]);
                    gapSum = __fma_rn(g, g, gapSum);
                    farSum = __fma_rn(f, f, farSum);
                }
            }
            lb = fmax(lb, sqrt(gapSum) * (1.0 - 1e-12));
            ub = fmin(ub, sqrt(farSum) * (1.0 + 1e-12));
        }
        cc = nr.cnt;
        const uint32_t q = qc.q;
        double tau = __ldcg(a.query.tau + q);
        // Any child with K points below it bounds the K-th neighbour distance by its far distance.
        if (ub < tau && __ldg(a.child.leaf + kk) >= __ldg(a.query.k + q)) {
            atomicMin(reinterpret_cast<unsigned long long*>(a.query.tau + q), __double_as_longlong(ub));
            tau = ub;
        }
        return (cc > 0) && (lb <= tau);
    } else {  // kPredKnnPoint
        if (a.wave == 1) return true;  // every point of a selected entry
        const double t = __ldcg(a.query.tau + qc.q);
        return pointDist2<DM>(y, qc.lo, dim, 1) <= t * t * (1.0 + 1e-9);
    }
}

template <int D, int PRED, bool TO_RESULT, bool STAGED>
__global__ void __launch_bounds__(kExpandThreads, TBLAEQ_EXPAND_MIN_BLOCKS) expandKernel(ExpandArgs a) {
    using S = Staging<D, STAGED>;
    constexpr int R = S::kRounds;
    constexpr int DM = (D > 0) ? D : 32;
    constexpr bool NODE = needsNode<PRED, TO_RESULT>();
    constexpr uint32_t FULL = 0xffffffffu;
    extern __shared__ __align__(16) unsigned char smem[];
    const int dim = (D > 0) ? D : a.D;
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint32_t lanesLe = (2u << lane) - 1u;  // lanes 0..lane (wraps to all lanes for lane 31)
    const uint32_t lanesLt = (1u << lane) - 1u;
    unsigned char* warpSmem = smem + static_cast<size_t>(w) * S::kWarpBytes;
    unsigned char* rowBuf = warpSmem;                                    // [kStages][32][kStride]
    NodeRec* nodeBuf = reinterpret_cast<NodeRec*>(warpSmem + S::kRowBytes);  // [kStages][32]
    uint32_t* sRow = reinterpret_cast<uint32_t*>(warpSmem + S::kRowBytes + S::kNodeBytes);  // [R][32]
    uint32_t* sEnt = sRow + R * 32;
    uint32_t* sQ = sEnt + R * 32;
    uint32_t* wCp = sQ + R * 32;  // window of the tile's entries: prefix, first child, query
    uint32_t* wCb = wCp + S::kWindow;
    uint32_t* wQ = wCb + S::kWindow;

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
        const uint32_t t0 = tile * kWarpTile;

        // ---- phase A: stage the tile's entries in shared memory (one round of parallel loads),
        // then map every item of the tile to its entry and child row.
        const uint32_t eLo = a.in.tileStart[tile];
        uint32_t eHi = (tile + 1 < nTiles) ? a.in.tileStart[tile + 1] : entries - 1;
        if (eHi >= entries) eHi = entries - 1;
        uint32_t W = eHi - eLo + 1;
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
            if (rs >= total) continue;  // warp-uniform
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
            sEnt[r * 32 + lane] = eLo + e;
            sQ[r * 32 + lane] = wQ[e];
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
                if ((validBits >> r) & 1u) {
                    const uint32_t j = sRow[r * 32 + lane];
                    const int slot = r % S::kStages;
                    const unsigned char* src = reinterpret_cast<const unsigned char*>(a.child.rows) +
                                               static_cast<size_t>(j) * (8 * D);
                    unsigned char* dst = rowBuf + (slot * 32 + lane) * S::kStride;
#pragma unroll
                    for (int c = 0; c < S::kChunks; ++c) {
                        if constexpr (S::kChunk == 16) {
                            cpAsync16(dst + 16 * c, src + 16 * c);
                        } else {
                            cpAsync8(dst + 8 * c, src + 8 * c);
                        }
                    }
                    if constexpr (NODE) {
                        const uint32_t kk = a.child.keys ? static_cast<uint32_t>(a.child.keys[j]) : j;
                        cpAsync16(&nodeBuf[slot * 32 + lane], &a.child.nodes[kk]);
                    }
                }
            }
        };
        if constexpr (S::kOn) {
#pragma unroll
            for (int r = 0; r < S::kStages - 1; ++r) {
                if (r < R) issue(r);
                cpAsyncCommit();
            }
        }
        uint32_t keepBits = 0, aggCnt = 0, aggSum = 0;
        QueryCache<DM, PRED> qc;
        ParentCache<D, DM> pc;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if constexpr (S::kOn) {
                if (r + S::kStages - 1 < R) issue(r + S::kStages - 1);
                cpAsyncCommit();
                cpAsyncWait<S::kStages - 1>();
            }
            if (t0 + r * 32 >= total) continue;  // warp-uniform
            const bool valid = (validBits >> r) & 1u;
            bool keep = false;
            uint32_t cc = 0;
            bool work = valid;
            if (PRED == kPredKnnPoint && valid && a.wave != 0) {
                // Two-wave KNN: decide from the entry alone before touching the child's row.
                const uint32_t e = sEnt[r * 32 + lane];
                const bool sel = __ldg(a.child.entrySel + e) != 0;
                if (a.wave == 1) {
                    work = sel;
                } else {
                    work = !sel && __ldg(a.child.entryLb + e) <= __ldcg(a.query.tau + sQ[r * 32 + lane]);
                }
            }
            if (work) {
                const uint32_t j = sRow[r * 32 + lane];
                const uint32_t e = sEnt[r * 32 + lane];
                const uint32_t q = sQ[r * 32 + lane];
                double y[DM];
                NodeRec nr{0.0, 0u, 0u};
                uint32_t kk = j;
                qc.load(a, dim, q);
                pc.load(a, dim, e);
                if constexpr (S::kOn) {
                    const int slot = r % S::kStages;
                    const double* rowp = reinterpret_cast<const double*>(rowBuf + (slot * 32 + lane) * S::kStride);
                    if constexpr (D % 2 == 0) {
#pragma unroll
                        for (int d = 0; d < D; d += 2) {
                            const double2 pv = *reinterpret_cast<const double2*>(rowp + d);
                            y[d] = __dmul_rn(pv.x, pc.x[d]);
                            y[d + 1] = __dmul_rn(pv.y, pc.x[d + 1]);
                        }
                    } else {
#pragma unroll
                        for (int d = 0; d < D; ++d) y[d] = __dmul_rn(rowp[d], pc.x[d]);
                    }
                    if constexpr (NODE) nr = nodeBuf[slot * 32 + lane];
                    kk = a.child.keys ? static_cast<uint32_t>(a.child.keys[j]) : j;
                } else {
                    const double* rp = a.child.rows + static_cast<size_t>(j) * dim;
                    if constexpr (D > 0 && (D % 2) == 0) {
#pragma unroll
                        for (int d = 0; d < D; d += 2) {
                            const double2 pv = __ldg(reinterpret_cast<const double2*>(rp + d));
                            y[d] = __dmul_rn(pv.x, pc.x[d]);
                            y[d + 1] = __dmul_rn(pv.y, pc.x[d + 1]);
                        }
                    } else {
#pragma unroll
                        for (int d = 0; d < DM; ++d)
                            if (d < dim) y[d] = __dmul_rn(__ldg(rp + d), pc.x[d]);
                    }
                    kk = a.child.keys ? static_cast<uint32_t>(a.child.keys[j]) : j;
                    if constexpr (NODE) nr = a.child.nodes[kk];
                }
                keep = testItem<DM, PRED, TO_RESULT>(a, dim, y, qc, j, kk, nr, cc);
            }
            if (a.scratch.work) warpRows += __popc(__ballot_sync(FULL, work));
            // Per-query generated-children counts (the reference's levelFineMeshSize).
            if (a.scratch.levelItems) {
                const uint32_t vm = __ballot_sync(FULL, valid);
                if (valid) {
                    const uint32_t q = sQ[r * 32 + lane];
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

        // ---- publish the tile's counts and learn where its output starts.
        unsigned long long exCnt, exSum;
        lookback(a.scratch.desc, tile, aggCnt, aggSum, a.scratch.status, exCnt, exSum);
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
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const bool keep = (keepBits >> r) & 1u;
            const uint32_t kb = __ballot_sync(FULL, keep);
            if (kb == 0) continue;  // warp-uniform
            const uint32_t j = sRow[r * 32 + lane];
            const uint32_t qr = sQ[r * 32 + lane];
            uint32_t cc = 0, ncb = 0, kk = 0;
            double y[DM];
            if (keep) {
                rebuild<D, DM>(a, dim, sEnt[r * 32 + lane], j, y);
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
                        a.rout.ids[pos] = a.child.outMap ? a.child.outMap[j] : static_cast<uint64_t>(kk);
                        if (a.rout.vals) {
#pragma unroll
                            for (int d = 0; d < DM; ++d)
                                if (d < dim) a.rout.vals[pos * dim + d] = y[d];
                        }
                        if (a.rout.q) a.rout.q[pos] = qr;
                        if constexpr (PRED == kPredKnnPoint) {
                            if (a.rout.dist2) {
                                const double* p = a.query.points + static_cast<size_t>(qr) * dim;
                                a.rout.dist2[pos] = pointDist2<DM>(y, p, dim, 1);
                            }
                        }
                    }
                } else if (pos < a.fout.cap) {
                    const unsigned long long cp = runSum + (inc - v);
                    a.fout.q[pos] = qr;
                    a.fout.node[pos] = kk;
                    a.fout.cbeg[pos] = ncb;
                    a.fout.cpre[pos] = static_cast<uint32_t>(cp);
#pragma unroll
                    for (int d = 0; d < DM; ++d)
                        if (d < dim) a.fout.x[pos * dim + d] = y[d];
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

__global__ void exclusiveScanKernel(const uint32_t* counts, uint64_t* offsets, uint32_t n) {
    __shared__ unsigned long long sCarry;
    __shared__ unsigned long long sWarp[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) sCarry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n; base += blockDim.x) {
        const uint32_t i = base + tid;
        const unsigned long long v = (i < n) ? counts[i] : 0;
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
        if (i < n) offsets[i] = carry + sWarp[warp] + inc - v;
        __syncthreads();
        if (tid == blockDim.x - 1) sCarry = carry + sWarp[warp] + inc;
        __syncthreads();
    }
    if (tid == 0) offsets[n] = sCarry;
}

template <int D, int PRED, bool TO_RESULT, bool STAGED>
void launchOne(const ExpandArgs& a, int gridBlocks, cudaStream_t s) {
    auto kern = expandKernel<D, PRED, TO_RESULT, STAGED>;
    constexpr size_t smemBytes = expandSmemBytes<D, STAGED>();
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
    if (gridBlocks <= 0) gridBlocks = cached;
    kern<<<gridBlocks, kExpandThreads, smemBytes, s>>>(a);
    TBLAEQ_CUDA(cudaGetLastError());
}

template <int D, bool ST>
void dispatchPred(const ExpandArgs& a, int pred, bool toResult, int g, cudaStream_t s) {
    if (toResult) {
        switch (pred) {
            case kPredAll: return launchOne<D, kPredAll, true, ST>(a, g, s);
            case kPredRangeBox: return launchOne<D, kPredRangeBox, true, ST>(a, g, s);
            case kPredMask: return launchOne<D, kPredMask, true, ST>(a, g, s);
            case kPredKnnPoint: return launchOne<D, kPredKnnPoint, true, ST>(a, g, s);
            default: break;
        }
    } else {
        switch (pred) {
            case kPredRangeRadius: return launchOne<D, kPredRangeRadius, false, ST>(a, g, s);
            case kPredMask: return launchOne<D, kPredMask, false, ST>(a, g, s);
            case kPredAll: return launchOne<D, kPredAll, false, ST>(a, g, s);
            case kPredKnnBound: return launchOne<D, kPredKnnBound, false, ST>(a, g, s);
            default: break;
        }
    }
    throw std::invalid_argument("expand: unsupported predicate/output combination");
}

template <int D>
void dispatchStaged(const ExpandArgs& a, int pred, bool toResult, int g, cudaStream_t s) {
    if (a.variant == kVariantStaged) return dispatchPred<D, true>(a, pred, toResult, g, s);
    return dispatchPred<D, false>(a, pred, toResult, g, s);
}

}  // namespace

void launchExpand(const ExpandArgs& a, int pred, bool toResult, int gridBlocks, cudaStream_t stream) {
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
    TBLAEQ_CUDA(cudaGetLastError());
}

void launchExclusiveScan(const uint32_t* counts, uint64_t* offsets, uint32_t n, cudaStream_t stream) {
    exclusiveScanKernel<<<1, 1024, 0, stream>>>(counts, offsets, n);
    TBLAEQ_CUDA(cudaGetLastError());
}

}  // namespace tblaeq
