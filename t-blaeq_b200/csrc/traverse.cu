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

// Up to D = 8 the rebuilt coordinates fit 64 registers (4 CTAs per SM); wider rows get 2 CTAs.
template <int D>
constexpr int minBlocksFor() {
    return (D > 0 && D <= 8) ? 4 : 2;
}

template <int D, int PRED, bool TO_RESULT>
__global__ void __launch_bounds__(kThreads, minBlocksFor<D>()) expandKernel(ExpandArgs a) {
    constexpr int R = kWarpTile / 32;  // rounds of 32 items per warp tile
    // Per-warp cache of every item's row, entry and query between the two passes.
    __shared__ uint32_t sRow[kThreads / 32][R][32];
    __shared__ uint32_t sEnt[kThreads / 32][R][32];
    __shared__ uint32_t sQ[kThreads / 32][R][32];
    constexpr int DM = (D > 0) ? D : 32;
    constexpr uint32_t FULL = 0xffffffffu;
    const int dim = (D > 0) ? D : a.D;
    const int lane = threadIdx.x & 31;
    const uint32_t lanesLe = (2u << lane) - 1u;  // lanes 0..lane (wraps to all lanes for lane 31)
    const uint32_t lanesLt = (1u << lane) - 1u;

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

    while (true) {
        uint32_t tile = 0;
        if (lane == 0) tile = atomicAdd(a.scratch.ticket, 1u);
        tile = __shfl_sync(FULL, tile, 0);
        if (tile >= nTiles) break;
        const uint32_t t0 = tile * kWarpTile;

        // ---- pass 1: map every item to its entry, rebuild it and test it; keep one bit per item.
        uint32_t keepBits = 0, aggCnt = 0, aggSum = 0;
        const int w = threadIdx.x >> 5;
        uint32_t cur = a.in.tileStart[tile];  // entry holding the first item of the round
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const uint32_t rs = t0 + r * 32;
            if (rs >= total) continue;  // warp-uniform
            const uint32_t k = rs + lane;
            const bool valid = k < total;
            // The 32 entries from `cur` cover every entry overlapping this round unless entries with
            // fewer than one child per lane follow (then each lane searches on its own).
            const uint32_t ce = cur + lane;
            const bool inRange = ce < entries;
            const uint32_t cp = inRange ? a.in.cpre[ce] : 0xffffffffu;
            const uint32_t cp31 = __shfl_sync(FULL, cp, 31);
            uint32_t e, eCp, eCb, eQ;
            if (cp31 + 1 < rs + 32 && cur + 32 < entries) {
                uint32_t lo = cur, hi = entries - 1;
                const uint32_t kk = valid ? k : rs;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi + 1) >> 1;
                    if (a.in.cpre[mid] <= kk) lo = mid; else hi = mid - 1;
                }
                e = lo;
                eCp = a.in.cpre[e];
                eCb = a.in.cbeg[e];
                eQ = a.in.q[e];
            } else {
                const uint32_t cb = inRange ? a.in.cbeg[ce] : 0u;
                const uint32_t cq = inRange ? a.in.q[ce] : 0u;
                const uint32_t base = __popc(__ballot_sync(FULL, cp <= rs)) - 1u;
                const uint32_t off = cp - rs;
                const uint32_t starts = __reduce_or_sync(FULL, (cp > rs && off < 32u) ? (1u << off) : 0u);
                const uint32_t my = base + __popc(starts & lanesLe);
                e = cur + my;
                eCp = __shfl_sync(FULL, cp, my);
                eCb = __shfl_sync(FULL, cb, my);
                eQ = __shfl_sync(FULL, cq, my);
            }
            cur = __shfl_sync(FULL, e, 31);
            const uint32_t j = eCb + (k - eCp);
            sRow[w][r][lane] = j;
            sEnt[w][r][lane] = e;
            sQ[w][r][lane] = eQ;

            bool keep = false;
            uint32_t cc = 0;
            if (valid) {
                double y[DM];
                rebuild<D, DM>(a, dim, e, j, y);
                const uint32_t kk = a.child.keys ? static_cast<uint32_t>(a.child.keys[j]) : j;
                if constexpr (PRED == kPredRangeRadius) {
                    const double* box = a.query.boxes + static_cast<size_t>(eQ) * 2 * dim;
                    const double dist = boxDist2<DM>(y, box, box + dim, dim, a.useFma);
                    const NodeRec nr = a.child.nodes[kk];
                    cc = nr.cnt;
                    keep = (cc > 0) && (dist <= __dmul_rn(nr.rad, nr.rad));
                } else if constexpr (PRED == kPredMask) {
                    keep = a.child.mask[j] != 0;
                    if constexpr (!TO_RESULT) {
                        cc = a.child.nodes[kk].cnt;
                        keep = keep && cc > 0;
                    }
                } else if constexpr (PRED == kPredAll) {
                    keep = true;
                    if constexpr (!TO_RESULT) {
                        cc = a.child.nodes[kk].cnt;
                        keep = cc > 0;
                    }
                } else if constexpr (PRED == kPredRangeBox) {
                    const double* box = a.query.boxes + static_cast<size_t>(eQ) * 2 * dim;
                    bool in = true;
#pragma unroll
                    for (int d = 0; d < DM; ++d) {
                        if (d < dim) in = in && (box[d] <= y[d]) && (y[d] <= box[dim + d]);
                    }
                    keep = in;
                } else if constexpr (PRED == kPredKnnBound) {
                    const double* p = a.query.points + static_cast<size_t>(eQ) * dim;
                    const double dd = sqrt(pointDist2<DM>(y, p, dim, 1));
                    const NodeRec nr = a.child.nodes[kk];
                    cc = nr.cnt;
                    keep = (cc > 0) && (dd - nr.rad <= a.query.tau[eQ]);
                } else if constexpr (PRED == kPredKnnPoint) {
                    const double* p = a.query.points + static_cast<size_t>(eQ) * dim;
                    const double t = a.query.tau[eQ];
                    keep = pointDist2<DM>(y, p, dim, 1) <= t * t;
                }
            }
            // Per-query generated-children counts (the reference's levelFineMeshSize).
            if (a.scratch.levelItems) {
                const uint32_t vm = __ballot_sync(FULL, valid);
                if (valid) {
                    const uint32_t peers = __match_any_sync(vm, eQ);
                    if (lane == __ffs(peers) - 1) atomicAdd(&a.scratch.levelItems[eQ], __popc(peers));
                }
            }
            const uint32_t kb = __ballot_sync(FULL, keep);
            keepBits |= (keep ? 1u : 0u) << r;
            aggCnt += __popc(kb);
            uint32_t s = keep ? cc : 0u;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
            aggSum += s;
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
            const uint32_t j = sRow[w][r][lane];
            const uint32_t qr = sQ[w][r][lane];
            uint32_t cc = 0, ncb = 0, kk = 0;
            double y[DM];
            if (keep) {
                rebuild<D, DM>(a, dim, sEnt[w][r][lane], j, y);
                kk = a.child.keys ? static_cast<uint32_t>(a.child.keys[j]) : j;
                if constexpr (!TO_RESULT) {
                    const NodeRec nr = a.child.nodes[kk];
                    cc = nr.cnt;
                    ncb = nr.cbeg;
                }
            }
            const uint32_t v = keep ? cc : 0u;
            uint32_t inc = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(FULL, inc, o);
                if (lane >= o) inc += t;
            }
            const uint32_t roundSum = __shfl_sync(FULL, inc, 31);
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
            if constexpr (TO_RESULT) {
                if (a.rout.qcount && keep) {
                    const uint32_t peers = __match_any_sync(kb, qr);
                    if (lane == __ffs(peers) - 1) atomicAdd(&a.rout.qcount[qr], __popc(peers));
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

template <int D, int PRED, bool TO_RESULT>
void launchOne(const ExpandArgs& a, int gridBlocks, cudaStream_t s) {
    auto kern = expandKernel<D, PRED, TO_RESULT>;
    if (gridBlocks <= 0) {
        static int cached = 0;
        if (cached == 0) {
            int dev = 0, sms = 0, perSm = 0;
            TBLAEQ_CUDA(cudaGetDevice(&dev));
            TBLAEQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            TBLAEQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kThreads, 0));
            cached = std::max(1, sms * std::max(1, perSm));
        }
        gridBlocks = cached;
    }
    kern<<<gridBlocks, kThreads, 0, s>>>(a);
    TBLAEQ_CUDA(cudaGetLastError());
}

template <int D>
void dispatchPred(const ExpandArgs& a, int pred, bool toResult, int g, cudaStream_t s) {
    if (toResult) {
        switch (pred) {
            case kPredAll: return launchOne<D, kPredAll, true>(a, g, s);
            case kPredRangeBox: return launchOne<D, kPredRangeBox, true>(a, g, s);
            case kPredMask: return launchOne<D, kPredMask, true>(a, g, s);
            case kPredKnnPoint: return launchOne<D, kPredKnnPoint, true>(a, g, s);
            default: break;
        }
    } else {
        switch (pred) {
            case kPredRangeRadius: return launchOne<D, kPredRangeRadius, false>(a, g, s);
            case kPredMask: return launchOne<D, kPredMask, false>(a, g, s);
            case kPredAll: return launchOne<D, kPredAll, false>(a, g, s);
            case kPredKnnBound: return launchOne<D, kPredKnnBound, false>(a, g, s);
            default: break;
        }
    }
    throw std::invalid_argument("expand: unsupported predicate/output combination");
}

}  // namespace

void launchExpand(const ExpandArgs& a, int pred, bool toResult, int gridBlocks, cudaStream_t stream) {
    switch (a.D) {
        case 2: return dispatchPred<2>(a, pred, toResult, gridBlocks, stream);
        case 3: return dispatchPred<3>(a, pred, toResult, gridBlocks, stream);
        case 4: return dispatchPred<4>(a, pred, toResult, gridBlocks, stream);
        case 5: return dispatchPred<5>(a, pred, toResult, gridBlocks, stream);
        case 8: return dispatchPred<8>(a, pred, toResult, gridBlocks, stream);
        case 16: return dispatchPred<16>(a, pred, toResult, gridBlocks, stream);
        default:
            if (a.D < 1 || a.D > 32) throw std::invalid_argument("expand: D must be in [1, 32]");
            return dispatchPred<0>(a, pred, toResult, gridBlocks, stream);
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
