// Level-synchronous traversal kernels (see traverse.cuh for the design).
#include "traverse.cuh"

#include <cuda/atomic>

#include <algorithm>

namespace tblaeq {

namespace {

constexpr int kWarps = kThreads / 32;
constexpr uint32_t kFlagAggregate = 1;
constexpr uint32_t kFlagPrefix = 2;
constexpr uint32_t kMaxCount30 = (1u << 30) - 1;
constexpr uint32_t kSpinLimit = 1u << 21;  // ~0.2-2 s of polling before giving up

// Items per thread per tile: keep IPT*D doubles of rebuilt coordinates in registers.
template <int D>
struct Ipt {
    static constexpr int value = (D == 0) ? 1 : (D <= 4 ? 4 : (D <= 8 ? 2 : 1));
};

template <int D>
constexpr int tileOf() {
    return kThreads * Ipt<D>::value;
}

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

template <int D, int PRED, bool TO_RESULT>
__global__ void __launch_bounds__(kThreads) expandKernel(ExpandArgs a) {
    constexpr int IPT = Ipt<D>::value;
    constexpr int TILE = kThreads * IPT;
    constexpr int DM = (D > 0) ? D : 32;
    const int dim = (D > 0) ? D : a.D;

    __shared__ uint32_t sTile;
    __shared__ uint32_t sWinBase, sWinLen;
    __shared__ uint32_t sCpre[TILE + 1];
    __shared__ uint32_t sCbeg[TILE + 1];
    __shared__ uint32_t sQ[TILE + 1];
    __shared__ uint32_t sWarpCnt[IPT * kWarps];
    __shared__ uint32_t sWarpSum[IPT * kWarps];
    __shared__ unsigned long long sExCnt, sExSum;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const uint32_t entries = a.in.hdr[0];
    const uint32_t total = a.in.hdr[1];
    const uint32_t nTiles = (total + TILE - 1) / TILE;
    if (entries == 0 || total == 0) return;
    // A producer that overflowed its capacities left this frontier incomplete: never read past
    // the arrays (the host sees the status bit, grows the workspace and reruns the batch).
    if (entries > a.in.cap || nTiles > a.in.tileCap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(a.scratch.status, kStatusOverflowEntries);
        return;
    }

    while (true) {
        if (tid == 0) sTile = atomicAdd(a.scratch.ticket, 1u);
        __syncthreads();
        const uint32_t tile = sTile;
        if (tile >= nTiles) break;
        const uint32_t t0 = tile * TILE;

        // Stage the frontier entries this tile touches.
        if (tid == 0) {
            const uint32_t eLo = a.in.tileStart[tile];
            uint32_t eHi = (tile + 1 < nTiles) ? a.in.tileStart[tile + 1] : entries - 1;
            if (eHi >= entries) eHi = entries - 1;
            uint32_t len = eHi - eLo + 1;
            if (len > TILE + 1) {
                atomicOr(a.scratch.status, kStatusWindowOverflow);
                len = TILE + 1;
            }
            sWinBase = eLo;
            sWinLen = len;
        }
        __syncthreads();
        const uint32_t wb = sWinBase, wl = sWinLen;
        for (uint32_t i = tid; i < wl; i += kThreads) {
            sCpre[i] = a.in.cpre[wb + i];
            sCbeg[i] = a.in.cbeg[wb + i];
            sQ[i] = a.in.q[wb + i];
        }
        __syncthreads();

        // Rebuild and test every item of the tile.
        bool keep[IPT];
        uint32_t row[IPT], qs[IPT], ccnt[IPT], ncb[IPT], key[IPT];
        double y[IPT][DM];
        double d2[IPT];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const uint32_t k = t0 + r * kThreads + tid;
            keep[r] = false;
            ccnt[r] = 0;
            ncb[r] = 0;
            d2[r] = 0.0;
            row[r] = 0;
            qs[r] = 0;
            key[r] = 0;
            if (k < total) {
                uint32_t lo = 0, hi = wl - 1;
                while (lo < hi) {  // last entry whose prefix <= k
                    const uint32_t mid = (lo + hi + 1) >> 1;
                    if (sCpre[mid] <= k) lo = mid; else hi = mid - 1;
                }
                const uint32_t e = lo;
                const uint32_t j = sCbeg[e] + (k - sCpre[e]);
                const uint32_t qi = sQ[e];
                row[r] = j;
                qs[r] = qi;
                const double* xp = a.in.x + static_cast<size_t>(wb + e) * dim;
                const double* rp = a.child.rows + static_cast<size_t>(j) * dim;
                if constexpr (D > 0 && (D % 2) == 0) {
#pragma unroll
                    for (int d = 0; d < D; d += 2) {
                        const double2 pv = __ldg(reinterpret_cast<const double2*>(rp + d));
                        const double2 xv = __ldg(reinterpret_cast<const double2*>(xp + d));
                        y[r][d] = __dmul_rn(pv.x, xv.x);
                        y[r][d + 1] = __dmul_rn(pv.y, xv.y);
                    }
                } else {
#pragma unroll
                    for (int d = 0; d < DM; ++d) {
                        if (d < dim) y[r][d] = __dmul_rn(__ldg(rp + d), __ldg(xp + d));
                    }
                }
                const uint32_t kk = a.child.keys ? static_cast<uint32_t>(a.child.keys[j]) : j;
                key[r] = kk;
                if constexpr (PRED == kPredRangeRadius) {
                    const double* box = a.query.boxes + static_cast<size_t>(qi) * 2 * dim;
                    const double dist = boxDist2<DM>(y[r], box, box + dim, dim, a.useFma);
                    const double rr = a.child.rad[kk];
                    ccnt[r] = a.child.ncnt[kk];
                    keep[r] = (ccnt[r] > 0) && (dist <= __dmul_rn(rr, rr));
                } else if constexpr (PRED == kPredMask) {
                    keep[r] = a.child.mask[j] != 0;
                    if constexpr (!TO_RESULT) {
                        ccnt[r] = a.child.ncnt[kk];
                        keep[r] = keep[r] && ccnt[r] > 0;
                    }
                } else if constexpr (PRED == kPredAll) {
                    keep[r] = true;
                    if constexpr (!TO_RESULT) {
                        ccnt[r] = a.child.ncnt[kk];
                        keep[r] = ccnt[r] > 0;
                    }
                } else if constexpr (PRED == kPredRangeBox) {
                    const double* box = a.query.boxes + static_cast<size_t>(qi) * 2 * dim;
                    bool in = true;
#pragma unroll
                    for (int d = 0; d < DM; ++d) {
                        if (d < dim) in = in && (box[d] <= y[r][d]) && (y[r][d] <= box[dim + d]);
                    }
                    keep[r] = in;
                } else if constexpr (PRED == kPredKnnBound) {
                    const double* p = a.query.points + static_cast<size_t>(qi) * dim;
                    const double dd = sqrt(pointDist2<DM>(y[r], p, dim, 1));
                    ccnt[r] = a.child.ncnt[kk];
                    keep[r] = (ccnt[r] > 0) && (dd - a.child.rad[kk] <= a.query.tau[qi]);
                } else if constexpr (PRED == kPredKnnPoint) {
                    const double* p = a.query.points + static_cast<size_t>(qi) * dim;
                    d2[r] = pointDist2<DM>(y[r], p, dim, 1);
                    const double t = a.query.tau[qi];
                    keep[r] = d2[r] <= t * t;
                }
                if constexpr (!TO_RESULT) {
                    if (keep[r]) ncb[r] = a.child.ncbeg[kk];
                }
            }
            // Per-query generated-children counts (the reference's levelFineMeshSize).
            if (a.scratch.levelItems) {
                const bool valid = k < total;
                const uint32_t vm = __ballot_sync(0xffffffffu, valid);
                if (valid) {
                    const uint32_t peers = __match_any_sync(vm, qs[r]);
                    if (lane == __ffs(peers) - 1) atomicAdd(&a.scratch.levelItems[qs[r]], __popc(peers));
                }
            }
        }

        // Tile-local order-preserving ranks: round-major, then thread order.
        uint32_t rankCnt[IPT], rankSum[IPT];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const uint32_t ballot = __ballot_sync(0xffffffffu, keep[r]);
            rankCnt[r] = __popc(ballot & ((1u << lane) - 1));
            uint32_t s = keep[r] ? ccnt[r] : 0;
            uint32_t inc = s;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += v;
            }
            rankSum[r] = inc - s;
            if (lane == 31) {
                sWarpCnt[r * kWarps + warp] = __popc(ballot);
                sWarpSum[r * kWarps + warp] = inc;
            }
        }
        __syncthreads();
        if (warp == 0) {
            // Exclusive scan of the IPT*kWarps warp totals (<= 32 of them) in round-major order.
            constexpr int NW = IPT * kWarps;
            const uint32_t c = (lane < NW) ? sWarpCnt[lane] : 0;
            const uint32_t s = (lane < NW) ? sWarpSum[lane] : 0;
            uint32_t ic = c, is = s;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t vc = __shfl_up_sync(0xffffffffu, ic, o);
                const uint32_t vs = __shfl_up_sync(0xffffffffu, is, o);
                if (lane >= o) {
                    ic += vc;
                    is += vs;
                }
            }
            const uint32_t aggCnt = __shfl_sync(0xffffffffu, ic, 31);
            const uint32_t aggSum = __shfl_sync(0xffffffffu, is, 31);
            if (lane < NW) {
                sWarpCnt[lane] = ic - c;
                sWarpSum[lane] = is - s;
            }
            unsigned long long exC, exS;
            lookback(a.scratch.desc, tile, aggCnt, aggSum, a.scratch.status, exC, exS);
            if (lane == 0) {
                sExCnt = exC;
                sExSum = exS;
                if (tile == nTiles - 1) {
                    const unsigned long long totC = exC + aggCnt;
                    const unsigned long long totS = exS + aggSum;
                    if constexpr (TO_RESULT) {
                        a.rout.hdr[0] = static_cast<uint32_t>(min(totC, 0xffffffffull));
                        if (totC > a.rout.cap) atomicOr(a.scratch.status, kStatusOverflowEntries);
                    } else {
                        a.fout.hdr[0] = static_cast<uint32_t>(min(totC, 0xffffffffull));
                        a.fout.hdr[1] = static_cast<uint32_t>(min(totS, 0xffffffffull));
                        if (totC > a.fout.cap) atomicOr(a.scratch.status, kStatusOverflowEntries);
                        if (totS > 0xffffffffull) atomicOr(a.scratch.status, kStatusOverflowSum);
                        const unsigned long long tilesNeeded = (totS + TILE - 1) / TILE;
                        if (tilesNeeded > a.fout.tileCap) atomicOr(a.scratch.status, kStatusOverflowItems);
                    }
                }
            }
        }
        __syncthreads();
        const unsigned long long exCnt = sExCnt, exSum = sExSum;

        // Write kept items.
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            if (!keep[r]) continue;
            const unsigned long long pos = exCnt + sWarpCnt[r * kWarps + warp] + rankCnt[r];
            if constexpr (TO_RESULT) {
                if (pos >= a.rout.cap) continue;
                const uint32_t j = row[r];
                a.rout.ids[pos] = a.child.outMap ? a.child.outMap[j] : static_cast<uint64_t>(key[r]);
                if (a.rout.vals) {
#pragma unroll
                    for (int d = 0; d < DM; ++d)
                        if (d < dim) a.rout.vals[pos * dim + d] = y[r][d];
                }
                if (a.rout.q) a.rout.q[pos] = qs[r];
                if (a.rout.dist2) a.rout.dist2[pos] = d2[r];
            } else {
                if (pos >= a.fout.cap) continue;
                const unsigned long long cp = exSum + sWarpSum[r * kWarps + warp] + rankSum[r];
                a.fout.q[pos] = qs[r];
                a.fout.node[pos] = key[r];
                a.fout.cbeg[pos] = ncb[r];
                a.fout.cpre[pos] = static_cast<uint32_t>(cp);
#pragma unroll
                for (int d = 0; d < DM; ++d)
                    if (d < dim) a.fout.x[pos * dim + d] = y[r][d];
                // Tile starts of the next level: every tile boundary inside this entry's children.
                const unsigned long long cend = cp + ccnt[r];
                for (unsigned long long b = (cp + TILE - 1) / TILE; b * TILE < cend; ++b) {
                    if (b < a.fout.tileCap) a.fout.tileStart[b] = static_cast<uint32_t>(pos);
                }
            }
        }
        if constexpr (TO_RESULT) {
            if (a.rout.qcount) {
#pragma unroll
                for (int r = 0; r < IPT; ++r) {
                    const uint32_t km = __ballot_sync(0xffffffffu, keep[r]);
                    if (keep[r]) {
                        const uint32_t peers = __match_any_sync(km, qs[r]);
                        if (lane == __ffs(peers) - 1) atomicAdd(&a.rout.qcount[qs[r]], __popc(peers));
                    }
                }
            }
        }
        __syncthreads();  // shared staging is reused by the next tile
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

int expandTile(int D) {
    switch (D) {
        case 2: return tileOf<2>();
        case 3: return tileOf<3>();
        case 4: return tileOf<4>();
        case 5: return tileOf<5>();
        case 8: return tileOf<8>();
        case 16: return tileOf<16>();
        default: return tileOf<0>();
    }
}

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
