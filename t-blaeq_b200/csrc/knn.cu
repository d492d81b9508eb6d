// KNN building blocks (see knn.cuh).
#include "knn.cuh"

#include <algorithm>
#include <cfloat>

namespace tblaeq {

namespace {

constexpr int kSortTile = 2048;  // pairs per bitonic tile (1024 threads x 2)
constexpr int kMergeItems = 8;   // outputs per thread in a merge pass

__device__ __forceinline__ bool pairLess(uint64_t ka, uint32_t va, uint64_t kb, uint32_t vb) {
    return ka < kb || (ka == kb && va < vb);
}

__global__ void knnLowerBoundKernel(const uint64_t* ids, const double* vals, uint64_t p, int D, const double* q,
                                    const NodeRec* nodes, uint64_t* keys, uint32_t* labels, uint32_t* cnt,
                                    double* rr) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < p;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        double dist = 0.0;
        for (int d = 0; d < D; ++d) {
            const double diff = q[d] - vals[i * D + d];
            dist = __fma_rn(diff, diff, dist);  // the reference kernel's contracted accumulation
        }
        const NodeRec nr = nodes[ids[i]];
        const double lb = __dsqrt_rd(dist) - nr.rad;
        keys[i] = orderKey(lb);
        labels[i] = static_cast<uint32_t>(i);
        cnt[i] = nr.cnt;
        rr[i] = lb + 2.0 * nr.rad;
    }
}

// Sorts one 2048-pair tile in shared memory (bitonic network), padding with +inf keys.
__global__ void __launch_bounds__(1024) bitonicTileKernel(uint64_t* keys, uint32_t* labels, uint64_t n) {
    __shared__ uint64_t sk[kSortTile];
    __shared__ uint32_t sv[kSortTile];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kSortTile;
    for (int i = threadIdx.x; i < kSortTile; i += blockDim.x) {
        const uint64_t g = base + i;
        sk[i] = g < n ? keys[g] : ~0ull;
        sv[i] = g < n ? labels[g] : 0xffffffffu;
    }
    __syncthreads();
    for (int size = 2; size <= kSortTile; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < kSortTile / 2; t += blockDim.x) {
                const int lo = 2 * t - (t & (stride - 1));
                const int hi = lo + stride;
                const bool asc = ((lo & size) == 0);
                const bool swap = asc ? pairLess(sk[hi], sv[hi], sk[lo], sv[lo]) : pairLess(sk[lo], sv[lo], sk[hi], sv[hi]);
                if (swap) {
                    const uint64_t k = sk[lo];
                    sk[lo] = sk[hi];
                    sk[hi] = k;
                    const uint32_t v = sv[lo];
                    sv[lo] = sv[hi];
                    sv[hi] = v;
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < kSortTile; i += blockDim.x) {
        const uint64_t g = base + i;
        if (g < n) {
            keys[g] = sk[i];
            labels[g] = sv[i];
        }
    }
}

// One merge pass: sorted runs of `width` pairs are merged pairwise into runs of 2 * width. Each
// thread finds its start on the merge path by a binary search and merges kMergeItems outputs.
__global__ void mergePassKernel(const uint64_t* ki, const uint32_t* vi, uint64_t* ko, uint32_t* vo, uint64_t n,
                                uint64_t width) {
    const uint64_t nOut = (n + kMergeItems - 1) / kMergeItems;
    for (uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; t < nOut;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t o0 = t * kMergeItems;
        const uint64_t pairStart = (o0 / (2 * width)) * (2 * width);
        const uint64_t aBeg = pairStart, aEnd = std::min(pairStart + width, n);
        const uint64_t bBeg = aEnd, bEnd = std::min(pairStart + 2 * width, n);
        const uint64_t aLen = aEnd - aBeg, bLen = bEnd - bBeg;
        const uint64_t diag = o0 - pairStart;  // outputs of this pair before o0
        // Largest i in [max(0, diag - bLen), min(diag, aLen)] with A[i-1] <= B[diag-i] (stable: A first).
        uint64_t lo = diag > bLen ? diag - bLen : 0, hi = std::min(diag, aLen);
        while (lo < hi) {
            const uint64_t i = (lo + hi + 1) >> 1;  // candidate count taken from A
            const uint64_t j = diag - i;
            // Taking i from A is valid iff A[i-1] <= B[j] (ties go to A).
            if (!pairLess(ki[bBeg + j], vi[bBeg + j], ki[aBeg + i - 1], vi[aBeg + i - 1])) lo = i; else hi = i - 1;
        }
        uint64_t ia = aBeg + lo, ib = bBeg + (diag - lo);
        for (int r = 0; r < kMergeItems && o0 + r < n && o0 + r < pairStart + aLen + bLen; ++r) {
            bool takeA;
            if (ia >= aEnd) takeA = false;
            else if (ib >= bEnd) takeA = true;
            else takeA = !pairLess(ki[ib], vi[ib], ki[ia], vi[ia]);
            if (takeA) {
                ko[o0 + r] = ki[ia];
                vo[o0 + r] = vi[ia];
                ++ia;
            } else {
                ko[o0 + r] = ki[ib];
                vo[o0 + r] = vi[ib];
                ++ib;
            }
        }
    }
}

// STEP in one CTA: n1 = entries whose preceding child count is below K (the part that feeds the
// running bound), cur = max(0, max rr over them), then every later entry with lb <= cur.
__global__ void __launch_bounds__(1024) stepKernel(const uint64_t* keys, const uint32_t* labels, const uint32_t* cnt,
                                                   const double* rr, uint64_t n, uint64_t K, uint8_t* mask) {
    __shared__ unsigned long long sCarry;
    __shared__ unsigned long long sFirst;
    __shared__ unsigned long long sWarp[32];
    __shared__ double sMax[32];
    __shared__ unsigned long long sEnd;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x / 32;
    if (tid == 0) {
        sCarry = 0;
        sFirst = ~0ull;
    }
    __syncthreads();
    // First index whose inclusive child-count prefix reaches K.
    if (K > 0) {
        for (uint64_t base = 0; base < n; base += blockDim.x) {
            const uint64_t i = base + tid;
            const unsigned long long c = i < n ? cnt[labels[i]] : 0;
            unsigned long long inc = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += t;
            }
            if (lane == 31) sWarp[warp] = inc;
            __syncthreads();
            if (warp == 0) {
                unsigned long long w = lane < nw ? sWarp[lane] : 0, wi = w;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned long long t = __shfl_up_sync(0xffffffffu, wi, o);
                    if (lane >= o) wi += t;
                }
                if (lane < nw) sWarp[lane] = wi - w;
            }
            __syncthreads();
            const unsigned long long carry = sCarry;
            const unsigned long long total = carry + sWarp[warp] + inc;
            if (i < n && total >= K) atomicMin(&sFirst, static_cast<unsigned long long>(i));
            __syncthreads();
            if (tid == blockDim.x - 1) sCarry = carry + sWarp[warp] + inc;
            __syncthreads();
            if (sFirst != ~0ull) break;
        }
    }
    __syncthreads();
    const uint64_t n1 = (K == 0) ? 0 : (sFirst == ~0ull ? n : sFirst + 1);
    // cur = max(0, max rr over the first n1 entries).
    double m = 0.0;
    for (uint64_t i = tid; i < n1; i += blockDim.x) m = fmax(m, rr[labels[i]]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) sMax[warp] = m;
    __syncthreads();
    if (tid == 0) {
        double cur = 0.0;
        for (int w = 0; w < nw; ++w) cur = fmax(cur, sMax[w]);
        // Entries after n1 are taken while lb <= cur; keys are sorted, so find the first key above.
        const uint64_t kc = orderKey(cur);
        uint64_t lo = n1, hi = n;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (keys[mid] > kc) hi = mid; else lo = mid + 1;
        }
        sEnd = (n1 >= n) ? n : lo;
    }
    __syncthreads();
    const uint64_t end = sEnd;
    for (uint64_t i = tid; i < end; i += blockDim.x) mask[labels[i]] = 1;
}

constexpr int kTopKStage = 4096;  // candidates a CTA sorts in shared memory

__global__ void __launch_bounds__(512) topKKernel(const uint64_t* offA, const uint64_t* idsA, const double* d2A,
                                                  uint64_t capA, const uint64_t* offB, const uint64_t* idsB,
                                                  const double* d2B, uint64_t capB, const uint32_t* Kq,
                                                  const uint64_t* outOff, uint64_t* outIds, double* outD2,
                                                  uint32_t* outCount, uint32_t* status) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* sk = reinterpret_cast<uint64_t*>(smem);
    uint64_t* sv = sk + kTopKStage;
    const uint32_t q = blockIdx.x;
    const uint64_t a0 = offA[q], na = offA[q + 1] - a0;
    const uint64_t b0 = offB ? offB[q] : 0, nb = offB ? offB[q + 1] - b0 : 0;
    const uint64_t n = na + nb;
    const uint32_t K = Kq[q];
    // Candidates beyond the arrays mean the producer overflowed: never read them.
    if (a0 + na > capA || (offB && b0 + nb > capB)) {
        if (threadIdx.x == 0) {
            outCount[q] = 0;
            atomicOr(status, kStatusOverflowEntries);
        }
        return;
    }
    const uint64_t keep = std::min<uint64_t>(K, n);
    auto keyAt = [&](uint64_t i) -> uint64_t { return i < na ? orderKey(d2A[a0 + i]) : orderKey(d2B[b0 + i - na]); };
    auto idAt = [&](uint64_t i) -> uint64_t {
        if (i < na) return idsA ? idsA[a0 + i] : a0 + i;  // no id array: the candidate's position
        return idsB ? idsB[b0 + i - na] : b0 + i - na;
    };
    if (threadIdx.x == 0) outCount[q] = static_cast<uint32_t>(keep);
    if (keep == 0) return;
    const uint64_t o = outOff[q];
    // Sorts sk/sv[0, count) by (key, id) with a bitonic network and writes the first `keep`.
    auto sortAndWrite = [&](uint32_t count) {
        int size = 1;
        while (size < static_cast<int>(count)) size <<= 1;
        for (int i = static_cast<int>(count) + threadIdx.x; i < size; i += blockDim.x) {
            sk[i] = ~0ull;
            sv[i] = ~0ull;
        }
        __syncthreads();
        for (int s = 2; s <= size; s <<= 1) {
            for (int stride = s >> 1; stride > 0; stride >>= 1) {
                for (int t = threadIdx.x; t < size / 2; t += blockDim.x) {
                    const int lo = 2 * t - (t & (stride - 1));
                    const int hi = lo + stride;
                    const bool asc = ((lo & s) == 0);
                    const bool gt = sk[lo] > sk[hi] || (sk[lo] == sk[hi] && sv[lo] > sv[hi]);
                    if (asc == gt) {
                        const uint64_t k = sk[lo];
                        sk[lo] = sk[hi];
                        sk[hi] = k;
                        const uint64_t v = sv[lo];
                        sv[lo] = sv[hi];
                        sv[hi] = v;
                    }
                }
                __syncthreads();
            }
        }
        for (uint64_t i = threadIdx.x; i < keep; i += blockDim.x) {
            outIds[o + i] = sv[i];
            uint64_t b = sk[i];
            b = (b & 0x8000000000000000ull) ? (b & 0x7fffffffffffffffull) : ~b;
            double d;
            memcpy(&d, &b, 8);
            outD2[o + i] = d;
        }
    };
    if (n <= kTopKStage) {
        for (int i = threadIdx.x; i < static_cast<int>(n); i += blockDim.x) {
            sk[i] = keyAt(i);
            sv[i] = idAt(i);
        }
        sortAndWrite(static_cast<uint32_t>(n));
        return;
    }
    if (keep <= kTopKStage) {
        // Radix selection of the keep-th smallest key: eight passes over the candidates, each a
        // 256-bin histogram of the next 8-bit digit among the keys that share the digits chosen
        // so far. Then every key below the boundary and the ties on it are gathered and sorted.
        __shared__ uint32_t hist[256];
        __shared__ unsigned long long sPrefix, sMask;
        __shared__ uint32_t sNeed, sLess, sEq;
        if (threadIdx.x == 0) {
            sPrefix = 0;
            sMask = 0;
            sNeed = static_cast<uint32_t>(keep);
        }
        __syncthreads();
        for (int shift = 56; shift >= 0; shift -= 8) {
            for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
            __syncthreads();
            const uint64_t prefix = sPrefix, mask = sMask;
            for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
                const uint64_t key = keyAt(i);
                if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                uint32_t need = sNeed, cum = 0, d = 0;
                while (d < 255u && cum + hist[d] < need) cum += hist[d++];
                sNeed = need - cum;
                sPrefix = prefix | (static_cast<unsigned long long>(d) << shift);
                sMask = mask | (255ull << shift);
            }
            __syncthreads();
        }
        const uint64_t kb = sPrefix;
        const uint32_t less = static_cast<uint32_t>(keep) - sNeed;
        const uint32_t room = static_cast<uint32_t>(kTopKStage) - less;
        if (threadIdx.x == 0) {
            sLess = 0;
            sEq = 0;
        }
        __syncthreads();
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t key = keyAt(i);
            if (key < kb) {
                const uint32_t slot = atomicAdd(&sLess, 1u);
                if (slot < less) {
                    sk[slot] = key;
                    sv[slot] = idAt(i);
                }
            } else if (key == kb) {
                const uint32_t slot = atomicAdd(&sEq, 1u);
                if (slot < room) {
                    sk[less + slot] = key;
                    sv[less + slot] = idAt(i);
                }
            }
        }
        __syncthreads();
        if (sLess == less && sEq <= room) {
            sortAndWrite(less + sEq);
            return;
        }
        __syncthreads();
        // (ties on the boundary key overflow the stage: fall back to the rounds below)
    }
    // More candidates than the stage holds: K rounds of a block-wide minimum above the last pick.
    __shared__ unsigned long long sBestK, sBestV;
    uint64_t lastK = 0, lastV = 0;
    bool haveLast = false;
    for (uint64_t r = 0; r < keep; ++r) {
        if (threadIdx.x == 0) {
            sBestK = ~0ull;
            sBestV = ~0ull;
        }
        __syncthreads();
        uint64_t bk = ~0ull, bv = ~0ull;
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t k = keyAt(i), v = idAt(i);
            const bool above = !haveLast || k > lastK || (k == lastK && v > lastV);
            if (above && (k < bk || (k == bk && v < bv))) {
                bk = k;
                bv = v;
            }
        }
        // (key, id) minimum: first the key, then the id among equal keys.
        atomicMin(&sBestK, static_cast<unsigned long long>(bk));
        __syncthreads();
        if (bk == sBestK) atomicMin(&sBestV, static_cast<unsigned long long>(bv));
        __syncthreads();
        lastK = sBestK;
        lastV = sBestV;
        haveLast = true;
        if (threadIdx.x == 0) {
            outIds[o + r] = lastV;
            uint64_t b = lastK;
            b = (b & 0x8000000000000000ull) ? (b & 0x7fffffffffffffffull) : ~b;
            double d;
            memcpy(&d, &b, 8);
            outD2[o + r] = d;
        }
        __syncthreads();
    }
}

__global__ void fillDoubleKernel(double* v, double value, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = value;
}

__global__ void clampCountsKernel(const uint64_t* off, const uint32_t* K, uint32_t nq, uint32_t* out) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        const uint64_t n = off[q + 1] - off[q];
        out[q] = static_cast<uint32_t>(n < K[q] ? n : K[q]);
    }
}

// Lower bound of the distance from each frontier entry's query point to the points below its
// cluster: the larger of (centre distance - subtree radius) and the distance to the cluster's box.
// D > 0 specialises the dimension loop (pairs of dimensions per 16-byte load when D is even); the
// products are accumulated in the same order either way, so the bounds are identical.
template <int D>
__global__ void entryBoundsKernel(const uint32_t* q, const uint32_t* node, const double* x, const uint32_t* hdr,
                                  uint32_t cap, int dimRt, const double* points, const NodeRec* nodes,
                                  const float* aabb, double* lb, double* score) {
    const int dim = D > 0 ? D : dimRt;
    const uint32_t n = min(hdr[0], cap);
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const double* p = points + static_cast<size_t>(q[e]) * dim;
        const double* c = x + static_cast<size_t>(e) * dim;
        const uint32_t k = node[e];
        const float* b = aabb + static_cast<size_t>(k) * 2 * dim;
        double dist = 0.0, gap = 0.0;
        auto step = [&](double pd, double cd, float lo, float hi) {
            const double diff = pd - cd;
            dist = __fma_rn(diff, diff, dist);
            const double l = static_cast<double>(lo), h = static_cast<double>(hi);
            const double g = fmax(fmax(l - pd, pd - h), 0.0);
            gap = __fma_rn(g, g, gap);
        };
        if constexpr (D > 0 && D % 2 == 0) {
#pragma unroll
            for (int d = 0; d < D; d += 2) {
                const double2 pp = __ldg(reinterpret_cast<const double2*>(p + d));
                const double2 cc = __ldg(reinterpret_cast<const double2*>(c + d));
                const float2 lo = __ldg(reinterpret_cast<const float2*>(b + d));
                const float2 hi = __ldg(reinterpret_cast<const float2*>(b + D + d));
                step(pp.x, cc.x, lo.x, hi.x);
                step(pp.y, cc.y, lo.y, hi.y);
            }
        } else {
            for (int d = 0; d < dim; ++d) step(p[d], c[d], b[d], b[dim + d]);
        }
        const double v = fmax(sqrt(dist) - nodes[k].rad, sqrt(gap) * (1.0 - 1e-12));
        lb[e] = v;
        score[e] = v;
    }
}

__global__ void waveWidthKernel(const uint32_t* K, uint32_t nq, double factor, uint32_t* M) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) {
        const double m = ceil(factor * static_cast<double>(K[i])) + 1.0;
        M[i] = static_cast<uint32_t>(fmin(32.0, fmax(2.0, m)));
    }
}

// The selection offsets are counted before the selection top-K runs; a query the top-K had to
// skip (its frontier overflowed: the batch is rerun after growth) leaves its slots unwritten, so
// every id is checked against the entry capacity before it is used as an index.
__global__ void scatterSelKernel(const uint64_t* ids, const uint64_t* off, uint32_t nq, uint64_t cap, uint8_t* sel) {
    const uint64_t n = off[nq];
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t e = ids[i];
        if (e < cap) sel[e] = 1;
    }
}

__global__ void tauFromTopKKernel(const uint64_t* off, const double* d2, const uint32_t* K, uint32_t nq, double* tau) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        const uint64_t n = off[q + 1] - off[q];
        if (K[q] > 0 && n == K[q]) {
            const double t = sqrt(d2[off[q + 1] - 1]) * (1.0 + 1e-12);
            if (t < tau[q]) tau[q] = t;
        }
    }
}

__global__ void clampCounts2Kernel(const uint64_t* offA, const uint64_t* offB, const uint32_t* K, uint32_t nq,
                                   uint32_t* out) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        const uint64_t n = (offA[q + 1] - offA[q]) + (offB[q + 1] - offB[q]);
        out[q] = static_cast<uint32_t>(n < K[q] ? n : K[q]);
    }
}

int gridFor(uint64_t n, int threads) {
    const uint64_t b = (n + threads - 1) / threads;
    return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(b, 148ull * 16)));
}

}  // namespace

void launchEntryBounds(const uint32_t* q, const uint32_t* node, const double* x, const uint32_t* hdr, uint32_t cap,
                       int D, const double* points, const NodeRec* nodes, const float* aabb, double* lb, double* score,
                       cudaStream_t s) {
    auto go = [&](auto kern) { kern<<<148 * 8, 256, 0, s>>>(q, node, x, hdr, cap, D, points, nodes, aabb, lb, score); };
    switch (D) {
        case 2: go(entryBoundsKernel<2>); break;
        case 3: go(entryBoundsKernel<3>); break;
        case 4: go(entryBoundsKernel<4>); break;
        case 5: go(entryBoundsKernel<5>); break;
        case 8: go(entryBoundsKernel<8>); break;
        case 16: go(entryBoundsKernel<16>); break;
        default: go(entryBoundsKernel<0>); break;
    }
    TBLAEQ_LAUNCHED();
}

void launchWaveWidth(const uint32_t* K, uint32_t nq, double factor, uint32_t* M, cudaStream_t s) {
    if (nq == 0) return;
    waveWidthKernel<<<gridFor(nq, 256), 256, 0, s>>>(K, nq, factor, M);
    TBLAEQ_LAUNCHED();
}

void launchScatterSel(const uint64_t* ids, const uint64_t* off, uint32_t nq, uint64_t cap, uint8_t* sel,
                      cudaStream_t s) {
    scatterSelKernel<<<148 * 4, 256, 0, s>>>(ids, off, nq, cap, sel);
    TBLAEQ_LAUNCHED();
}

void launchTauFromTopK(const uint64_t* off, const double* d2, const uint32_t* K, uint32_t nq, double* tau,
                       cudaStream_t s) {
    if (nq == 0) return;
    tauFromTopKKernel<<<gridFor(nq, 256), 256, 0, s>>>(off, d2, K, nq, tau);
    TBLAEQ_LAUNCHED();
}

void launchClampCounts2(const uint64_t* offA, const uint64_t* offB, const uint32_t* K, uint32_t nq, uint32_t* out,
                        cudaStream_t s) {
    if (nq == 0) return;
    clampCounts2Kernel<<<gridFor(nq, 256), 256, 0, s>>>(offA, offB, K, nq, out);
    TBLAEQ_LAUNCHED();
}

void launchFillDouble(double* v, double value, uint32_t n, cudaStream_t s) {
    if (n == 0) return;
    fillDoubleKernel<<<gridFor(n, 256), 256, 0, s>>>(v, value, n);
    TBLAEQ_LAUNCHED();
}

void launchClampCounts(const uint64_t* off, const uint32_t* K, uint32_t nq, uint32_t* out, cudaStream_t s) {
    if (nq == 0) return;
    clampCountsKernel<<<gridFor(nq, 256), 256, 0, s>>>(off, K, nq, out);
    TBLAEQ_LAUNCHED();
}

void launchKnnLowerBound(const uint64_t* ids, const double* vals, uint64_t p, int D, const double* dPoint,
                         const NodeRec* nodes, uint64_t* keys, uint32_t* labels, uint32_t* cnt, double* rr,
                         cudaStream_t s) {
    if (p == 0) return;
    knnLowerBoundKernel<<<gridFor(p, 256), 256, 0, s>>>(ids, vals, p, D, dPoint, nodes, keys, labels, cnt, rr);
    TBLAEQ_LAUNCHED();
}

void sortPairs(uint64_t* keys, uint32_t* labels, uint64_t* keys2, uint32_t* labels2, uint64_t n, cudaStream_t s) {
    if (n <= 1) return;
    const uint64_t tiles = (n + kSortTile - 1) / kSortTile;
    bitonicTileKernel<<<static_cast<unsigned>(tiles), 1024, 0, s>>>(keys, labels, n);
    TBLAEQ_LAUNCHED();
    uint64_t* ka = keys;
    uint32_t* va = labels;
    uint64_t* kb = keys2;
    uint32_t* vb = labels2;
    for (uint64_t w = kSortTile; w < n; w *= 2) {
        mergePassKernel<<<gridFor((n + kMergeItems - 1) / kMergeItems, 256), 256, 0, s>>>(ka, va, kb, vb, n, w);
        TBLAEQ_LAUNCHED();
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    if (ka != keys) {
        TBLAEQ_CUDA(cudaMemcpyAsync(keys, ka, n * 8, cudaMemcpyDeviceToDevice, s));
        TBLAEQ_CUDA(cudaMemcpyAsync(labels, va, n * 4, cudaMemcpyDeviceToDevice, s));
    }
}

void launchStep(const uint64_t* keys, const uint32_t* labels, const uint32_t* cnt, const double* rr, uint64_t n,
                uint64_t K, uint8_t* mask, cudaStream_t s) {
    if (n == 0) return;
    stepKernel<<<1, 1024, 0, s>>>(keys, labels, cnt, rr, n, K, mask);
    TBLAEQ_LAUNCHED();
}

void launchTopK(const uint64_t* offA, const uint64_t* idsA, const double* d2A, uint64_t capA, const uint64_t* offB,
                const uint64_t* idsB, const double* d2B, uint64_t capB, const uint32_t* K, uint32_t nq,
                const uint64_t* outOff, uint64_t* outIds, double* outD2, uint32_t* outCount, uint32_t* status,
                cudaStream_t s) {
    if (nq == 0) return;
    const size_t smem = static_cast<size_t>(kTopKStage) * 16;
    static bool attr = false;
    if (!attr) {
        TBLAEQ_CUDA(cudaFuncSetAttribute(topKKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem)));
        attr = true;
    }
    topKKernel<<<nq, 512, smem, s>>>(offA, idsA, d2A, capA, offB, idsB, d2B, capB, K, outOff, outIds, outD2, outCount,
                                     status);
    TBLAEQ_LAUNCHED();
}

// ---- frontier compaction for the two finest-level waves ------------------------------------------
namespace {

constexpr int kCompactThreads = 256;

__device__ __forceinline__ bool keepEntry(int mode, uint64_t e, uint32_t q, const uint8_t* sel, const double* lb,
                                          const double* tau) {
    return mode == 1 ? sel[e] != 0 : (sel[e] == 0 && lb[e] <= tau[q]);
}

__device__ __forceinline__ uint32_t childrenOf(const FrontierIn& F, uint64_t e, uint32_t entries) {
    const uint32_t end = (e + 1 < entries) ? F.cpre[e + 1] : F.hdr[1];
    return end - F.cpre[e];
}

// A frontier whose producer overflowed its capacity is incomplete (the batch is rerun after the
// workspace grows): it compacts to nothing rather than to entries with inconsistent prefixes.
__device__ __forceinline__ uint32_t usableEntries(const FrontierIn& F) { return F.hdr[0] <= F.cap ? F.hdr[0] : 0u; }

constexpr uint32_t kSegment = 4096;  // frontier entries per compaction block

// Pass 1, one block per segment of the (query-major) frontier: kept entries and their children.
__global__ void __launch_bounds__(kCompactThreads) compactCountKernel(FrontierIn F, int mode, const uint8_t* sel,
                                                                     const double* lb, const double* tau,
                                                                     uint32_t* cnt, uint32_t* kids) {
    __shared__ uint32_t sC[kCompactThreads / 32], sK[kCompactThreads / 32];
    const uint32_t entries = usableEntries(F);
    const uint64_t e0 = static_cast<uint64_t>(blockIdx.x) * kSegment;
    const uint64_t e1 = min(e0 + kSegment, static_cast<uint64_t>(entries));
    uint32_t c = 0, k = 0;
    for (uint64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        if (keepEntry(mode, e, F.q[e], sel, lb, tau)) {
            ++c;
            k += childrenOf(F, e, entries);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_xor_sync(0xffffffffu, c, o);
        k += __shfl_xor_sync(0xffffffffu, k, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sC[threadIdx.x >> 5] = c;
        sK[threadIdx.x >> 5] = k;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tc = 0, tk = 0;
        for (int w = 0; w < kCompactThreads / 32; ++w) {
            tc += sC[w];
            tk += sK[w];
        }
        cnt[blockIdx.x] = tc;
        kids[blockIdx.x] = tk;
    }
}

// Pass 2, one block per segment: writes the kept entries in order, with their child prefix and
// the tile starts of the compacted item space (as the expand producer would have).
__global__ void __launch_bounds__(kCompactThreads) compactWriteKernel(FrontierIn F, int mode, const uint8_t* sel,
                                                                     const double* lb, const double* tau,
                                                                     const uint64_t* entryOff, const uint64_t* kidOff,
                                                                     int D, FrontierOut out) {
    __shared__ uint32_t sCnt[kCompactThreads / 32], sKid[kCompactThreads / 32];
    __shared__ uint32_t sRunC, sRunK;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t entries = usableEntries(F);
    const uint64_t e0 = static_cast<uint64_t>(blockIdx.x) * kSegment;
    const uint64_t e1 = min(e0 + kSegment, static_cast<uint64_t>(entries));
    if (threadIdx.x == 0) {
        sRunC = 0;
        sRunK = 0;
    }
    __syncthreads();
    for (uint64_t base = e0; base < e1; base += blockDim.x) {
        const uint64_t e = base + threadIdx.x;
        const uint32_t q = e < e1 ? F.q[e] : 0u;
        const bool keep = e < e1 && keepEntry(mode, e, q, sel, lb, tau);
        const uint32_t kc = keep ? childrenOf(F, e, entries) : 0u;
        uint32_t c = keep ? 1u : 0u, k = kc;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t tc = __shfl_up_sync(0xffffffffu, c, o), tk = __shfl_up_sync(0xffffffffu, k, o);
            if (lane >= o) {
                c += tc;
                k += tk;
            }
        }
        if (lane == 31) {
            sCnt[warp] = c;
            sKid[warp] = k;
        }
        __syncthreads();
        uint32_t wc = 0, wk = 0;
        for (int w = 0; w < warp; ++w) {
            wc += sCnt[w];
            wk += sKid[w];
        }
        if (keep) {
            const uint64_t pos = entryOff[blockIdx.x] + sRunC + wc + c - 1u;
            const uint64_t cp = kidOff[blockIdx.x] + sRunK + wk + k - kc;
            if (pos < out.cap && cp + kc <= 0xffffffffull) {
                out.q[pos] = q;
                out.cbeg[pos] = F.cbeg[e];
                out.cpre[pos] = static_cast<uint32_t>(cp);
                for (int d = 0; d < D; ++d) out.x[pos * D + d] = F.x[e * D + d];
                for (unsigned long long b = (cp + kWarpTile - 1) / kWarpTile; b * kWarpTile < cp + kc; ++b)
                    if (b < out.tileCap) out.tileStart[b] = static_cast<uint32_t>(pos);
            }
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) {
            uint32_t tc = 0, tk = 0;
            for (int w = 0; w < kCompactThreads / 32; ++w) {
                tc += sCnt[w];
                tk += sKid[w];
            }
            sRunC += tc;
            sRunK += tk;
        }
        __syncthreads();
    }
}

__global__ void compactHeaderKernel(const uint64_t* entryOff, const uint64_t* kidOff, uint32_t nSeg, uint32_t* hdr) {
    const unsigned long long c = entryOff[nSeg], k = kidOff[nSeg];
    hdr[0] = static_cast<uint32_t>(c < 0xffffffffull ? c : 0xffffffffull);
    hdr[1] = static_cast<uint32_t>(k < 0xffffffffull ? k : 0xffffffffull);
}

}  // namespace

void launchCompactFrontier(const FrontierIn& F, uint32_t cap, int mode, const uint8_t* sel, const double* lb,
                           const double* tau, int D, uint32_t* cnt, uint32_t* kids, uint64_t* entryOff,
                           uint64_t* kidOff, const FrontierOut& out, cudaStream_t s) {
    const uint32_t nSeg = std::max<uint32_t>(1u, (cap + kSegment - 1) / kSegment);
    compactCountKernel<<<nSeg, kCompactThreads, 0, s>>>(F, mode, sel, lb, tau, cnt, kids);
    TBLAEQ_LAUNCHED();
    launchExclusiveScan(cnt, entryOff, nSeg, s);
    launchExclusiveScan(kids, kidOff, nSeg, s);
    compactWriteKernel<<<nSeg, kCompactThreads, 0, s>>>(F, mode, sel, lb, tau, entryOff, kidOff, D, out);
    TBLAEQ_LAUNCHED();
    compactHeaderKernel<<<1, 1, 0, s>>>(entryOff, kidOff, nSeg, out.hdr);
    TBLAEQ_LAUNCHED();
}

uint32_t compactSegments(uint64_t cap) { return static_cast<uint32_t>(std::max<uint64_t>(1, (cap + kSegment - 1) / kSegment)); }

}  // namespace tblaeq
