// Exact KNN completion, node-major (see knn.cuh for the design).
#include <algorithm>

#include "knn.cuh"

namespace tblaeq {

namespace {

constexpr int kThreadsNm = 128;
constexpr uint32_t FULL = 0xffffffffu;

// The unit (node, up to 32 of its pairs) of ticket u: the node is the last one whose units start at
// or before u (nodes without pairs own no unit).
struct Unit {
    uint32_t node, base, count;
};
__device__ __forceinline__ Unit unitOf(uint32_t u, const uint32_t* nodeOff, const uint32_t* unitOff, uint32_t nNodes,
                                      const uint32_t* unitNode) {
    uint32_t lo = 0, hi = nNodes - 1;
    if (unitNode) {
        lo = min(__ldg(unitNode + u), nNodes - 1);  // the transpose's map (clamped for safety)
    } else {
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(unitOff + mid) <= u) lo = mid; else hi = mid - 1;
        }
    }
    Unit r;
    r.node = lo;
    r.base = __ldg(nodeOff + lo) + (u - __ldg(unitOff + lo)) * 32u;
    r.count = min(32u, __ldg(nodeOff + lo + 1) - r.base);
    return r;
}

// Appends the pairs of the lanes in `keep` at consecutive positions of a shared counter. A counter
// past 2^31 raises kStatusOverflowSum (the batch must be split) before it could wrap, and returns
// positions no capacity reaches.
__device__ __forceinline__ uint32_t appendPos(bool keep, uint32_t* counter, uint32_t* status, int lane) {
    const uint32_t kb = __ballot_sync(FULL, keep);
    if (kb == 0) return 0xffffffffu;
    const int leader = __ffs(kb) - 1;
    uint32_t base = 0;
    if (lane == leader) {
        base = atomicAdd(counter, static_cast<uint32_t>(__popc(kb)));
        if (base >= 0x80000000u) atomicOr(status, kStatusOverflowSum);
    }
    base = __shfl_sync(FULL, base, leader);
    if (base >= 0x80000000u) return 0xffffffffu;
    return base + __popc(kb & ((1u << lane) - 1u));
}

template <int D>
__global__ void __launch_bounds__(kThreadsNm) knnBoundLevelKernel(KnnBoundLevelArgs a) {
    constexpr int DM = D > 0 ? D : 32;
    if (*a.status & kStatusInconsistent) return;
    const int dim = D > 0 ? D : a.D;
    const int lane = threadIdx.x & 31;
    const bool root = a.nNodes == 0;
    const uint32_t entries = root ? a.nq : *a.inCount;
    if (!root && entries > a.inCap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(a.status, kStatusOverflowEntries);
        return;
    }
    const uint32_t units = root ? (entries + 31u) / 32u : a.unitOff[a.nNodes];
    while (true) {
        uint32_t u = 0;
        if (lane == 0) u = atomicAdd(a.ticket, 1u);
        u = __shfl_sync(FULL, u, 0);
        if (u >= units) break;
        Unit un;
        uint32_t cbeg = 0, cnt = a.rootChildren;
        if (root) {
            un.node = 0;
            un.base = u * 32u;
            un.count = min(32u, entries - un.base);
        } else {
            un = unitOf(u, a.nodeOff, a.unitOff, a.nNodes, a.unitNode);
            const NodeRec pr = a.parents[un.node];
            cbeg = pr.cbeg;
            cnt = pr.cnt;
        }
        const bool active = static_cast<uint32_t>(lane) < un.count;
        uint32_t q = 0;
        if (active) q = root ? un.base + lane : __ldg(a.inQ + __ldg(a.list + un.base + lane));
        double p[DM];
#pragma unroll
        for (int d = 0; d < DM; ++d)
            if (D > 0 || d < dim) p[d] = active ? __ldg(a.points + static_cast<size_t>(q) * dim + d) : 0.0;
        const double tau = active ? __ldcg(a.tau + q) : -1.0;
        for (uint32_t c = 0; c < cnt; ++c) {
            const uint32_t j = cbeg + c;
            const NodeRec nr = a.nodes[j];
            const double* xc = a.x + static_cast<size_t>(j) * dim;
            const float* b = a.aabb + static_cast<size_t>(j) * 2 * dim;
            // The expand kernel's KNN bound (kPredKnnBound): centre distance minus the subtree radius,
            // and the distance to the outward-rounded box, slightly reduced.
            double dist = 0.0, gap = 0.0;
#pragma unroll
            for (int d = 0; d < DM; ++d) {
                if (D > 0 || d < dim) {
                    const double diff = p[d] - __ldg(xc + d);
                    dist = __fma_rn(diff, diff, dist);
                    const double l = static_cast<double>(__ldg(b + d)), h = static_cast<double>(__ldg(b + dim + d));
                    const double g = fmax(fmax(l - p[d], p[d] - h), 0.0);
                    gap = __fma_rn(g, g, gap);
                }
            }
            const double lb = fmax(sqrt(dist) - nr.rad, sqrt(gap) * (1.0 - 1e-12));
            const bool keep = active && nr.cnt > 0 && lb <= tau;
            if (__ballot_sync(FULL, keep) == 0) continue;
            const uint32_t pos = appendPos(keep, a.outCount, a.status, lane);
            if (keep) {
                if (pos < a.outCap) {
                    a.outQ[pos] = q;
                    a.outNode[pos] = j;
                } else {
                    atomicOr(a.status, kStatusOverflowEntries);
                }
            }
        }
    }
}

template <int D>
__global__ void __launch_bounds__(kThreadsNm) knnClusterPointsKernel(KnnClusterArgs a) {
    constexpr int DM = D > 0 ? D : 32;
    if (*a.status & kStatusInconsistent) return;
    const int dim = D > 0 ? D : a.D;
    const int lane = threadIdx.x & 31;
    const uint32_t entries = *a.inCount;
    if (entries > a.inCap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(a.status, kStatusOverflowEntries);
        return;
    }
    const uint32_t units = a.unitOff[a.nNodes];
    unsigned long long rows = 0;
    while (true) {
        uint32_t u = 0;
        if (lane == 0) u = atomicAdd(a.ticket, 1u);
        u = __shfl_sync(FULL, u, 0);
        if (u >= units) break;
        const Unit un = unitOf(u, a.nodeOff, a.unitOff, a.nNodes, a.unitNode);
        const NodeRec cr = a.clusters[un.node];
        bool active = static_cast<uint32_t>(lane) < un.count;
        uint32_t q = 0;
        if (active) {
            q = __ldg(a.inQ + __ldg(a.list + un.base + lane));
            // Wave 1's clusters of this query fill its row from the start; ~0 ends them.
            for (uint32_t i = 0; i < a.exclStride; ++i) {
                const uint32_t c = __ldg(a.excl + static_cast<size_t>(q) * a.exclStride + i);
                if (c == 0xffffffffu) break;
                if (c == un.node) active = false;
            }
        }
        const uint32_t am = __ballot_sync(FULL, active);
        if (am == 0) continue;
        double p[DM];
#pragma unroll
        for (int d = 0; d < DM; ++d)
            if (D > 0 || d < dim) p[d] = active ? __ldg(a.points + static_cast<size_t>(q) * dim + d) : 0.0;
        const double t = active ? __ldcg(a.tau + q) : 0.0;
        const double t2 = t * t * (1.0 + 1e-9);
        if (active) {
            // The pair was listed under an earlier (looser) bound: skip it when the cluster's sphere
            // lies beyond the current one (the slack keeps the test conservative).
            const double* xc = a.x + static_cast<size_t>(un.node) * dim;
            double dc = 0.0;
#pragma unroll
            for (int d = 0; d < DM; ++d) {
                if (D > 0 || d < dim) {
                    const double diff = p[d] - __ldg(xc + d);
                    dc = __fma_rn(diff, diff, dc);
                }
            }
            if ((sqrt(dc) - cr.rad) * (1.0 - 1e-9) > t + 1e-12) active = false;
        }
        const uint32_t live = __ballot_sync(FULL, active);
        if (live == 0) continue;
        const uint32_t stride = a.sampleStride > 1 ? a.sampleStride : 1u;
        const uint32_t nPts = (cr.cnt + stride - 1) / stride;  // points this pass tests
        if (lane == 0) rows += static_cast<unsigned long long>(__popc(live)) * nPts;
        // Appends the candidate (query q, row j; a position when decoded is in group order) when kept.
        auto emit = [&](bool keep, uint32_t j, double dist) {
            if (__ballot_sync(FULL, keep) == 0) return;
            const uint32_t pos = appendPos(keep, a.outCount, a.status, lane);
            if (keep) {
                atomicAdd(&a.qcount[q], 1u);
                if (pos < a.outCap) {
                    a.outQ[pos] = q;
                    a.outId[pos] = a.map[(a.decoded && a.perm) ? __ldg(a.perm + j) : j];
                    a.outD2[pos] = dist;
                } else {
                    atomicOr(a.status, kStatusOverflowEntries);
                }
            }
        };
        // Four decoded points at a time (the products below, made once when the index was
        // prepared): four independent fma chains per lane instead of one. A run past its end
        // repeats its last point, which is never emitted twice.
        auto run = [&](bool act, uint32_t first, uint32_t n, uint32_t step) {
            const double* yb = a.decoded + static_cast<size_t>(first) * dim;
            for (uint32_t c0 = 0; c0 < n; c0 += 4) {
                const uint32_t nIn = min(4u, n - c0);
                double dist[4] = {0.0, 0.0, 0.0, 0.0};
                const double* y4[4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    y4[i] = yb + static_cast<size_t>((c0 + min(static_cast<uint32_t>(i), nIn - 1)) * step) * dim;
#pragma unroll
                for (int d = 0; d < DM; ++d) {
                    if (D > 0 || d < dim) {
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const double diff = p[d] - __ldg(y4[i] + d);
                            dist[i] = __fma_rn(diff, diff, dist[i]);
                        }
                    }
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (static_cast<uint32_t>(i) < nIn) emit(act && dist[i] <= t2, first + (c0 + i) * step, dist[i]);
            }
        };
        if (a.decoded && a.groupRec && stride == 1) {
            // The cluster's point groups: a lane skips a group whose box lies beyond its bound.
            const NodeRec cg = a.clusterGroups[un.node];
            unsigned long long tested = 0;
            for (uint32_t g = cg.cbeg; g < cg.cbeg + cg.cnt; ++g) {
                const NodeRec gr = a.groupRec[g];
                bool act = active;
                if (act) {
                    const float* b = a.groupBox + static_cast<size_t>(g) * 2 * dim;
                    double gap = 0.0;
#pragma unroll
                    for (int d = 0; d < DM; ++d) {
                        if (D > 0 || d < dim) {
                            const double lo = static_cast<double>(__ldg(b + d)), hi = static_cast<double>(__ldg(b + dim + d));
                            const double e = fmax(fmax(lo - p[d], p[d] - hi), 0.0);
                            gap = __fma_rn(e, e, gap);
                        }
                    }
                    act = gap * (1.0 - 1e-9) <= t2;
                }
                const uint32_t gm = __ballot_sync(FULL, act);
                if (gm == 0) continue;
                tested += static_cast<unsigned long long>(__popc(gm)) * gr.cnt;
                run(act, gr.cbeg, gr.cnt, 1);
            }
            if (lane == 0) rows += tested - static_cast<unsigned long long>(__popc(live)) * nPts;
        } else if (a.decoded) {
            run(active, cr.cbeg, nPts, stride);
        } else {
            for (uint32_t c = 0; c < nPts; ++c) {
                const uint32_t j = cr.cbeg + c * stride;
                const double* row = a.rows + static_cast<size_t>(j) * dim;
                const double* xc = a.x + static_cast<size_t>(un.node) * dim;
                // The expand kernel's point test (kPredKnnPoint): the point rebuilt with one rounded
                // multiply per dimension, the squared distance accumulated with fma in dimension order.
                double dist = 0.0;
#pragma unroll
                for (int d = 0; d < DM; ++d) {
                    if (D > 0 || d < dim) {
                        const double r = a.rowsOnHost ? row[d] : __ldg(row + d);
                        const double diff = p[d] - __dmul_rn(r, __ldg(xc + d));
                        dist = __fma_rn(diff, diff, dist);
                    }
                }
                emit(active && dist <= t2, j, dist);
            }
        }
    }
    if (a.work && lane == 0 && rows) atomicAdd(a.work, rows);
}

template <int D>
__global__ void __launch_bounds__(256) knnFilterPairsKernel(KnnFilterArgs a) {
    constexpr int DM = D > 0 ? D : 32;
    if (*a.status & kStatusInconsistent) return;
    const int dim = D > 0 ? D : a.D;
    const int lane = threadIdx.x & 31;
    const uint32_t n = *a.inCount;
    if (n > a.inCap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(a.status, kStatusOverflowEntries);
        return;
    }
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {  // warp-uniform
        const uint32_t i = base + lane;
        bool keep = i < n;
        uint32_t q = 0, c = 0;
        if (keep) {
            q = __ldg(a.inQ + i);
            c = __ldg(a.inNode + i);
            for (uint32_t k = 0; k < a.exclStride; ++k) {
                const uint32_t e = __ldg(a.excl + static_cast<size_t>(q) * a.exclStride + k);
                if (e == 0xffffffffu) break;
                if (e == c) keep = false;
            }
        }
        if (keep) {
            const double* p = a.points + static_cast<size_t>(q) * dim;
            const double* xc = a.x + static_cast<size_t>(c) * dim;
            double dc = 0.0;
#pragma unroll
            for (int d = 0; d < DM; ++d) {
                if (D > 0 || d < dim) {
                    const double diff = __ldg(p + d) - __ldg(xc + d);
                    dc = __fma_rn(diff, diff, dc);
                }
            }
            const double t = __ldcg(a.tau + q);
            keep = !((sqrt(dc) - a.clusters[c].rad) * (1.0 - 1e-9) > t + 1e-12);
        }
        const uint32_t pos = appendPos(keep, a.outCount, a.status, lane);
        if (keep && pos < a.outCap) {
            a.outQ[pos] = q;
            a.outNode[pos] = c;
        } else if (keep) {
            atomicOr(a.status, kStatusOverflowEntries);
        }
    }
}

__global__ void waveOneClustersKernel(const uint64_t* selIds, const uint64_t* selOff, const uint32_t* selCount,
                                      const uint32_t* node, uint64_t cap, uint32_t nq, uint32_t stride, uint32_t* excl) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nq * stride; i += gridDim.x * blockDim.x) {
        const uint32_t q = i / stride, k = i % stride;
        uint32_t v = 0xffffffffu;
        if (k < selCount[q]) {
            const uint64_t e = selIds[selOff[q] + k];
            if (e < cap) v = node[e];
        }
        excl[i] = v;
    }
}

__global__ void fillU32Kernel(uint32_t* v, uint32_t value, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = value;
}

template <class K>
int persistentGrid(K kern) {
    int dev = 0, sms = 0, perSm = 0;
    TBLAEQ_CUDA(cudaGetDevice(&dev));
    TBLAEQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    TBLAEQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kThreadsNm, 0));
    return std::max(1, sms * std::max(1, perSm));
}

template <int D>
void boundLevelD(const KnnBoundLevelArgs& a, cudaStream_t s) {
    static const int g = persistentGrid(knnBoundLevelKernel<D>);
    knnBoundLevelKernel<D><<<g, kThreadsNm, 0, s>>>(a);
    TBLAEQ_LAUNCHED();
}

template <int D>
void clusterPointsD(const KnnClusterArgs& a, cudaStream_t s) {
    static const int g = persistentGrid(knnClusterPointsKernel<D>);
    knnClusterPointsKernel<D><<<g, kThreadsNm, 0, s>>>(a);
    TBLAEQ_LAUNCHED();
}

int smallGridNm(uint64_t n) { return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 148 * 8))); }

}  // namespace

void launchKnnBoundLevel(const KnnBoundLevelArgs& a, cudaStream_t s) {
    switch (a.D) {
        case 2: return boundLevelD<2>(a, s);
        case 3: return boundLevelD<3>(a, s);
        case 4: return boundLevelD<4>(a, s);
        case 5: return boundLevelD<5>(a, s);
        case 8: return boundLevelD<8>(a, s);
        case 16: return boundLevelD<16>(a, s);
        default:
            if (a.D < 1 || a.D > 32) throw std::invalid_argument("KNN bound level: D must be in [1, 32]");
            return boundLevelD<0>(a, s);
    }
}

void launchKnnClusterPoints(const KnnClusterArgs& a, cudaStream_t s) {
    switch (a.D) {
        case 2: return clusterPointsD<2>(a, s);
        case 3: return clusterPointsD<3>(a, s);
        case 4: return clusterPointsD<4>(a, s);
        case 5: return clusterPointsD<5>(a, s);
        case 8: return clusterPointsD<8>(a, s);
        case 16: return clusterPointsD<16>(a, s);
        default:
            if (a.D < 1 || a.D > 32) throw std::invalid_argument("KNN point level: D must be in [1, 32]");
            return clusterPointsD<0>(a, s);
    }
}

template <int D>
void filterPairsD(const KnnFilterArgs& a, cudaStream_t s) {
    knnFilterPairsKernel<D><<<148 * 8, 256, 0, s>>>(a);
    TBLAEQ_LAUNCHED();
}

void launchKnnFilterPairs(const KnnFilterArgs& a, cudaStream_t s) {
    switch (a.D) {
        case 8: return filterPairsD<8>(a, s);
        case 16: return filterPairsD<16>(a, s);
        default:
            if (a.D < 1 || a.D > 32) throw std::invalid_argument("KNN pair filter: D must be in [1, 32]");
            return filterPairsD<0>(a, s);
    }
}

void launchWaveOneClusters(const uint64_t* selIds, const uint64_t* selOff, const uint32_t* selCount,
                           const uint32_t* node, uint64_t cap, uint32_t nq, uint32_t stride, uint32_t* excl,
                           cudaStream_t s) {
    if (nq == 0 || stride == 0) return;
    waveOneClustersKernel<<<smallGridNm(static_cast<uint64_t>(nq) * stride), 256, 0, s>>>(selIds, selOff, selCount, node,
                                                                                        cap, nq, stride, excl);
    TBLAEQ_LAUNCHED();
}

void launchFillU32(uint32_t* v, uint32_t value, uint32_t n, cudaStream_t s) {
    if (n == 0) return;
    fillU32Kernel<<<smallGridNm(n), 256, 0, s>>>(v, value, n);
    TBLAEQ_LAUNCHED();
}

}  // namespace tblaeq
