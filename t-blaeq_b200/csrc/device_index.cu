// Device-resident index and its derived position-space arrays.
#include "device_index.hpp"
#include "traverse.cuh"

#include <omp.h>

#include <algorithm>
#include <functional>
#include <atomic>
#include <cmath>
#include <limits>
#include <mutex>

namespace tblaeq {

namespace {
std::mutex gHookMutex;
AllocHook gHook;
std::atomic<size_t> gLiveBytes{0};
}  // namespace

void setAllocHook(AllocHook hook) {
    std::lock_guard<std::mutex> g(gHookMutex);
    gHook = std::move(hook);
}

size_t liveDeviceBytes() { return gLiveBytes.load(); }

void DeviceMem::alloc(size_t bytes) {
    release();
    if (bytes == 0) return;
    {
        std::lock_guard<std::mutex> g(gHookMutex);
        if (gHook && !gHook(bytes)) {
            throw CudaError(cudaErrorMemoryAllocation,
                            "device allocation of " + std::to_string(bytes) + " bytes refused by allocation hook");
        }
    }
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw CudaError(e, "cudaMalloc(" + std::to_string(bytes) + ") failed: " + cudaGetErrorString(e));
    }
    p_ = p;
    n_ = bytes;
    gLiveBytes += bytes;
}

void DeviceMem::release() {
    if (p_) {
        cudaFree(p_);
        gLiveBytes -= n_;
    }
    p_ = nullptr;
    n_ = 0;
}

DerivedArrays computeDerived(const HostIndex& idx) {
    const uint64_t D = idx.D, H = idx.height;
    DerivedArrays out;
    out.cbeg.resize(H - 1);
    out.ccnt.resize(H - 1);
    out.leaf.resize(H - 1);
    out.radRef.resize(H - 1);
    out.radSub.resize(H - 1);

    auto origOf = [&](uint64_t m, uint64_t pos) -> uint64_t {
        return (m == 0) ? idx.coarsest.ids[pos] : idx.maps[m][pos];
    };
    // Position of each node of mesh m given its original id.
    std::vector<std::vector<uint64_t>> posOf(H);
    for (uint64_t m = 0; m + 1 < H; ++m) {
        const uint64_t n = idx.meshCount(m);
        posOf[m].resize(n);
        for (uint64_t s = 0; s < n; ++s) posOf[m][origOf(m, s)] = s;
    }
    for (uint64_t m = 0; m + 1 < H; ++m) {
        const uint64_t n = idx.meshCount(m);
        const PTensor& P = idx.pTensors[m];
        out.cbeg[m].resize(n);
        out.ccnt[m].resize(n);
        out.radRef[m].resize(n);
        for (uint64_t s = 0; s < n; ++s) {
            const uint64_t o = origOf(m, s);
            out.cbeg[m][s] = static_cast<uint32_t>(P.colRes[o]);
            out.ccnt[m][s] = static_cast<uint32_t>(P.colRes[o + 1] - P.colRes[o]);
            out.radRef[m][s] = idx.radius[m][o];
        }
    }

    // Decoded coordinates of every mesh in position order, and each node's parent position.
    std::vector<std::vector<double>> dec(H);
    std::vector<std::vector<uint32_t>> parent(H);
    dec[0] = idx.coarsest.vals;
    for (uint64_t m = 0; m + 1 < H; ++m) {
        const PTensor& P = idx.pTensors[m];
        dec[m + 1].resize(idx.meshCount(m + 1) * D);
        parent[m + 1].resize(idx.meshCount(m + 1));
        const int64_t cols = static_cast<int64_t>(P.cols);
#pragma omp parallel for schedule(static)
        for (int64_t o = 0; o < cols; ++o) {
            const uint64_t ppos = posOf[m][o];
            const double* x = &dec[m][ppos * D];
            for (uint64_t j = P.colRes[o]; j < P.colRes[o + 1]; ++j) {
                parent[m + 1][j] = static_cast<uint32_t>(ppos);
                for (uint64_t d = 0; d < D; ++d) dec[m + 1][j * D + d] = P.vals[j * D + d] * x[d];
            }
        }
    }

    out.nodeX.resize(H - 1);
    for (uint64_t m = 0; m + 1 < H; ++m) out.nodeX[m] = dec[m];
    if (floatPointsSupported(D) && H >= 2) {
        // Point groups: every finest cluster's rows, reordered within the cluster's own row range by
        // median splits along the widest dimension until at most kPointGroup rows remain, and the
        // float copy of the points in that order.
        const std::vector<double>& pts = dec[H - 1];
        const uint64_t nRows = pts.size() / D;
        const uint64_t nCl = out.cbeg[H - 2].size();
        std::function<uint32_t(uint32_t)> leaves = [&](uint32_t n) -> uint32_t {
            return n <= kPointGroup ? 1u : leaves(n / 2) + leaves(n - n / 2);
        };
        out.clusterGroup.assign(nCl + 1, 0);
        for (uint64_t c = 0; c < nCl; ++c)
            out.clusterGroup[c + 1] = out.clusterGroup[c] + (out.ccnt[H - 2][c] ? leaves(out.ccnt[H - 2][c]) : 0u);
        const uint64_t G = out.clusterGroup[nCl];
        out.pointPerm.resize(nRows);
        out.pointsF.resize(nRows * D);
        out.groupFirst.resize(G);
        out.groupCount.resize(G);
        out.groupBox.resize(G * 2 * D);
        auto down = [](double v) {
            float f = static_cast<float>(v);
            if (static_cast<double>(f) > v) f = std::nextafter(f, -std::numeric_limits<float>::infinity());
            return f;
        };
        auto up = [](double v) {
            float f = static_cast<float>(v);
            if (static_cast<double>(f) < v) f = std::nextafter(f, std::numeric_limits<float>::infinity());
            return f;
        };
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t c = 0; c < static_cast<int64_t>(nCl); ++c) {
            const uint32_t b = out.cbeg[H - 2][c], n = out.ccnt[H - 2][c];
            std::vector<uint32_t> rows(n);
            for (uint32_t i = 0; i < n; ++i) rows[i] = b + i;
            uint32_t g = out.clusterGroup[c];
            // Explicit stack of (first, count) ranges of `rows`, split in order (left before right).
            std::vector<std::pair<uint32_t, uint32_t>> stack;
            if (n) stack.emplace_back(0u, n);
            while (!stack.empty()) {
                const auto [f, k] = stack.back();
                stack.pop_back();
                if (k <= kPointGroup) {
                    out.groupFirst[g] = b + f;
                    out.groupCount[g] = k;
                    float* box = &out.groupBox[static_cast<size_t>(g) * 2 * D];
                    for (uint64_t d = 0; d < D; ++d) {
                        double lo = std::numeric_limits<double>::infinity(), hi = -lo;
                        for (uint32_t i = f; i < f + k; ++i) {
                            lo = std::min(lo, pts[rows[i] * D + d]);
                            hi = std::max(hi, pts[rows[i] * D + d]);
                        }
                        box[d] = down(lo);
                        box[D + d] = up(hi);
                    }
                    ++g;
                    continue;
                }
                uint64_t best = 0;
                double bestExt = -1.0;
                for (uint64_t d = 0; d < D; ++d) {
                    double lo = std::numeric_limits<double>::infinity(), hi = -lo;
                    for (uint32_t i = f; i < f + k; ++i) {
                        lo = std::min(lo, pts[rows[i] * D + d]);
                        hi = std::max(hi, pts[rows[i] * D + d]);
                    }
                    if (hi - lo > bestExt) {
                        bestExt = hi - lo;
                        best = d;
                    }
                }
                const uint32_t h = k / 2;
                std::nth_element(rows.begin() + f, rows.begin() + f + h, rows.begin() + f + k,
                                 [&](uint32_t x, uint32_t y) {
                                     const double vx = pts[x * D + best], vy = pts[y * D + best];
                                     return vx < vy || (vx == vy && x < y);
                                 });
                stack.emplace_back(f + h, k - h);
                stack.emplace_back(f, h);
            }
            for (uint32_t i = 0; i < n; ++i) {
                out.pointPerm[b + i] = rows[i];
                for (uint64_t d = 0; d < D; ++d)
                    out.pointsF[(static_cast<size_t>(b) + i) * D + d] = static_cast<float>(pts[static_cast<size_t>(rows[i]) * D + d]);
            }
        }
    }
    // Box of the finest points below every node (exact min / max of decoded coordinates), stored
    // as floats rounded outward.
    {
        std::vector<std::vector<double>> bl(H - 1), bh(H - 1);
        for (uint64_t m = 0; m + 1 < H; ++m) {
            bl[m].assign(idx.meshCount(m) * D, std::numeric_limits<double>::infinity());
            bh[m].assign(idx.meshCount(m) * D, -std::numeric_limits<double>::infinity());
        }
        const uint64_t nLeaf = idx.meshCount(H - 1);
        for (uint64_t leafPos = 0; leafPos < nLeaf; ++leafPos) {
            const double* x = &dec[H - 1][leafPos * D];
            uint64_t pos = leafPos;
            for (uint64_t m = H - 1; m > 0; --m) {
                pos = parent[m][pos];  // position in mesh m-1
                double* l = &bl[m - 1][pos * D];
                double* u = &bh[m - 1][pos * D];
                for (uint64_t d = 0; d < D; ++d) {
                    l[d] = std::min(l[d], x[d]);
                    u[d] = std::max(u[d], x[d]);
                }
            }
        }
        out.aabb.resize(H - 1);
        auto down = [](double v) {
            float f = static_cast<float>(v);
            if (static_cast<double>(f) > v) f = std::nextafter(f, -std::numeric_limits<float>::infinity());
            return f;
        };
        auto up = [](double v) {
            float f = static_cast<float>(v);
            if (static_cast<double>(f) < v) f = std::nextafter(f, std::numeric_limits<float>::infinity());
            return f;
        };
        for (uint64_t m = 0; m + 1 < H; ++m) {
            const uint64_t n = idx.meshCount(m);
            out.aabb[m].resize(n * 2 * D);
            for (uint64_t s = 0; s < n; ++s)
                for (uint64_t d = 0; d < D; ++d) {
                    out.aabb[m][s * 2 * D + d] = down(bl[m][s * D + d]);
                    out.aabb[m][s * 2 * D + D + d] = up(bh[m][s * D + d]);
                }
        }
    }

    // Subtree radius and leaf count: walk every finest point up to the root. The finest
    // clusters (mesh H-2) own their points directly, so they are done cluster by cluster; the
    // small upper meshes use per-thread partial maxima.
    std::vector<std::vector<double>> R(H - 1);
    std::vector<std::vector<uint64_t>> C(H - 1);
    for (uint64_t m = 0; m + 1 < H; ++m) {
        R[m].assign(idx.meshCount(m), 0.0);
        C[m].assign(idx.meshCount(m), 0);
    }
    {
        const uint64_t m = H - 2;
        const int64_t n = static_cast<int64_t>(idx.meshCount(m));
        const PTensor& P = idx.pTensors[m];
#pragma omp parallel for schedule(static)
        for (int64_t s = 0; s < n; ++s) {
            const uint64_t o = origOf(m, s);
            const double* c = &dec[m][s * D];
            double best = 0.0;
            for (uint64_t j = P.colRes[o]; j < P.colRes[o + 1]; ++j) {
                const double* x = &dec[H - 1][j * D];
                double sum = 0.0;
                for (uint64_t d = 0; d < D; ++d) {
                    const double diff = c[d] - x[d];
                    sum += diff * diff;
                }
                best = std::max(best, std::sqrt(sum));
            }
            R[m][s] = best;
            C[m][s] = P.colRes[o + 1] - P.colRes[o];
        }
    }
    if (H >= 3) {
        const int nt = omp_get_max_threads();
        std::vector<std::vector<std::vector<double>>> partR(nt);
        std::vector<std::vector<std::vector<uint64_t>>> partC(nt);
        const int64_t nLeaf = static_cast<int64_t>(idx.meshCount(H - 1));
#pragma omp parallel
        {
            const int t = omp_get_thread_num();
            auto& pr = partR[t];
            auto& pc = partC[t];
            pr.resize(H - 2);
            pc.resize(H - 2);
            for (uint64_t m = 0; m + 2 < H; ++m) {
                pr[m].assign(idx.meshCount(m), 0.0);
                pc[m].assign(idx.meshCount(m), 0);
            }
#pragma omp for schedule(static)
            for (int64_t leafPos = 0; leafPos < nLeaf; ++leafPos) {
                const double* x = &dec[H - 1][leafPos * D];
                uint64_t pos = parent[H - 1][leafPos];  // mesh H-2
                for (uint64_t m = H - 2; m > 0; --m) {
                    pos = parent[m][pos];  // now in mesh m-1
                    const double* c = &dec[m - 1][pos * D];
                    double sum = 0.0;
                    for (uint64_t d = 0; d < D; ++d) {
                        const double diff = c[d] - x[d];
                        sum += diff * diff;
                    }
                    pr[m - 1][pos] = std::max(pr[m - 1][pos], std::sqrt(sum));
                    pc[m - 1][pos] += 1;
                }
            }
        }
        for (int t = 0; t < nt; ++t) {
            if (partR[t].empty()) continue;
            for (uint64_t m = 0; m + 2 < H; ++m) {
                for (uint64_t s = 0; s < idx.meshCount(m); ++s) {
                    R[m][s] = std::max(R[m][s], partR[t][m][s]);
                    C[m][s] += partC[t][m][s];
                }
            }
        }
    }
    for (uint64_t m = 0; m + 1 < H; ++m) {
        const uint64_t n = idx.meshCount(m);
        out.radSub[m].resize(n);
        out.leaf[m].resize(n);
        for (uint64_t s = 0; s < n; ++s) {
            out.radSub[m][s] = R[m][s] * (1.0 + kSubRadiusRelSlack) + kSubRadiusAbsSlack;
            out.leaf[m][s] = static_cast<uint32_t>(C[m][s]);
        }
    }
    if (!out.pointPerm.empty()) {
        // In point-group order, like the float copy (the KNN point kernel walks the groups).
        const std::vector<double>& pts = dec[H - 1];
        out.pointsD.resize(pts.size());
        const int64_t n = static_cast<int64_t>(out.pointPerm.size());
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i)
            for (uint64_t d = 0; d < D; ++d)
                out.pointsD[static_cast<size_t>(i) * D + d] = pts[static_cast<size_t>(out.pointPerm[i]) * D + d];
    } else {
        out.pointsD = std::move(dec[H - 1]);
    }
    return out;
}

HostMapping::HostMapping(const void* host, size_t bytes) {
    if (!host || bytes == 0) return;
    int dev = 0, readOnly = 0;
    TBLAEQ_CUDA(cudaGetDevice(&dev));
    TBLAEQ_CUDA(cudaDeviceGetAttribute(&readOnly, cudaDevAttrHostRegisterReadOnlySupported, dev));
    unsigned flags = cudaHostRegisterMapped | (readOnly ? cudaHostRegisterReadOnly : 0u);
    void* h = const_cast<void*>(host);
    TBLAEQ_CUDA(cudaHostRegister(h, bytes, flags));
    void* d = nullptr;
    const cudaError_t e = cudaHostGetDevicePointer(&d, h, 0);
    if (e != cudaSuccess) {
        cudaHostUnregister(h);
        throw CudaError(e, "cudaHostGetDevicePointer");
    }
    host_ = h;
    dev_ = d;
}

HostMapping::~HostMapping() {
    if (host_) cudaHostUnregister(host_);
}

HostMapping& HostMapping::operator=(HostMapping&& o) noexcept {
    if (this != &o) {
        if (host_) cudaHostUnregister(host_);
        host_ = o.host_;
        dev_ = o.dev_;
        o.host_ = o.dev_ = nullptr;
    }
    return *this;
}

std::unique_ptr<DeviceIndex> buildDeviceIndex(const HostIndex& idx, const DerivedArrays& der, cudaStream_t s,
                                              const std::vector<int>& residency) {
    if (!residency.empty() && residency.size() != idx.intervals)
        throw std::invalid_argument("buildDeviceIndex: one residency per interval");
    auto res = [&](uint64_t l) { return residency.empty() ? static_cast<int>(kResident) : residency[l]; };
    auto di = std::make_unique<DeviceIndex>();
    di->D = idx.D;
    di->height = idx.height;
    di->intervals = idx.intervals;
    di->meshCount.resize(idx.height);
    for (uint64_t m = 0; m < idx.height; ++m) di->meshCount[m] = idx.meshCount(m);

    di->coarseVals = upload(idx.coarsest.vals, s);
    di->coarseIds = upload(idx.coarsest.ids, s);
    di->pvals.resize(idx.intervals);
    di->rows.assign(idx.intervals, nullptr);
    di->rowsOnHost.assign(idx.intervals, 0);
    di->nodeOrig.resize(idx.intervals);
    di->hostMaps.reserve(2 * idx.intervals);
    for (uint64_t l = 0; l < idx.intervals; ++l) {
        const PTensor& P = idx.pTensors[l];
        if (res(l) == kResident || P.vals.empty()) {
            di->pvals[l] = upload(P.vals, s);
            di->rows[l] = di->pvals[l].as<double>();
        } else {
            di->hostMaps.emplace_back(P.vals.data(), P.vals.size() * sizeof(double));
            di->rows[l] = static_cast<const double*>(di->hostMaps.back().device());
            di->rowsOnHost[l] = 1;
        }
        std::vector<NodeRec> rec(P.cols);
        for (uint64_t o = 0; o < P.cols; ++o) {
            rec[o].rad = idx.radius[l][o];
            rec[o].cbeg = static_cast<uint32_t>(P.colRes[o]);
            rec[o].cnt = static_cast<uint32_t>(P.colRes[o + 1] - P.colRes[o]);
        }
        di->nodeOrig[l] = upload(rec, s);
        TBLAEQ_CUDA(cudaStreamSynchronize(s));
    }
    di->maps.resize(idx.height);
    di->mapPtr.assign(idx.height, nullptr);
    for (uint64_t m = 1; m < idx.height; ++m) {
        // Map m belongs to interval m-1 (it maps that interval's output rows to original ids).
        if (res(m - 1) == kRowsAndMapOnHost && !idx.maps[m].empty()) {
            di->hostMaps.emplace_back(idx.maps[m].data(), idx.maps[m].size() * sizeof(uint64_t));
            di->mapPtr[m] = static_cast<const uint64_t*>(di->hostMaps.back().device());
        } else {
            di->maps[m] = upload(idx.maps[m], s);
            di->mapPtr[m] = di->maps[m].as<uint64_t>();
        }
    }
    // The finest map doubles as the final-id map of the fused traversal.
    di->nodeRef.resize(idx.height - 1);
    di->nodeSub.resize(idx.height - 1);
    di->leaf.resize(idx.height - 1);
    di->aabb.resize(idx.height - 1);
    di->nodeX.resize(idx.height - 1);
    for (uint64_t m = 0; m + 1 < idx.height; ++m) {
        const size_t n = der.cbeg[m].size();
        std::vector<NodeRec> ref(n), sub(n);
        for (size_t i = 0; i < n; ++i) {
            ref[i] = NodeRec{der.radRef[m][i], der.cbeg[m][i], der.ccnt[m][i]};
            sub[i] = NodeRec{der.radSub[m][i], der.cbeg[m][i], der.ccnt[m][i]};
        }
        di->nodeRef[m] = upload(ref, s);
        di->nodeSub[m] = upload(sub, s);
        di->leaf[m] = upload(der.leaf[m], s);
        di->aabb[m] = upload(der.aabb[m], s);
        di->nodeX[m] = upload(der.nodeX[m], s);
        TBLAEQ_CUDA(cudaStreamSynchronize(s));
    }
    if (!der.pointsD.empty() && idx.intervals > 0 && res(idx.intervals - 1) == kResident) {
        di->pointsD = upload(der.pointsD, s);
        TBLAEQ_CUDA(cudaStreamSynchronize(s));
    }
    // The float copy and the point groups (about 0.6 of the last interval's rows at D = 8) stay on
    // the device even when those rows are streamed, as long as they take at most a quarter of the
    // free memory: the exact range batch then decides nearly every point on the device and reads
    // a row across the host link only near a face of a box.
    bool floatCopy = !der.pointsF.empty() && idx.intervals > 0;
    if (floatCopy && res(idx.intervals - 1) != kResident) {
        const size_t need = der.pointsF.size() * 4 + der.pointPerm.size() * 4 + der.groupBox.size() * 4 +
                            der.groupFirst.size() * 16 + der.clusterGroup.size() * 16;
        size_t freeB = 0, totalB = 0;
        TBLAEQ_CUDA(cudaMemGetInfo(&freeB, &totalB));
        floatCopy = need * 4 <= freeB;
    }
    if (floatCopy) {
        di->pointsF = upload(der.pointsF, s);
        di->pointPerm = upload(der.pointPerm, s);
        const size_t G = der.groupFirst.size(), nCl = der.clusterGroup.size() - 1;
        std::vector<NodeRec> grec(G), crec(nCl);
        for (size_t g = 0; g < G; ++g) grec[g] = NodeRec{0.0, der.groupFirst[g], der.groupCount[g]};
        for (size_t c = 0; c < nCl; ++c)
            crec[c] = NodeRec{der.radSub[idx.height - 2][c], der.clusterGroup[c],
                              der.clusterGroup[c + 1] - der.clusterGroup[c]};
        di->groupRec = upload(grec, s);
        di->groupBox = upload(der.groupBox, s);
        di->clusterGroups = upload(crec, s);
        TBLAEQ_CUDA(cudaStreamSynchronize(s));
    }
    TBLAEQ_CUDA(cudaStreamSynchronize(s));
    return di;
}

size_t DeviceIndex::deviceBytes() const {
    size_t t = coarseVals.bytes() + coarseIds.bytes();
    for (auto* v : {&pvals, &nodeRef, &nodeSub, &leaf, &aabb, &nodeX, &nodeOrig, &maps})
        for (auto& m : *v) t += m.bytes();
    return t + pointsD.bytes() + pointsF.bytes() + pointPerm.bytes() + groupRec.bytes() + groupBox.bytes() + clusterGroups.bytes();
}

}  // namespace tblaeq
