// Device-resident index for the B200 traversal engine.
//
// Besides the reference's arrays (P values, radii, maps, coarsest mesh; src/core/IndexData.cu:52-139)
// this keeps per-mesh node arrays in "position" order (mesh 0: coarsest list order; mesh m >= 1:
// sorted position = row of P_{m-1}), so a traversal never applies a Map until it writes final ids:
//   cbeg/ccnt[m][s]   first child row and child count of node s (its P_m column)
//   radRef[m][s]      the reference's max child radius (ref-parity pruning)
//   radSub[m][s]      largest distance to any finest point below s, with a conservative slack
//                     (exact pruning); leaf[m][s] = number of finest points below s
// plus the original-id arrays the per-level plugin (IQueryStrategy::runLevel) needs.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <vector>

#include "common.cuh"
#include "index.hpp"
#include "traverse.cuh"

namespace tblaeq {

// Allocation hook used by every device allocation of the library. Tests install a hook that
// fails the Nth allocation to check that errors surface cleanly without leaks.
using AllocHook = std::function<bool(size_t bytes)>;  // return false to fail the allocation
void setAllocHook(AllocHook hook);
size_t liveDeviceBytes();

class DeviceMem {
public:
    DeviceMem() = default;
    explicit DeviceMem(size_t bytes) { alloc(bytes); }
    ~DeviceMem() { release(); }
    DeviceMem(const DeviceMem&) = delete;
    DeviceMem& operator=(const DeviceMem&) = delete;
    DeviceMem(DeviceMem&& o) noexcept : p_(o.p_), n_(o.n_) {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    DeviceMem& operator=(DeviceMem&& o) noexcept {
        if (this != &o) {
            release();
            p_ = o.p_;
            n_ = o.n_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    void alloc(size_t bytes);
    void release();
    size_t bytes() const { return n_; }
    template <class T>
    T* as() const {
        return static_cast<T*>(p_);
    }
    void* get() const { return p_; }

private:
    void* p_ = nullptr;
    size_t n_ = 0;
};

template <class T>
DeviceMem upload(const std::vector<T>& v, cudaStream_t s = nullptr) {
    DeviceMem m(std::max<size_t>(v.size() * sizeof(T), 16));
    if (!v.empty()) TBLAEQ_CUDA(cudaMemcpyAsync(m.get(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    return m;
}

// Slack applied to subtree radii: R * (1 + kSubRadiusRelSlack) + kSubRadiusAbsSlack.
constexpr double kSubRadiusRelSlack = 1e-9;
constexpr double kSubRadiusAbsSlack = 1e-12;

struct DerivedArrays {
    // position-space per mesh m < height-1
    std::vector<std::vector<uint32_t>> cbeg, ccnt, leaf;
    std::vector<std::vector<double>> radRef, radSub;
    // Axis-aligned box of the finest points below each node: lo[D] then hi[D] per node, in float
    // rounded outward (lo down, hi up), so it always contains the decoded points.
    std::vector<std::vector<float>> aabb;
    // Decoded coordinates of every node (position order, D per node), as the traversal rebuilds
    // them (y = P[j] * x_parent, one rounded multiply per level).
    std::vector<std::vector<double>> nodeX;
    // Point groups of the finest exact range level (empty where its float test has no kernel: D not
    // 4, 8, 16). Every finest cluster's rows are reordered within the cluster's own row range by
    // median splits along the widest dimension until at most kPointGroup rows remain; each run so
    // formed is a point group, with the box of its points.
    std::vector<float> pointsF;          // decoded finest points in that order, floats rounded to nearest
    std::vector<uint32_t> pointPerm;     // reordered row -> row of the last interval's P tensor
    std::vector<uint32_t> groupFirst;    // per group: first reordered row
    std::vector<uint32_t> groupCount;    // per group: its rows
    std::vector<float> groupBox;         // per group: lo[D] hi[D] of its points, rounded outward
    std::vector<uint32_t> clusterGroup;  // per finest cluster (mesh H-2 position): first group; one more at the end
    // Decoded finest points (y = P[j] * x_parent, one rounded multiply per dimension), in
    // point-group order when the groups exist (pointPerm maps back to rows), else in row order.
    std::vector<double> pointsD;
};

// Most points of one point group.
constexpr uint32_t kPointGroup = 32;

// Host computation of the position-space node arrays, including subtree radii from the decoded
// hierarchy (decoded exactly like the traversal: y = P[j] * x_parent, one rounded multiply).
DerivedArrays computeDerived(const HostIndex& idx);

// A page-locked host range mapped into the device address space (zero-copy reads by kernels);
// unregistered when destroyed. The host memory must outlive it and must not move.
class HostMapping {
public:
    HostMapping() = default;
    HostMapping(const void* host, size_t bytes);
    ~HostMapping();
    HostMapping(const HostMapping&) = delete;
    HostMapping& operator=(const HostMapping&) = delete;
    HostMapping(HostMapping&& o) noexcept : host_(o.host_), dev_(o.dev_) { o.host_ = o.dev_ = nullptr; }
    HostMapping& operator=(HostMapping&& o) noexcept;
    const void* device() const { return dev_; }

private:
    void* host_ = nullptr;
    void* dev_ = nullptr;
};

// Residency of one interval's arrays, from the level policy (the reference's L0..L3,
// docs/memory_policies.md):
//   L0, L1  P values and maps in device memory (the library never allocates in the query path
//           either way, so the two coincide here);
//   L2      P values stay in page-locked host memory mapped into the device address space: the
//           traversal reads only the rows of the children it expands, across the host link, with
//           no host-side gather and no upload (the reference collects the surviving columns on
//           the host and uploads them, SpMSpV.cu:107-198);
//   L3      as L2, and the interval's sort-to-original map is read from host memory too.
// Node records, radii and boxes (one entry per cluster) and the coarsest mesh are always resident.
enum Residency : int { kResident = 0, kRowsOnHost = 1, kRowsAndMapOnHost = 2 };

struct DeviceIndex {
    uint64_t D = 0, height = 0, intervals = 0;
    std::vector<uint64_t> meshCount;  // by mesh m (0 = coarsest)

    // position space
    DeviceMem coarseVals;                    // mesh 0 rows (n0 * D)
    std::vector<DeviceMem> pvals;            // interval l: rows of P_l (n_{l+1} * D) when resident
    std::vector<const double*> rows;         // interval l: device-visible rows (pvals or mapped host memory)
    std::vector<uint8_t> rowsOnHost;         // interval l: rows are read from mapped host memory
    std::vector<const uint64_t*> mapPtr;     // mesh m >= 1: device-visible Map (maps or mapped host memory)
    std::vector<HostMapping> hostMaps;       // host ranges mapped for streamed intervals
    std::vector<DeviceMem> nodeRef, nodeSub; // mesh m < height-1: NodeRec {radius, first child, children}
    std::vector<DeviceMem> leaf;             // mesh m < height-1: finest points below each node (uint32)
    std::vector<DeviceMem> aabb;             // mesh m < height-1: outward-rounded float box of the points below
    std::vector<DeviceMem> nodeX;            // mesh m < height-1: decoded coordinates (D doubles per node)
    // Finest exact range level, when the last interval's rows are device-resident (else empty): the
    // points as floats in point-group order (DerivedArrays::pointsF), that order's row map, every
    // group's record {0, first row, rows} and box, and every finest cluster's record
    // {subtree radius, first group, groups}.
    DeviceMem pointsF, pointPerm, groupRec, groupBox, clusterGroups;
    // Decoded finest points (DerivedArrays::pointsD) for the KNN point kernels, when the last
    // interval's rows are device-resident; else empty.
    DeviceMem pointsD;

    // original-id space (per-level plugin)
    DeviceMem coarseIds;                     // uint64
    std::vector<DeviceMem> nodeOrig;         // interval l, NodeRec by original column id
    std::vector<DeviceMem> maps;             // mesh m >= 1 (uint64); maps[0] empty

    size_t deviceBytes() const;
};

// `residency` has one Residency per interval (empty: every interval resident).
std::unique_ptr<DeviceIndex> buildDeviceIndex(const HostIndex& idx, const DerivedArrays& der, cudaStream_t s,
                                              const std::vector<int>& residency = {});

}  // namespace tblaeq
