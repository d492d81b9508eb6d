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
};

// Host computation of the position-space node arrays, including subtree radii from the decoded
// hierarchy (decoded exactly like the traversal: y = P[j] * x_parent, one rounded multiply).
DerivedArrays computeDerived(const HostIndex& idx);

struct DeviceIndex {
    uint64_t D = 0, height = 0, intervals = 0;
    std::vector<uint64_t> meshCount;  // by mesh m (0 = coarsest)

    // position space
    DeviceMem coarseVals;                    // mesh 0 rows (n0 * D)
    std::vector<DeviceMem> pvals;            // interval l: rows of P_l (n_{l+1} * D)
    std::vector<DeviceMem> nodeRef, nodeSub; // mesh m < height-1: NodeRec {radius, first child, children}
    std::vector<DeviceMem> leaf;             // mesh m < height-1: finest points below each node (uint32)
    std::vector<DeviceMem> aabb;             // mesh m < height-1: outward-rounded float box of the points below

    // original-id space (per-level plugin)
    DeviceMem coarseIds;                     // uint64
    std::vector<DeviceMem> nodeOrig;         // interval l, NodeRec by original column id
    std::vector<DeviceMem> maps;             // mesh m >= 1 (uint64); maps[0] empty

    size_t deviceBytes() const;
};

std::unique_ptr<DeviceIndex> buildDeviceIndex(const HostIndex& idx, const DerivedArrays& der, cudaStream_t s);

}  // namespace tblaeq
