// C++ host facade with the reference's interfaces:
//   QueryHandler   (src/core/QueryHandler.cuh:50-247)   build / load / save / prepare / query
//   PolicyScheduler (src/core/MemoryPolicy.cuh:157-207) per-level L0..L3 recommendation
//   IQueryStrategy (src/core/strategies/IQueryStrategy.cuh:73-107) per-level plugin hook, whose
//                  B200 implementation runs each level on the device with no host round trip.
// The batched engine (engine.hpp) serves performBatch() and the plain one-query-at-a-time path.
#pragma once

#include <cstdint>
#include <iosfwd>
#include <memory>
#include <string>
#include <vector>

#include "device_index.hpp"
#include "engine.hpp"
#include "index.hpp"
#include "mlp.cuh"

namespace tblaeq {

// Same enumerator order as the reference (src/Data_Structures/File.cuh:39-43).
enum class QueryType { POINT = 0, RANGE = 1 };
enum class LevelPolicy { L0 = 0, L1 = 1, L2 = 2, L3 = 3 };

const char* levelPolicyName(LevelPolicy p);

struct IndexPolicy {
    std::vector<LevelPolicy> levels;
    static IndexPolicy uniform(size_t n, LevelPolicy p) {
        IndexPolicy r;
        r.levels.assign(n, p);
        return r;
    }
    static LevelPolicy parseLevel(const std::string& s);
};

// Byte accounting of src/core/IndexData.cu:141-194.
struct MemoryStats {
    uint64_t hostPTensors = 0, hostMaps = 0, hostRadius = 0, hostCoarsestMesh = 0, hostTotal = 0;
    uint64_t devicePTensorVals = 0, deviceMaps = 0, deviceRadius = 0, deviceCoarsestMesh = 0;
    uint64_t deviceSpTSpMBufs = 0, deviceTotal = 0, grandTotal = 0;
};
MemoryStats computeStats(const HostIndex& idx);

struct PolicyScheduler {
    static constexpr double kSafetyFactor = 0.85;
    // Greedy coarsest-first assignment of src/core/MemoryPolicy.cu:100-177 against `freeBytes`.
    static IndexPolicy recommend(const HostIndex& idx, uint64_t freeBytes);
};

// Non-owning view of a device-resident grid (ids + AOS coordinates).
struct Grid {
    uint64_t numRows = 0, dim = 0, nnz = 0;
    const uint64_t* ids = nullptr;
    const double* vals = nullptr;
};

struct LevelResult {
    Grid grid;
    bool ownsIds = false;   // the B200 strategy keeps ownership of its per-level output buffers
    bool ownsVals = false;
    bool onHost = false;
};

class IQueryStrategy {
public:
    virtual ~IQueryStrategy() = default;
    virtual void prepare(std::ostream& reportOs) = 0;
    virtual LevelResult runLevel(size_t l, const Grid& currentGrid, QueryType qType, const double* lo,
                                 const double* hi, const double* queryPoint, size_t K) = 0;
};

struct Runtime;  // device state shared by strategies and engines

// Per-level plugin: reference semantics (ref-parity), computed on the device.
class B200Strategy : public IQueryStrategy {
public:
    explicit B200Strategy(Runtime& rt) : rt_(rt) {}
    void prepare(std::ostream& reportOs) override;
    LevelResult runLevel(size_t l, const Grid& currentGrid, QueryType qType, const double* lo, const double* hi,
                         const double* queryPoint, size_t K) override;

private:
    Runtime& rt_;
};

struct QueryResult {
    QueryType type = QueryType::RANGE;
    int errorCode = 0;
    long totalTimeUs = 0;
    size_t queryCount = 0;
    std::string datasetName, queryParam, memoryPolicy;
    size_t datasetSize = 0, datasetDim = 0;
    std::vector<size_t> fineMeshSize;
    std::vector<size_t> levelOriginalSize;
    std::vector<std::vector<size_t>> levelFineMeshSize;
    std::vector<double> queryTimeUs;
    // Per query result ids (and KNN squared distances), on the host, when saveFineMesh is set.
    std::vector<std::vector<uint64_t>> ids;
    std::vector<std::vector<double>> dist2;
};

class QueryHandler {
public:
    explicit QueryHandler(const std::string& indexPath, bool loadFromIndex);
    explicit QueryHandler(const GenParams& gen);
    explicit QueryHandler(HostIndex&& built);  // an index built in memory (k-means build)
    ~QueryHandler();
    QueryHandler(const QueryHandler&) = delete;
    QueryHandler& operator=(const QueryHandler&) = delete;

    void saveIndex(const std::string& dirPath) const;
    void prepareForQuery();
    void prepareForQuery(const IndexPolicy& policy);
    void prepareForQuery(LevelPolicy level);
    bool prepared() const { return prepared_; }

    const HostIndex& index() const { return *host_; }
    const IndexPolicy& activePolicy() const { return policy_; }
    Runtime& runtime();

    // mode: kModeRefParity (reference candidate sets) or kModeExact.
    void setMode(int mode) { mode_ = mode; }
    int mode() const { return mode_; }

private:
    std::unique_ptr<HostIndex> host_;
    std::unique_ptr<Runtime> rt_;
    IndexPolicy policy_;
    bool prepared_ = false;
    int mode_ = kModeRefParity;
};

// Device state: device index, stream, batch engine and plugin workspaces.
struct Runtime {
    const HostIndex* host = nullptr;
    std::unique_ptr<DeviceIndex> dev;
    cudaStream_t stream = nullptr;
    std::unique_ptr<BatchEngine> engine;
    // Per-level plugin output buffers (level l owns the grid it returns until its next call).
    struct LevelBufs {
        DeviceMem ids, vals;
        uint64_t cap = 0;
    };
    std::vector<LevelBufs> levelOut;
    std::unique_ptr<BatchEngine> pluginEngine;  // workspace for the plugin's two expands
    // Per-level KNN plugin scratch: bound keys, labels (+ sort scratch), child counts, STEP bounds, mask.
    DeviceMem knnKeys, knnKeys2, knnLabels, knnLabels2, knnCnt, knnRr, pluginMask;
    uint64_t knnCap = 0;
    DeviceMem scratchQuery;  // lo|hi or point staged on the device
    // Learned frontier scorer and the maps its training labels need.
    std::unique_ptr<Mlp> scorer;
    double scorerInvScale = 1.0;
    uint64_t scorerSamples = 0, scorerPositives = 0;
    DeviceMem invMapFinest, parentFinest;
    ~Runtime();
};

}  // namespace tblaeq
