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

// Non-owning view of a device-resident grid (ids + AOS coordinates), with the accessors of the
// reference's SparseGrid (src/Data_Structures/Data_Structures.cuh:134-229; its raw-pointer
// constructor is non-owning too).
struct SparseGrid {
    uint64_t numRows = 0, dim = 0, nnz = 0;
    const uint64_t* ids = nullptr;
    const double* vals = nullptr;
    size_t get_num_rows() const { return numRows; }
    size_t get_dimensions() const { return dim; }
    size_t get_nnz_nums() const { return nnz; }
    size_t numNnz() const { return nnz; }
    const uint64_t* get_ids_() const { return ids; }
    const double* get_vals_() const { return vals; }
};
using Grid = SparseGrid;

// src/core/strategies/IQueryStrategy.cuh:38-43: the grid a level returns and who frees what. The
// grid object itself is always heap-allocated and deleted by the caller; ownsIds / ownsVals say
// whether its buffers go with it (the B200 strategy keeps its per-level output buffers, like L0).
struct LevelResult {
    SparseGrid* grid = nullptr;
    bool ownsIds = false;
    bool ownsVals = false;
    bool onHost = false;
};

// src/core/strategies/IQueryStrategy.cuh:73-107.
class IQueryStrategy {
public:
    virtual ~IQueryStrategy() = default;
    virtual void prepare(std::ostream& reportOs) = 0;
    virtual LevelResult runLevel(size_t l, SparseGrid* currentGrid, QueryType qType, const double* lo,
                                 const double* hi, const double* queryPoint, size_t K) = 0;
};

struct Runtime;  // device state shared by strategies and engines

// Per-level plugin: reference semantics (ref-parity), computed on the device.
class B200Strategy : public IQueryStrategy {
public:
    explicit B200Strategy(Runtime& rt) : rt_(rt) {}
    void prepare(std::ostream& reportOs) override;
    LevelResult runLevel(size_t l, SparseGrid* currentGrid, QueryType qType, const double* lo, const double* hi,
                         const double* queryPoint, size_t K) override;

private:
    Runtime& rt_;
};

// The reference's Query (src/Data_Structures/File.cuh:52-109): `length` rows of `dim` values
// (POINT) or 2 * dim values lo | hi (RANGE), row-major.
struct Query {
    QueryType type = QueryType::RANGE;
    size_t length = 0, dim = 0;
    std::vector<double> data;
    const double* getQueryPoint(size_t i) const { return data.data() + i * dim; }
    const double* getQueryLo(size_t i) const { return data.data() + i * 2 * dim; }
    const double* getQueryHi(size_t i) const { return data.data() + i * 2 * dim + dim; }
};
// Query files (src/Data_Structures/File.cu:159-205): a header "n D", then n rows of 2D (range) or D
// (point) values. Throws std::runtime_error with the reference's messages.
Query loadQueryFile(const std::string& path, QueryType type);

struct QueryResult {
    QueryType type = QueryType::RANGE;
    int errorCode = 0;
    long totalTimeUs = 0;
    size_t queryCount = 0;
    std::string datasetName, queryParam, memoryPolicy;
    size_t datasetSize = 0, datasetDim = 0;
    std::vector<double> queryRangeVolume;  // per query: log volume of the box (RANGE), 1.0 (KNN), as the reference
    std::vector<size_t> fineMeshSize;
    std::vector<size_t> levelOriginalSize;
    std::vector<std::vector<size_t>> levelFineMeshSize;
    std::vector<long> queryTimeUs;
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

    // src/core/QueryHandler.cuh:189-216. One query at a time through QueryEngine (ref-parity: the
    // per-level B200 strategy; exact: the batched engine with one query), timed per query like the
    // reference; performSingleRangeQuery keeps the reference's upper-bound-first order. With
    // saveFineMesh each query's result ids (and KNN squared distances) are copied to the host.
    QueryResult performQuery(const std::string& queryFilePath, QueryType type, bool saveFineMesh = false,
                             size_t maxQueryCount = static_cast<size_t>(-1), size_t K = 0);
    QueryResult performSingleKNNQuery(const std::vector<double>& point, size_t K, bool saveFineMesh = false);
    QueryResult performSingleRangeQuery(const std::vector<double>& upper, const std::vector<double>& lower,
                                        bool saveFineMesh = false);

private:
    std::unique_ptr<HostIndex> host_;
    std::unique_ptr<Runtime> rt_;
    IndexPolicy policy_;
    bool prepared_ = false;
    int mode_ = kModeRefParity;
};

// src/core/QueryEngine.cuh:78-100: runs queries level by level through the per-level strategy.
struct RunConfig {
    size_t maxQueryCount = static_cast<size_t>(-1);
    size_t K = 0;
    bool saveFineMesh = false;
};
class QueryEngine {
public:
    // One query: every level through B200Strategy (the reference's makeForLevel, every level on the
    // device), returning the last level's grid (owned by the strategy's buffers) and, when asked,
    // the grid size of every level (levelFineMeshSize).
    static LevelResult runSingleQuery(QueryHandler& h, QueryType qType, const double* lo, const double* hi,
                                      const double* queryPoint, size_t K, size_t* levelFineMeshSize);
    // Every query of `q` one at a time (QueryEngine::run, src/core/QueryEngine.cu:109-252): per-query
    // microseconds, level sizes, result counts, the mean without the fastest and slowest query.
    static QueryResult run(QueryHandler& h, const Query& q, const RunConfig& cfg);
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
