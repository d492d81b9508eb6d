// Host-side index container, on-disk layout and synthetic index generator.
//
// The container holds exactly what the reference's IndexData holds on the host
// (src/core/IndexData.cuh:89-110) in flat, aligned arrays:
//   * one CSC P-tensor per interval l (0 = coarsest interval): rows are the fine mesh nodes in
//     "sorted position" order, columns are the coarse mesh nodes by original id, and row j's
//     value is the D-vector of ratios fine[d] / coarse[d];
//   * one max-radius array per interval (indexed by coarse original id);
//   * one sort-to-original map per non-coarsest mesh (Map_m[s] = original id of sorted node s);
//   * the coarsest mesh (ids + AOS coordinates).
// Mesh sizes are kept finest -> coarsest like the reference (meshSizes[0] = N).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace tblaeq {

struct PTensor {
    uint64_t D = 0, rows = 0, cols = 0, nnz = 0;
    uint8_t isAos = 1;
    std::vector<uint64_t> rowIds;     // nnz (always iota for indexes built by the reference)
    std::vector<uint64_t> nnzPerCol;  // cols
    std::vector<uint64_t> colRes;     // cols + 1
    std::vector<double> vals;         // nnz * D, AOS
};

struct CoarsestMesh {
    uint64_t rows = 0, dim = 0, nnz = 0;
    uint8_t isAos = 1;
    std::vector<uint64_t> ids;   // nnz
    std::vector<double> vals;    // nnz * dim
};

struct HostIndex {
    uint64_t D = 0, N = 0, height = 0, intervals = 0;
    uint8_t isAos = 1;
    std::vector<uint64_t> ratios;               // intervals
    std::vector<uint64_t> meshSizes;            // height, finest -> coarsest
    std::vector<PTensor> pTensors;              // intervals, [0] = coarsest interval
    std::vector<std::vector<double>> radius;    // intervals, radius[l][coarse original id]
    std::vector<std::vector<uint64_t>> maps;    // height, maps[0] empty; maps[m] for mesh m >= 1
    CoarsestMesh coarsest;
    std::string datasetName;

    // Number of nodes of mesh m, m = 0 (coarsest) .. height-1 (finest points).
    uint64_t meshCount(uint64_t m) const { return meshSizes[intervals - m]; }

    // Validates internal consistency; throws std::runtime_error with a description on failure.
    void validate() const;
};

// IndexSerializer equivalents (src/core/IndexSerializer.cu:11-67). The byte layout of every
// file is identical to the reference's: metadata.bin, P_Tensor_{l}.bin, MaxRadius_{l}.bin,
// Map_{m}.bin and Coreast_Mesh.bin (sic). Errors throw std::runtime_error.
void saveIndex(const HostIndex& idx, const std::string& dir);
HostIndex loadIndex(const std::string& dir);

// Dataset text file (src/Data_Structures/File.cu:8-50): a header "N D" (both > 0), then N rows of
// whitespace-separated values; a row must hold at least D values (the rest of the row is ignored)
// and lines after row N are not read. Only the header is read when `points` is null; otherwise the
// rows are parsed into points (N * D values). Errors throw std::runtime_error with the reference's
// messages.
void loadPointsText(const std::string& path, uint64_t& n, uint64_t& d, std::vector<double>* points);

// Parameters of the synthetic RandomKmeans-style hierarchy
// (src/core/QueryHandler.cu:101-124 -> src/core/IndexBuilder.cu:153-234).
struct GenParams {
    uint64_t N = 1000000;
    uint64_t D = 3;
    double valMin = 1.0;
    double valMax = 100.0;
    bool isInt = false;
    uint64_t height = 4;
    std::vector<uint64_t> ratios{100, 50, 20};
    uint64_t seed = 12345;
    double sigmaDivisor = 3.0;
};

// Generates the same index, byte for byte, as the reference's `--gen-index`: the build plan is
// truncated like QueryHandler's adjustBuildPlan (src/core/QueryHandler.cu:23-45), the points come
// from one std::mt19937_64 stream (uniform coarsest mesh, then one fresh normal distribution per
// finer mesh, children assigned round-robin to parents, clamped), the sort-to-original maps come
// from std::sort over the labels, P values are fine/coarse ratios and radii are the largest
// distance from a centroid to its direct children (src/Setup/Setup.cuh:87-171).
HostIndex generateRandomIndex(const GenParams& p);

}  // namespace tblaeq
