// Hierarchical k-means index build on the device (the reference's IndexBuilder::build with cuVS
// k-means, src/core/IndexBuilder.cu:44-151 and src/Setup/Setup.cuh:87-171).
//
// Per level: Lloyd iterations (assign every point to its nearest centroid, then move each
// centroid to the mean of its points) from k = floor(n / ratio) centroids sampled from the data;
// the labels then become that interval's P-tensor (rows sorted stably by label, values
// fine / coarse), its sort-to-original map and its max radii, and the centroids become the next
// level's data, exactly as the reference assembles its index.
//
// The assignment is a distance GEMM with a per-point argmin, computed three ways:
//   * kTensor: tcgen05 tensor cores. ||x - c||^2 = ||x||^2 + ||c||^2 - 2 x.c, with x.c from TF32
//     operands split in two (v = hi + lo): x.c ~ xh.ch + xh.cl + xl.ch, six K=8 MMAs accumulated in
//     FP32 in tensor memory. A single BF16 or TF32 product cannot resolve the gaps between
//     neighbouring centroids of tight clusters (measured: a BF16 hi/lo split still mislabels 2.3%
//     of points); the TF32 split leaves ~2^-21 relative error. The epilogue adds ||c||^2 and keeps
//     the minimum.
//   * kFp32 / kFp64: plain CUDA-core loops in FP32 / FP64 (the FP64 build is the precision
//     reference the tensor build is compared against).
// Centroid sums accumulate in FP64; the reported objective sum ||x - c(x)||^2 is computed in FP64.
#pragma once

#include <cstdint>
#include <vector>

#include "common.cuh"
#include "device_index.hpp"
#include "index.hpp"

namespace tblaeq {

enum KmeansPrecision : int { kKmTensor = 0, kKmFp32 = 1, kKmFp64 = 2 };

enum AssemblyMode : int { kAssembleDevice = 0, kAssembleHost = 1, kAssembleBoth = 2 };

struct KmeansConfig {
    int iters = 20;
    uint64_t seed = 1;
    int precision = kKmTensor;
    // Where each interval (P-tensor, map, radii) is assembled: kAssembleDevice (labels and
    // centroids stay on the device), kAssembleHost (from downloaded labels and centroids, as the
    // reference does), or kAssembleBoth (device result, checked byte for byte against the host's
    // from the same labels and centroids; an error when they differ).
    int hostAssembly = 0;
};

struct KmeansLevelReport {
    uint64_t n = 0, k = 0;
    int iters = 0;
    double objective = 0.0;         // after the last update, FP64
    double assignSeconds = 0.0;     // device time of all assignment passes
    double assembleSeconds = 0.0;   // the index assembly of the level (grouping, P values, map, radii)
    double seconds = 0.0;           // the whole level (Lloyd + index assembly)
    std::vector<double> objectives; // after every iteration
};

// Lloyd's k-means on device-resident FP32 points (n x D). On return `centroids` (k x D, FP32)
// and `labels` (n) are device arrays owned by the caller's DeviceMem objects.
void kmeansRun(const float* dX, uint64_t n, uint64_t D, uint64_t k, const KmeansConfig& cfg, DeviceMem& centroids,
               DeviceMem& labels, KmeansLevelReport& report, cudaStream_t s);

// Builds the whole hierarchy from host FP32 points (N x D) with the reference's plan (height,
// ratios). Fills one report per interval, finest first.
HostIndex kmeansBuild(const float* hostPoints, uint64_t N, uint64_t D, uint64_t height,
                      const std::vector<uint64_t>& ratios, const KmeansConfig& cfg,
                      std::vector<KmeansLevelReport>& reports, cudaStream_t s);

// Whether the tensor-core assignment supports this dimension (D <= 16).
inline bool kmeansTensorSupports(uint64_t D) { return D >= 1 && D <= 16; }

}  // namespace tblaeq
