// Learned frontier scorer: a small MLP that ranks the clusters of the last KNN frontier so the
// two-wave finest level expands the clusters most likely to hold true neighbours first (a tighter
// bound sooner). Exactness never depends on it: every result still passes the bound-based pruning.
//
//   input  x = query coords (D) || cluster centre (D) || cluster radius (1) || level one-hot (H-1),
//          coordinates and radius scaled by 1 / extent of the data
//   h1 = relu(W1^T x + b1)   (64)        W1: in x 64
//   h2 = relu(W2^T h1 + b2)  (64)        W2: 64 x 64
//   z  = w3 . h2 + b3                    logit of "the cluster holds one of the query's K nearest"
//
// Weights are kept as an FP32 master copy for training and a BF16 copy used by every forward pass
// (training and inference); accumulation is FP32. Training runs on CUDA cores; frontier inference
// runs on the tcgen05 tensor cores.
#pragma once

#include <cstdint>
#include <vector>

#include "common.cuh"
#include "device_index.hpp"
#include "traverse.cuh"

namespace tblaeq {

constexpr int kMlpHidden = 64;
constexpr int kMlpMaxIn = 64;

struct MlpShape {
    int D = 0;
    int levels = 0;  // one-hot width (height - 1)
    int in() const { return 2 * D + 1 + levels; }
    // Parameter layout (floats): W1[in][64] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3
    size_t params() const { return static_cast<size_t>(in()) * kMlpHidden + kMlpHidden + kMlpHidden * kMlpHidden +
                                   kMlpHidden + kMlpHidden + 1; }
};

class Mlp {
public:
    explicit Mlp(MlpShape shape);
    const MlpShape& shape() const { return shape_; }

    // Host parameter vector (FP32 master) in the layout above.
    std::vector<float> getParams() const;
    void setParams(const std::vector<float>& p, cudaStream_t s);
    void initRandom(uint64_t seed, cudaStream_t s);

    // Features of n (query point, cluster) samples on the device: X[n][in].
    void buildFeatures(const double* points, const uint32_t* q, const double* centres, const double* radius,
                       uint32_t level, uint32_t n, double invScale, float* X, cudaStream_t s) const;

    // Loss (mean binary cross-entropy on logits) and gradients (same layout as the parameters) of a
    // batch, using the BF16 weights. Returns the loss; grad is a device array of params() floats.
    float lossAndGrad(const float* X, const float* y, uint32_t n, float* grad, cudaStream_t s);

    // One Adam step on the master weights with the gradient from lossAndGrad; refreshes BF16 copy.
    void adamStep(const float* grad, float lr, cudaStream_t s);

    // Logits of n samples.
    void logits(const float* X, uint32_t n, float* z, cudaStream_t s) const;

    // Features of the frontier entries listed in idx (n of them) into X[n][in].
    void frontierFeatures(const FrontierIn& f, const uint32_t* node, const uint32_t* idx, uint32_t n,
                          const double* points, const NodeRec* nodes, uint32_t level, double invScale, float* X,
                          cudaStream_t s) const;

    // Scores the entries of a KNN frontier on the tensor cores: score[e] = -logit (ascending order =
    // most promising). Features are built in the kernel; both layers are tcgen05 BF16 MMAs with FP32
    // accumulation in tensor memory, so h1 is rounded to BF16 between the layers.
    void scoreFrontier(const FrontierIn& f, const uint32_t* node, uint32_t cap, const double* points,
                       const NodeRec* nodes, uint32_t level, double invScale, double* score, cudaStream_t s) const;

    // Logits of n samples through the same tensor-core kernel as scoreFrontier.
    void logitsTensor(const float* X, uint32_t n, float* z, cudaStream_t s) const;

    // Nonzero once a tensor-core launch gave up waiting for its MMAs (sticky; never expected).
    // A frontier scored by such a launch only changes the expansion order, never a result.
    uint32_t tensorStatus(cudaStream_t s) const;

private:
    MlpShape shape_;
    DeviceMem master_, bf16_, adamM_, adamV_, work_, tcStatus_;
    size_t workCap_ = 0;
    int step_ = 0;
    void refreshBf16(cudaStream_t s);
    void launchTc(bool frontier, const void* src, const uint32_t* hdr, uint32_t n, uint32_t cap, void* out,
                  cudaStream_t s) const;
};

}  // namespace tblaeq
