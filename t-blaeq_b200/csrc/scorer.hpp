// Training and use of the learned frontier scorer on a prepared index.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "handler.hpp"
#include "mlp.cuh"

namespace tblaeq {

struct ScorerTrainConfig {
    uint64_t maxSamples = 200000;  // (query, cluster) examples taken from the traversal traces
    int epochs = 8;
    float lr = 3e-3f;
    uint32_t batch = 1024;
    uint64_t seed = 1;
};

// Creates (or returns) the handle's scorer with the right shape.
Mlp& ensureScorer(Runtime& rt);

// Runs exact KNN on the training queries, labels every cluster of the final frontier by whether it
// holds one of the query's true K nearest points, and trains the scorer with Adam on a sample of
// those traces. Returns the mean training loss of every epoch.
std::vector<float> trainScorer(Runtime& rt, const double* hostPoints, uint32_t nq, const std::vector<uint32_t>& K,
                               const ScorerTrainConfig& cfg);

// Turns the scorer on or off for the two-wave ranking of KNN batches.
void enableScorer(Runtime& rt, bool on);

// Whether the handle has a trained scorer, and hooking it into another engine (serving lanes).
bool scorerTrained(const Runtime& rt);
void attachScorer(Runtime& rt, BatchEngine& engine);

}  // namespace tblaeq
