// Training and use of the learned frontier scorer (see scorer.hpp).
#include "scorer.hpp"

#include <algorithm>
#include <numeric>
#include <random>

namespace tblaeq {

namespace {

// Labels the final-frontier entries of a KNN batch: label[e] = 1 when the cluster of entry e holds
// one of its query's result points. Results and entries are both query-major.
__global__ void labelFrontierKernel(const uint64_t* resOff, const uint64_t* resIds, const uint64_t* fOff,
                                    const uint32_t* fNode, const uint32_t* invMap, const uint32_t* parent, uint32_t nq,
                                    uint8_t* label) {
    for (uint32_t q = blockIdx.x; q < nq; q += gridDim.x) {
        for (uint64_t r = resOff[q] + threadIdx.x; r < resOff[q + 1]; r += blockDim.x) {
            const uint32_t cluster = parent[invMap[resIds[r]]];
            for (uint64_t e = fOff[q]; e < fOff[q + 1]; ++e)
                if (fNode[e] == cluster) label[e] = 1;
        }
    }
}

__global__ void gatherLabelsKernel(const uint8_t* label, const uint32_t* idx, uint32_t n, float* y) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = label[idx[i]] ? 1.f : 0.f;
}

__global__ void permuteKernel(const float* X, const float* y, const uint32_t* perm, uint32_t n, int in, float* Xo,
                              float* yo) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t s = perm[i];
        for (int k = 0; k < in; ++k) Xo[static_cast<size_t>(i) * in + k] = X[static_cast<size_t>(s) * in + k];
        yo[i] = y[s];
    }
}

void scorerHook(void* ctx, const FrontierIn& f, const uint32_t* node, uint32_t cap, const double* points,
                double* score, cudaStream_t s) {
    auto* rt = static_cast<Runtime*>(ctx);
    const uint32_t level = static_cast<uint32_t>(rt->dev->height - 2);
    rt->scorer->scoreFrontier(f, node, cap, points, rt->dev->nodeSub[level].as<NodeRec>(), level, rt->scorerInvScale,
                              score, s);
}

// Device arrays that map a point id to its cluster in the finest cluster mesh (for labels).
void ensureLabelMaps(Runtime& rt) {
    if (rt.invMapFinest.bytes()) return;
    const HostIndex& h = *rt.host;
    const uint64_t H = h.height, N = h.meshCount(H - 1), nc = h.meshCount(H - 2);
    std::vector<uint32_t> inv(N), parent(N);
    for (uint64_t s = 0; s < N; ++s) inv[h.maps[H - 1][s]] = static_cast<uint32_t>(s);
    const PTensor& P = h.pTensors[H - 2];
    for (uint64_t c = 0; c < nc; ++c) {
        const uint64_t o = (H - 2 == 0) ? h.coarsest.ids[c] : h.maps[H - 2][c];
        for (uint64_t j = P.colRes[o]; j < P.colRes[o + 1]; ++j) parent[j] = static_cast<uint32_t>(c);
    }
    rt.invMapFinest = upload(inv, rt.stream);
    rt.parentFinest = upload(parent, rt.stream);
    TBLAEQ_CUDA(cudaStreamSynchronize(rt.stream));
}

}  // namespace

Mlp& ensureScorer(Runtime& rt) {
    if (!rt.scorer) {
        MlpShape shape;
        shape.D = static_cast<int>(rt.dev->D);
        shape.levels = static_cast<int>(rt.dev->height - 1);
        rt.scorer = std::make_unique<Mlp>(shape);
        rt.scorer->initRandom(1, rt.stream);
        // Scale: 1 / largest extent of the coarsest mesh (the data's bounding box, up to the spread).
        const HostIndex& h = *rt.host;
        double lo = 1e300, hi = -1e300;
        for (double v : h.coarsest.vals) {
            lo = std::min(lo, v);
            hi = std::max(hi, v);
        }
        rt.scorerInvScale = (hi > lo) ? 1.0 / (hi - lo) : 1.0;
    }
    return *rt.scorer;
}

bool scorerTrained(const Runtime& rt) { return rt.scorer && rt.scorerSamples > 0; }

void attachScorer(Runtime& rt, BatchEngine& engine) { engine.setScorer(&scorerHook, &rt); }

void enableScorer(Runtime& rt, bool on) {
    if (on) {
        ensureScorer(rt);
        rt.engine->setScorer(&scorerHook, &rt);
    } else {
        rt.engine->setScorer(nullptr, nullptr);
    }
}

std::vector<float> trainScorer(Runtime& rt, const double* hostPoints, uint32_t nq, const std::vector<uint32_t>& K,
                               const ScorerTrainConfig& cfg) {
    Mlp& mlp = ensureScorer(rt);
    ensureLabelMaps(rt);
    const int D = static_cast<int>(rt.dev->D);
    const uint32_t level = static_cast<uint32_t>(rt.dev->height - 2);
    cudaStream_t s = rt.stream;
    BatchEngine& eng = *rt.engine;
    const int in = mlp.shape().in();

    // Traces: plain two-wave KNN (lower-bound ranking) over the training queries, in chunks small
    // enough for one traversal each. Every chunk contributes all its positives and its share of
    // random negatives; the union is subsampled to maxSamples at the end.
    DeviceMem dPoints(std::max<size_t>(nq, 1) * D * 8), dK(std::max<size_t>(nq, 1) * 4);
    TBLAEQ_CUDA(cudaMemcpyAsync(dPoints.get(), hostPoints, static_cast<size_t>(nq) * D * 8, cudaMemcpyHostToDevice, s));
    TBLAEQ_CUDA(cudaMemcpyAsync(dK.get(), K.data(), static_cast<size_t>(nq) * 4, cudaMemcpyHostToDevice, s));
    eng.setScorer(nullptr, nullptr);  // traces come from the lower-bound ranking
    const bool wasTwoWave = eng.twoWave();
    eng.setTwoWave(true);
    std::mt19937_64 rng(cfg.seed);
    std::vector<float> hostX, hostY;
    uint64_t positives = 0;
    uint32_t chunk = nq, i = 0;
    while (i < nq) {
        const uint32_t c = std::min(chunk, nq - i);
        uint64_t sumK = 0;
        for (uint32_t q = i; q < i + c; ++q) sumK += K[q];
        const double* pts = dPoints.as<double>() + static_cast<size_t>(i) * D;
        BatchOutput res;
        try {
            res = eng.runKnn(pts, c, dK.as<uint32_t>() + i, sumK, 0);
        } catch (const SplitBatch&) {
            if (c == 1) {
                eng.setTwoWave(wasTwoWave);
                throw;
            }
            chunk = (c + 1) / 2;
            continue;
        }
        const BatchEngine::FrontierView fv = eng.lastKnnFrontier();
        uint32_t fCount = 0;
        TBLAEQ_CUDA(cudaMemcpyAsync(&fCount, fv.in.hdr, 4, cudaMemcpyDeviceToHost, s));
        TBLAEQ_CUDA(cudaStreamSynchronize(s));
        fCount = std::min(fCount, fv.cap);
        if (fCount > 0) {
            DeviceMem label(fCount);
            TBLAEQ_CUDA(cudaMemsetAsync(label.get(), 0, fCount, s));
            labelFrontierKernel<<<std::min<uint32_t>(c, 4096), 128, 0, s>>>(
                res.offsets, res.ids, fv.offsets, fv.node, rt.invMapFinest.as<uint32_t>(),
                rt.parentFinest.as<uint32_t>(), c, label.as<uint8_t>());
            TBLAEQ_LAUNCHED();
            std::vector<uint8_t> hl(fCount);
            TBLAEQ_CUDA(cudaMemcpyAsync(hl.data(), label.get(), fCount, cudaMemcpyDeviceToHost, s));
            TBLAEQ_CUDA(cudaStreamSynchronize(s));
            std::vector<uint32_t> pos, neg;
            for (uint32_t e = 0; e < fCount; ++e) (hl[e] ? pos : neg).push_back(e);
            std::shuffle(neg.begin(), neg.end(), rng);
            const uint64_t quota = (static_cast<uint64_t>(cfg.maxSamples) * c + nq - 1) / nq;
            std::vector<uint32_t> idx = pos;
            if (quota > idx.size()) idx.insert(idx.end(), neg.begin(), neg.begin() + std::min<size_t>(quota - idx.size(), neg.size()));
            positives += pos.size();
            const uint32_t n = static_cast<uint32_t>(idx.size());
            DeviceMem dIdx = upload(idx, s), X(static_cast<size_t>(std::max<uint32_t>(n, 1)) * in * 4),
                      y(static_cast<size_t>(std::max<uint32_t>(n, 1)) * 4);
            mlp.frontierFeatures(fv.in, fv.node, dIdx.as<uint32_t>(), n, pts, rt.dev->nodeSub[level].as<NodeRec>(), level,
                                 rt.scorerInvScale, X.as<float>(), s);
            gatherLabelsKernel<<<148, 256, 0, s>>>(label.as<uint8_t>(), dIdx.as<uint32_t>(), n, y.as<float>());
            TBLAEQ_LAUNCHED();
            const size_t x0 = hostX.size(), y0 = hostY.size();
            hostX.resize(x0 + static_cast<size_t>(n) * in);
            hostY.resize(y0 + n);
            TBLAEQ_CUDA(cudaMemcpyAsync(hostX.data() + x0, X.get(), static_cast<size_t>(n) * in * 4,
                                        cudaMemcpyDeviceToHost, s));
            TBLAEQ_CUDA(cudaMemcpyAsync(hostY.data() + y0, y.get(), static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost, s));
            TBLAEQ_CUDA(cudaStreamSynchronize(s));
        }
        i += c;
    }
    eng.setTwoWave(wasTwoWave);
    if (hostY.empty()) throw std::runtime_error("scorer training: the traversal left no clusters to learn from");
    // Subsample the union to maxSamples (keeping the sample order random either way).
    std::vector<uint32_t> keep(hostY.size());
    std::iota(keep.begin(), keep.end(), 0u);
    std::shuffle(keep.begin(), keep.end(), rng);
    if (keep.size() > cfg.maxSamples) keep.resize(cfg.maxSamples);
    const uint32_t n = static_cast<uint32_t>(keep.size());
    std::vector<float> sx(static_cast<size_t>(n) * in), sy(n);
    for (uint32_t t = 0; t < n; ++t) {
        std::copy_n(hostX.data() + static_cast<size_t>(keep[t]) * in, in, sx.data() + static_cast<size_t>(t) * in);
        sy[t] = hostY[keep[t]];
    }
    DeviceMem X = upload(sx, s), y = upload(sy, s);

    // Adam over shuffled mini-batches.
    DeviceMem Xp(static_cast<size_t>(n) * in * 4), yp(static_cast<size_t>(n) * 4), grad(mlp.shape().params() * 4);
    std::vector<uint32_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0u);
    std::vector<float> losses;
    for (int ep = 0; ep < cfg.epochs; ++ep) {
        std::shuffle(perm.begin(), perm.end(), rng);
        DeviceMem dPerm = upload(perm, s);
        permuteKernel<<<148 * 2, 256, 0, s>>>(X.as<float>(), y.as<float>(), dPerm.as<uint32_t>(), n, in, Xp.as<float>(),
                                              yp.as<float>());
        TBLAEQ_LAUNCHED();
        double sum = 0.0;
        int batches = 0;
        for (uint32_t b = 0; b < n; b += cfg.batch) {
            const uint32_t m = std::min(cfg.batch, n - b);
            sum += mlp.lossAndGrad(Xp.as<float>() + static_cast<size_t>(b) * in, yp.as<float>() + b, m,
                                   grad.as<float>(), s);
            mlp.adamStep(grad.as<float>(), cfg.lr, s);
            ++batches;
        }
        losses.push_back(static_cast<float>(sum / std::max(1, batches)));
    }
    TBLAEQ_CUDA(cudaStreamSynchronize(s));
    rt.scorerPositives = positives;
    rt.scorerSamples = n;
    return losses;
}

}  // namespace tblaeq
