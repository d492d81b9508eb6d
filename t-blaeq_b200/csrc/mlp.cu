// Learned frontier scorer (see mlp.cuh): feature build, forward, backward and Adam kernels.
#include "mlp.cuh"

#include <cuda_bf16.h>

#include <cmath>
#include <random>

namespace tblaeq {

namespace {

constexpr int H = kMlpHidden;

struct Offsets {
    int in;
    size_t w1, b1, w2, b2, w3, b3, total;
};

Offsets offsetsOf(const MlpShape& s) {
    Offsets o;
    o.in = s.in();
    o.w1 = 0;
    o.b1 = o.w1 + static_cast<size_t>(o.in) * H;
    o.w2 = o.b1 + H;
    o.b2 = o.w2 + static_cast<size_t>(H) * H;
    o.w3 = o.b2 + H;
    o.b3 = o.w3 + H;
    o.total = o.b3 + 1;
    return o;
}

// Loads the BF16 parameters into shared memory as floats.
__device__ void loadWeights(const __nv_bfloat16* p, int n, float* s) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) s[i] = __bfloat162float(p[i]);
    __syncthreads();
}

// Forward pass of one sample in registers; returns the logit and (optionally) the activations.
template <bool KEEP>
__device__ float forwardOne(const float* x, int in, const float* w, float* h1out, float* h2out) {
    const float* W1 = w;
    const float* b1 = W1 + in * H;
    const float* W2 = b1 + H;
    const float* b2 = W2 + H * H;
    const float* w3 = b2 + H;
    const float b3 = w3[H];
    float h1[H];
#pragma unroll
    for (int j = 0; j < H; ++j) h1[j] = b1[j];
    for (int k = 0; k < in; ++k) {
        const float xk = x[k];
#pragma unroll
        for (int j = 0; j < H; ++j) h1[j] = fmaf(xk, W1[k * H + j], h1[j]);
    }
#pragma unroll
    for (int j = 0; j < H; ++j) {
        h1[j] = fmaxf(h1[j], 0.f);
        if (KEEP) h1out[j] = h1[j];
    }
    float z = b3;
#pragma unroll 4
    for (int j = 0; j < H; ++j) {
        float a = b2[j];
#pragma unroll
        for (int i = 0; i < H; ++i) a = fmaf(h1[i], W2[i * H + j], a);
        a = fmaxf(a, 0.f);
        if (KEEP) h2out[j] = a;
        z = fmaf(a, w3[j], z);
    }
    return z;
}

__global__ void featuresKernel(const double* points, const uint32_t* q, const double* centres, const double* radius,
                               uint32_t level, uint32_t n, int D, int levels, double inv, float* X) {
    const int in = 2 * D + 1 + levels;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float* x = X + static_cast<size_t>(i) * in;
        const double* p = points + static_cast<size_t>(q[i]) * D;
        const double* c = centres + static_cast<size_t>(i) * D;
        for (int d = 0; d < D; ++d) {
            x[d] = static_cast<float>(p[d] * inv);
            x[D + d] = static_cast<float>(c[d] * inv);
        }
        x[2 * D] = static_cast<float>(radius[i] * inv);
        for (int l = 0; l < levels; ++l) x[2 * D + 1 + l] = (l == static_cast<int>(level)) ? 1.f : 0.f;
    }
}

__global__ void logitsKernel(const __nv_bfloat16* p, int nParams, const float* X, uint32_t n, int in, float* z) {
    extern __shared__ float w[];
    loadWeights(p, nParams, w);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        z[i] = forwardOne<false>(X + static_cast<size_t>(i) * in, in, w, nullptr, nullptr);
}

// Per-sample forward + backward through the activations: writes dLogit, h1, h2 and the
// pre-activation gradients dh1, dh2 (zero where the ReLU was inactive), and the loss terms.
__global__ void sampleGradKernel(const __nv_bfloat16* p, int nParams, const float* X, const float* y, uint32_t n,
                                 int in, float* h1s, float* h2s, float* dh1s, float* dh2s, float* dz, float* lossTerm) {
    extern __shared__ float w[];
    loadWeights(p, nParams, w);
    const float* W2 = w + in * H + H;
    const float* w3 = W2 + H * H + H;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float* h1 = h1s + static_cast<size_t>(i) * H;
        float* h2 = h2s + static_cast<size_t>(i) * H;
        const float z = forwardOne<true>(X + static_cast<size_t>(i) * in, in, w, h1, h2);
        const float t = y[i];
        // Mean binary cross-entropy on logits: softplus(z) - t z; dL/dz = (sigmoid(z) - t) / n.
        const float sp = z > 0.f ? z + log1pf(expf(-z)) : log1pf(expf(z));
        lossTerm[i] = sp - t * z;
        const float g = (1.f / (1.f + expf(-z)) - t) / static_cast<float>(n);
        dz[i] = g;
        float* dh2 = dh2s + static_cast<size_t>(i) * H;
        for (int j = 0; j < H; ++j) dh2[j] = h2[j] > 0.f ? g * w3[j] : 0.f;
        float* dh1 = dh1s + static_cast<size_t>(i) * H;
        for (int k = 0; k < H; ++k) {
            float a = 0.f;
            if (h1[k] > 0.f) {
                for (int j = 0; j < H; ++j) a = fmaf(W2[k * H + j], dh2[j], a);
            }
            dh1[k] = a;
        }
    }
}

// Parameter gradients as sums over the batch: one thread per parameter.
__global__ void paramGradKernel(const float* X, const float* h1s, const float* h2s, const float* dh1s,
                                const float* dh2s, const float* dz, uint32_t n, int in, float* grad) {
    const size_t nW1 = static_cast<size_t>(in) * H;
    const size_t total = nW1 + H + H * H + H + H + 1;
    for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<size_t>(gridDim.x) * blockDim.x) {
        float acc = 0.f;
        if (t < nW1) {  // dW1[k][j] = sum x[k] dh1[j]
            const int k = static_cast<int>(t / H), j = static_cast<int>(t % H);
            for (uint32_t i = 0; i < n; ++i) acc = fmaf(X[static_cast<size_t>(i) * in + k], dh1s[static_cast<size_t>(i) * H + j], acc);
        } else if (t < nW1 + H) {  // db1
            const int j = static_cast<int>(t - nW1);
            for (uint32_t i = 0; i < n; ++i) acc += dh1s[static_cast<size_t>(i) * H + j];
        } else if (t < nW1 + H + H * H) {  // dW2[k][j] = sum h1[k] dh2[j]
            const size_t u = t - nW1 - H;
            const int k = static_cast<int>(u / H), j = static_cast<int>(u % H);
            for (uint32_t i = 0; i < n; ++i) acc = fmaf(h1s[static_cast<size_t>(i) * H + k], dh2s[static_cast<size_t>(i) * H + j], acc);
        } else if (t < nW1 + 2 * H + H * H) {  // db2
            const int j = static_cast<int>(t - nW1 - H - H * H);
            for (uint32_t i = 0; i < n; ++i) acc += dh2s[static_cast<size_t>(i) * H + j];
        } else if (t < nW1 + 3 * H + H * H) {  // dw3[j] = sum h2[j] dz
            const int j = static_cast<int>(t - nW1 - 2 * H - H * H);
            for (uint32_t i = 0; i < n; ++i) acc = fmaf(h2s[static_cast<size_t>(i) * H + j], dz[i], acc);
        } else {  // db3
            for (uint32_t i = 0; i < n; ++i) acc += dz[i];
        }
        grad[t] = acc;
    }
}

__global__ void sumKernel(const float* v, uint32_t n, float* out) {
    __shared__ float s[1024];
    float a = 0.f;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) a += v[i];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = s[0] / static_cast<float>(n);
}

__global__ void adamKernel(float* w, float* m, float* v, const float* g, size_t n, float lr, float b1, float b2,
                           float eps, float c1, float c2, __nv_bfloat16* wb) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        m[i] = b1 * m[i] + (1.f - b1) * gi;
        v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
        w[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
        wb[i] = __float2bfloat16(w[i]);
    }
}

__global__ void toBf16Kernel(const float* w, size_t n, __nv_bfloat16* wb) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        wb[i] = __float2bfloat16(w[i]);
}

// Scores the entries of a KNN frontier in place: features from the entry's centre, its query
// point and its subtree radius; score = -logit.
__global__ void scoreFrontierKernel(const __nv_bfloat16* p, int nParams, const uint32_t* q, const uint32_t* node,
                                    const double* x, const uint32_t* hdr, uint32_t cap, const double* points,
                                    const NodeRec* nodes, uint32_t level, int levels, int D, double inv,
                                    double* score) {
    extern __shared__ float w[];
    loadWeights(p, nParams, w);
    const int in = 2 * D + 1 + levels;
    const uint32_t n = min(hdr[0], cap);
    float feat[kMlpMaxIn];
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const double* pt = points + static_cast<size_t>(q[e]) * D;
        const double* c = x + static_cast<size_t>(e) * D;
        for (int d = 0; d < D; ++d) {
            feat[d] = static_cast<float>(pt[d] * inv);
            feat[D + d] = static_cast<float>(c[d] * inv);
        }
        feat[2 * D] = static_cast<float>(nodes[node[e]].rad * inv);
        for (int l = 0; l < levels; ++l) feat[2 * D + 1 + l] = (l == static_cast<int>(level)) ? 1.f : 0.f;
        score[e] = -static_cast<double>(forwardOne<false>(feat, in, w, nullptr, nullptr));
    }
}

__global__ void frontierFeaturesKernel(const uint32_t* q, const uint32_t* node, const double* x, const uint32_t* idx,
                                       uint32_t n, const double* points, const NodeRec* nodes, uint32_t level,
                                       int levels, int D, double inv, float* X) {
    const int in = 2 * D + 1 + levels;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t e = idx[i];
        float* f = X + static_cast<size_t>(i) * in;
        const double* pt = points + static_cast<size_t>(q[e]) * D;
        const double* c = x + static_cast<size_t>(e) * D;
        for (int d = 0; d < D; ++d) {
            f[d] = static_cast<float>(pt[d] * inv);
            f[D + d] = static_cast<float>(c[d] * inv);
        }
        f[2 * D] = static_cast<float>(nodes[node[e]].rad * inv);
        for (int l = 0; l < levels; ++l) f[2 * D + 1 + l] = (l == static_cast<int>(level)) ? 1.f : 0.f;
    }
}

int gridFor(size_t n, int t) { return static_cast<int>(std::max<size_t>(1, std::min<size_t>((n + t - 1) / t, 148 * 8))); }

}  // namespace

Mlp::Mlp(MlpShape shape) : shape_(shape) {
    if (shape.in() > kMlpMaxIn) throw std::invalid_argument("scorer input wider than 64 features");
    const size_t n = shape.params();
    master_.alloc(n * 4);
    bf16_.alloc(n * 2);
    adamM_.alloc(n * 4);
    adamV_.alloc(n * 4);
}

void Mlp::refreshBf16(cudaStream_t s) {
    const size_t n = shape_.params();
    toBf16Kernel<<<gridFor(n, 256), 256, 0, s>>>(master_.as<float>(), n, bf16_.as<__nv_bfloat16>());
    TBLAEQ_CUDA(cudaGetLastError());
}

std::vector<float> Mlp::getParams() const {
    std::vector<float> p(shape_.params());
    TBLAEQ_CUDA(cudaMemcpy(p.data(), master_.get(), p.size() * 4, cudaMemcpyDeviceToHost));
    return p;
}

void Mlp::setParams(const std::vector<float>& p, cudaStream_t s) {
    if (p.size() != shape_.params()) throw std::invalid_argument("scorer parameter count mismatch");
    TBLAEQ_CUDA(cudaMemcpyAsync(master_.get(), p.data(), p.size() * 4, cudaMemcpyHostToDevice, s));
    TBLAEQ_CUDA(cudaMemsetAsync(adamM_.get(), 0, p.size() * 4, s));
    TBLAEQ_CUDA(cudaMemsetAsync(adamV_.get(), 0, p.size() * 4, s));
    step_ = 0;
    refreshBf16(s);
    TBLAEQ_CUDA(cudaStreamSynchronize(s));
}

void Mlp::initRandom(uint64_t seed, cudaStream_t s) {
    const Offsets o = offsetsOf(shape_);
    std::vector<float> p(o.total, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](size_t off, int fanIn, size_t n) {
        std::normal_distribution<float> nd(0.f, std::sqrt(2.f / static_cast<float>(fanIn)));
        for (size_t i = 0; i < n; ++i) p[off + i] = nd(rng);
    };
    fill(o.w1, o.in, static_cast<size_t>(o.in) * H);
    fill(o.w2, H, static_cast<size_t>(H) * H);
    fill(o.w3, H, H);
    setParams(p, s);
}

void Mlp::buildFeatures(const double* points, const uint32_t* q, const double* centres, const double* radius,
                        uint32_t level, uint32_t n, double invScale, float* X, cudaStream_t s) const {
    if (n == 0) return;
    featuresKernel<<<gridFor(n, 256), 256, 0, s>>>(points, q, centres, radius, level, n, shape_.D, shape_.levels,
                                                   invScale, X);
    TBLAEQ_CUDA(cudaGetLastError());
}

float Mlp::lossAndGrad(const float* X, const float* y, uint32_t n, float* grad, cudaStream_t s) {
    const Offsets o = offsetsOf(shape_);
    const size_t need = static_cast<size_t>(n) * (4 * H + 2) + 1;
    if (workCap_ < need) {
        work_.alloc(need * 4);
        workCap_ = need;
    }
    float* h1 = work_.as<float>();
    float* h2 = h1 + static_cast<size_t>(n) * H;
    float* dh1 = h2 + static_cast<size_t>(n) * H;
    float* dh2 = dh1 + static_cast<size_t>(n) * H;
    float* dz = dh2 + static_cast<size_t>(n) * H;
    float* lt = dz + n;
    float* loss = lt + n;
    const size_t smem = o.total * 4;
    TBLAEQ_CUDA(cudaFuncSetAttribute(sampleGradKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    sampleGradKernel<<<gridFor(n, 128), 128, smem, s>>>(bf16_.as<__nv_bfloat16>(), static_cast<int>(o.total), X, y, n,
                                                       o.in, h1, h2, dh1, dh2, dz, lt);
    TBLAEQ_CUDA(cudaGetLastError());
    paramGradKernel<<<gridFor(o.total, 128), 128, 0, s>>>(X, h1, h2, dh1, dh2, dz, n, o.in, grad);
    TBLAEQ_CUDA(cudaGetLastError());
    sumKernel<<<1, 1024, 0, s>>>(lt, n, loss);
    TBLAEQ_CUDA(cudaGetLastError());
    float hl = 0.f;
    TBLAEQ_CUDA(cudaMemcpyAsync(&hl, loss, 4, cudaMemcpyDeviceToHost, s));
    TBLAEQ_CUDA(cudaStreamSynchronize(s));
    return hl;
}

void Mlp::adamStep(const float* grad, float lr, cudaStream_t s) {
    ++step_;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, static_cast<float>(step_));
    const float c2 = 1.f - std::pow(b2, static_cast<float>(step_));
    const size_t n = shape_.params();
    adamKernel<<<gridFor(n, 256), 256, 0, s>>>(master_.as<float>(), adamM_.as<float>(), adamV_.as<float>(), grad, n, lr,
                                               b1, b2, 1e-8f, c1, c2, bf16_.as<__nv_bfloat16>());
    TBLAEQ_CUDA(cudaGetLastError());
}

void Mlp::logits(const float* X, uint32_t n, float* z, cudaStream_t s) const {
    if (n == 0) return;
    const Offsets o = offsetsOf(shape_);
    const size_t smem = o.total * 4;
    TBLAEQ_CUDA(cudaFuncSetAttribute(logitsKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    logitsKernel<<<gridFor(n, 128), 128, smem, s>>>(bf16_.as<__nv_bfloat16>(), static_cast<int>(o.total), X, n, o.in, z);
    TBLAEQ_CUDA(cudaGetLastError());
}

void Mlp::frontierFeatures(const FrontierIn& f, const uint32_t* node, const uint32_t* idx, uint32_t n,
                           const double* points, const NodeRec* nodes, uint32_t level, double invScale, float* X,
                           cudaStream_t s) const {
    if (n == 0) return;
    frontierFeaturesKernel<<<gridFor(n, 256), 256, 0, s>>>(f.q, node, f.x, idx, n, points, nodes, level, shape_.levels,
                                                           shape_.D, invScale, X);
    TBLAEQ_CUDA(cudaGetLastError());
}

void Mlp::scoreFrontier(const FrontierIn& f, const uint32_t* node, uint32_t cap, const double* points,
                        const NodeRec* nodes, uint32_t level, double invScale, double* score, cudaStream_t s) const {
    const Offsets o = offsetsOf(shape_);
    const size_t smem = o.total * 4;
    TBLAEQ_CUDA(cudaFuncSetAttribute(scoreFrontierKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
    scoreFrontierKernel<<<148 * 2, 128, smem, s>>>(bf16_.as<__nv_bfloat16>(), static_cast<int>(o.total), f.q, node,
                                                  f.x, f.hdr, cap, points, nodes, level, shape_.levels, shape_.D,
                                                  invScale, score);
    TBLAEQ_CUDA(cudaGetLastError());
}

}  // namespace tblaeq
