// Learned frontier scorer (see mlp.cuh): feature build, forward, backward and Adam kernels.
#include "mlp.cuh"
#include "tcgen05.cuh"

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

// ---- tensor-core forward (tcgen05, BF16 operands, FP32 accumulation in tensor memory) ----------
//
// One CTA of 128 threads takes 128 samples at a time: thread r builds sample r's features into a
// BF16 K-major operand image, one thread issues layer 1 (M=128, N=64, K=16 per MMA) into tensor
// memory columns 0-63, every thread reads its row back, applies bias + ReLU and writes BF16 h1 into
// a second image, layer 2 lands in columns 64-127, and the epilogue finishes ReLU, the w3 dot
// product and the logit. The weights' BF16 images stay in shared memory for the CTA's lifetime.
constexpr int kTcRows = 128;
constexpr uint32_t kTcCols = 128;
constexpr uint32_t kTcSpin = 1u << 22;
constexpr uint32_t kTcIdesc = tc::instrDesc(tc::kFmtBf16, kTcRows, H);
// Shared memory requested per CTA: at most four CTAs share an SM, so their 4 x 128 tensor-memory
// columns always fit and an allocation never waits.
constexpr size_t kTcSmemRequest = 54 * 1024;
constexpr int kTcCtasPerSm = 4;

// Byte offset of (row r, column k) in a K-major, non-swizzled BF16 image with K columns: 8-row x
// 16-byte core matrices (8 values per row), K-adjacent core matrices 128 B apart, 8-row groups
// K * 16 B apart. One K=16 MMA reads two core matrices; the next K slice starts 256 B further.
__host__ __device__ constexpr uint32_t bf16Offset(uint32_t r, uint32_t k, uint32_t K) {
    return (r >> 3) * (K / 8u) * 128u + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

struct TcLayout {
    uint32_t kp = 0;  // input width rounded up to 16
    uint32_t w1 = 0, w2 = 0, f = 0, h = 0, b1 = 0, b2 = 0, w3 = 0, bar = 0, tmem = 0, end = 0;  // byte offsets
    __host__ __device__ constexpr explicit TcLayout(int in) {
        kp = (static_cast<uint32_t>(in) + 15u) & ~15u;
        w1 = 0;                             // B of layer 1: 64 rows (hidden unit) x kp (input)
        w2 = w1 + 64u * kp * 2u;            // B of layer 2: 64 x 64
        f = w2 + 64u * 64u * 2u;            // A of layer 1: 128 samples x kp
        h = f + 128u * kp * 2u;             // A of layer 2: 128 samples x 64
        b1 = h + 128u * 64u * 2u;           // FP32 b1[64], b2[64], w3[64], b3
        b2 = b1 + 256u;
        w3 = b2 + 256u;
        bar = (w3 + 260u + 7u) & ~7u;
        tmem = bar + 8u;
        end = tmem + 4u;
    }
};
static_assert(TcLayout(kMlpMaxIn).end <= kTcSmemRequest, "scorer tile layout exceeds its shared memory");

// Eight consecutive values packed as BF16 into one 16-byte core-matrix row.
__device__ __forceinline__ uint4 packBf16x8(const float (&v)[8]) {
    uint4 u;
    uint32_t* w = reinterpret_cast<uint32_t*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const __nv_bfloat162 b = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
        w[i] = *reinterpret_cast<const uint32_t*>(&b);
    }
    return u;
}

struct FeatureSrc {
    // Frontier features: query point, cluster centre, subtree radius, level one-hot.
    const uint32_t* q;
    const uint32_t* node;
    const double* x;
    const double* points;
    const NodeRec* nodes;
    uint32_t level;
    double inv;
    // Plain features: X[n][in].
    const float* X;
};

// Feature k (< in) of frontier entry e, as frontierFeaturesKernel builds it.
__device__ __forceinline__ float frontierFeature(const FeatureSrc& s, uint32_t e, int k, int D) {
    if (k < D) return static_cast<float>(s.points[static_cast<size_t>(s.q[e]) * D + k] * s.inv);
    if (k < 2 * D) return static_cast<float>(s.x[static_cast<size_t>(e) * D + (k - D)] * s.inv);
    if (k == 2 * D) return static_cast<float>(s.nodes[s.node[e]].rad * s.inv);
    return (k - 2 * D - 1 == static_cast<int>(s.level)) ? 1.f : 0.f;
}

// FRONTIER: n = min(hdr[0], cap) frontier entries, out = score (double, -logit).
// Plain:    n samples of X[n][in], out = logit (float).
template <bool FRONTIER>
__global__ void __launch_bounds__(kTcRows) forwardTcKernel(const __nv_bfloat16* p, int D, int levels,
                                                          FeatureSrc src, const uint32_t* hdr, uint32_t nPlain,
                                                          uint32_t cap, void* out, uint32_t* status) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const int in = 2 * D + 1 + levels;
    const TcLayout L(in);
    const uint32_t n = FRONTIER ? min(hdr[0], cap) : nPlain;
    if (static_cast<uint64_t>(blockIdx.x) * kTcRows >= n) return;
    const int tid = threadIdx.x, warp = tid >> 5;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L.bar);
    uint32_t* sTmem = reinterpret_cast<uint32_t*>(smem + L.tmem);
    float* b1 = reinterpret_cast<float*>(smem + L.b1);
    float* b2 = reinterpret_cast<float*>(smem + L.b2);
    float* w3 = reinterpret_cast<float*>(smem + L.w3);

    // Weights: B images hold W^T (row = hidden unit j, column = input k), zero past `in`.
    const size_t oB1 = static_cast<size_t>(in) * H, oW2 = oB1 + H, oB2 = oW2 + H * H, oW3 = oB2 + H;
    for (uint32_t i = tid; i < 64u * L.kp; i += blockDim.x) {
        const uint32_t j = i / L.kp, k = i % L.kp;
        *reinterpret_cast<__nv_bfloat16*>(smem + L.w1 + bf16Offset(j, k, L.kp)) =
            k < static_cast<uint32_t>(in) ? p[static_cast<size_t>(k) * H + j] : __float2bfloat16(0.f);
    }
    for (uint32_t i = tid; i < 64u * 64u; i += blockDim.x) {
        const uint32_t j = i / 64u, k = i % 64u;
        *reinterpret_cast<__nv_bfloat16*>(smem + L.w2 + bf16Offset(j, k, 64)) = p[oW2 + static_cast<size_t>(k) * H + j];
    }
    for (int j = tid; j < H; j += blockDim.x) {
        b1[j] = __bfloat162float(p[oB1 + j]);
        b2[j] = __bfloat162float(p[oB2 + j]);
        w3[j] = __bfloat162float(p[oW3 + j]);
    }
    if (tid == 0) {
        w3[H] = __bfloat162float(p[oW3 + H]);
        tc::mbarInit(bar, 1);
        tc::mbarInitFence();
    }
    if (warp == 0) tc::tmemAlloc(sTmem, kTcCols);
    tc::fenceProxyAsync();
    tc::tcFenceBefore();
    __syncthreads();
    tc::tcFenceAfter();
    const uint32_t tbase = *sTmem;
    const uint32_t laneBase = static_cast<uint32_t>(warp * 32) << 16;
    const uint32_t fAddr = tc::smemAddr(smem + L.f), hAddr = tc::smemAddr(smem + L.h);
    const uint32_t w1Addr = tc::smemAddr(smem + L.w1), w2Addr = tc::smemAddr(smem + L.w2);
    uint32_t phase = 0, pending = 0;
    bool ok = true;

    for (uint64_t tile = blockIdx.x; tile * kTcRows < n; tile += gridDim.x) {
        const uint32_t e = static_cast<uint32_t>(tile * kTcRows) + tid;
        const bool live = e < n;
        // Features of this thread's sample, 8 columns (one 16-byte core-matrix row) at a time.
        if constexpr (FRONTIER) {
            // The entry's query point and centre are rows of D doubles: chunks of eight features
            // that lie inside one of them (D even) are read as four 16-byte loads.
            const double* pt = src.points + static_cast<size_t>(live ? src.q[e] : 0u) * D;
            const double* xr = src.x + static_cast<size_t>(live ? e : 0u) * D;
            const bool even = (D & 1) == 0;
            for (uint32_t k0 = 0; k0 < L.kp; k0 += 8) {
                const int kb = static_cast<int>(k0);
                float v[8];
                const double* run = nullptr;
                if (live && even && kb + 8 <= D) run = pt + kb;
                if (live && even && kb >= D && kb + 8 <= 2 * D) run = xr + (kb - D);
                if (run) {
#pragma unroll
                    for (int i = 0; i < 8; i += 2) {
                        const double2 t = __ldg(reinterpret_cast<const double2*>(run + i));
                        v[i] = static_cast<float>(t.x * src.inv);
                        v[i + 1] = static_cast<float>(t.y * src.inv);
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 8; ++i) v[i] = (live && kb + i < in) ? frontierFeature(src, e, kb + i, D) : 0.f;
                }
                *reinterpret_cast<uint4*>(smem + L.f + bf16Offset(tid, k0, L.kp)) = packBf16x8(v);
            }
        } else {
            for (uint32_t k0 = 0; k0 < L.kp; k0 += 8) {
                float v[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int k = static_cast<int>(k0) + i;
                    v[i] = (live && k < in) ? src.X[static_cast<size_t>(e) * in + k] : 0.f;
                }
                *reinterpret_cast<uint4*>(smem + L.f + bf16Offset(tid, k0, L.kp)) = packBf16x8(v);
            }
        }
        tc::fenceProxyAsync();
        tc::tcFenceBefore();
        __syncthreads();
        tc::tcFenceAfter();
        if (tid == 0) {
            for (uint32_t ks = 0; ks < L.kp / 16; ++ks)
                tc::mma<tc::kKindF16>(tbase, tc::smemDesc(fAddr + ks * 256u, 128, L.kp * 16u),
                                      tc::smemDesc(w1Addr + ks * 256u, 128, L.kp * 16u), kTcIdesc, ks);
            tc::mmaCommit(bar);
        }
        ++pending;
        ok = __syncthreads_and(tc::mbarWait(bar, phase, kTcSpin)) != 0;
        phase ^= 1u;
        if (!ok) break;
        --pending;
        tc::tcFenceAfter();
        // h1 = relu(acc + b1) as BF16 into the layer-2 A image.
#pragma unroll
        for (int c = 0; c < 64; c += 32) {
            uint32_t r[32];
            tc::tmemLoad32(tbase + laneBase + static_cast<uint32_t>(c), r);
            tc::tmemWaitLoad();
#pragma unroll
            for (int g = 0; g < 32; g += 8) {
                float v[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) v[i] = fmaxf(__uint_as_float(r[g + i]) + b1[c + g + i], 0.f);
                *reinterpret_cast<uint4*>(smem + L.h + bf16Offset(tid, c + g, 64)) = packBf16x8(v);
            }
        }
        tc::fenceProxyAsync();
        tc::tcFenceBefore();
        __syncthreads();
        tc::tcFenceAfter();
        if (tid == 0) {
#pragma unroll
            for (uint32_t ks = 0; ks < 4; ++ks)
                tc::mma<tc::kKindF16>(tbase + 64u, tc::smemDesc(hAddr + ks * 256u, 128, 1024),
                                      tc::smemDesc(w2Addr + ks * 256u, 128, 1024), kTcIdesc, ks);
            tc::mmaCommit(bar);
        }
        ++pending;
        ok = __syncthreads_and(tc::mbarWait(bar, phase, kTcSpin)) != 0;
        phase ^= 1u;
        if (!ok) break;
        --pending;
        tc::tcFenceAfter();
        float z = w3[H];
#pragma unroll
        for (int c = 0; c < 64; c += 32) {
            uint32_t r[32];
            tc::tmemLoad32(tbase + laneBase + 64u + static_cast<uint32_t>(c), r);
            tc::tmemWaitLoad();
#pragma unroll
            for (int i = 0; i < 32; ++i) z = fmaf(fmaxf(__uint_as_float(r[i]) + b2[c + i], 0.f), w3[c + i], z);
        }
        if (live) {
            if (FRONTIER)
                static_cast<double*>(out)[e] = -static_cast<double>(z);
            else
                static_cast<float*>(out)[e] = z;
        }
        tc::tcFenceBefore();
    }
    // A CTA that gave up waits once more (bounded) for its MMAs still in flight before freeing.
    if (!ok) {
        if (tid == 0) atomicOr(status, 1u);
        if (pending) tc::mbarWait(bar, phase ^ 1u, kTcSpin);
    }
    tc::tcFenceBefore();
    __syncthreads();
    tc::tcFenceAfter();
    if (warp == 0) tc::tmemDealloc(tbase, kTcCols);
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
    tcStatus_.alloc(4);
    TBLAEQ_CUDA(cudaMemset(tcStatus_.get(), 0, 4));
}

void Mlp::refreshBf16(cudaStream_t s) {
    const size_t n = shape_.params();
    toBf16Kernel<<<gridFor(n, 256), 256, 0, s>>>(master_.as<float>(), n, bf16_.as<__nv_bfloat16>());
    TBLAEQ_LAUNCHED();
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
    TBLAEQ_LAUNCHED();
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
    TBLAEQ_LAUNCHED();
    paramGradKernel<<<gridFor(o.total, 128), 128, 0, s>>>(X, h1, h2, dh1, dh2, dz, n, o.in, grad);
    TBLAEQ_LAUNCHED();
    sumKernel<<<1, 1024, 0, s>>>(lt, n, loss);
    TBLAEQ_LAUNCHED();
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
    TBLAEQ_LAUNCHED();
}

void Mlp::logits(const float* X, uint32_t n, float* z, cudaStream_t s) const {
    if (n == 0) return;
    const Offsets o = offsetsOf(shape_);
    const size_t smem = o.total * 4;
    TBLAEQ_CUDA(cudaFuncSetAttribute(logitsKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    logitsKernel<<<gridFor(n, 128), 128, smem, s>>>(bf16_.as<__nv_bfloat16>(), static_cast<int>(o.total), X, n, o.in, z);
    TBLAEQ_LAUNCHED();
}

void Mlp::frontierFeatures(const FrontierIn& f, const uint32_t* node, const uint32_t* idx, uint32_t n,
                           const double* points, const NodeRec* nodes, uint32_t level, double invScale, float* X,
                           cudaStream_t s) const {
    if (n == 0) return;
    frontierFeaturesKernel<<<gridFor(n, 256), 256, 0, s>>>(f.q, node, f.x, idx, n, points, nodes, level, shape_.levels,
                                                           shape_.D, invScale, X);
    TBLAEQ_LAUNCHED();
}

void Mlp::launchTc(bool frontier, const void* srcPtr, const uint32_t* hdr, uint32_t n, uint32_t cap, void* out,
                   cudaStream_t s) const {
    const FeatureSrc* src = static_cast<const FeatureSrc*>(srcPtr);
    const uint32_t rows = frontier ? cap : n;
    if (rows == 0) return;
    const uint32_t tiles = (rows + kTcRows - 1) / kTcRows;
    const unsigned grid = std::min<uint32_t>(tiles, 148u * kTcCtasPerSm);
    const auto kern = frontier ? forwardTcKernel<true> : forwardTcKernel<false>;
    TBLAEQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(kTcSmemRequest)));
    kern<<<grid, kTcRows, kTcSmemRequest, s>>>(bf16_.as<__nv_bfloat16>(), shape_.D, shape_.levels, *src, hdr, n, cap,
                                               out, tcStatus_.as<uint32_t>());
    TBLAEQ_LAUNCHED();
}

void Mlp::scoreFrontier(const FrontierIn& f, const uint32_t* node, uint32_t cap, const double* points,
                        const NodeRec* nodes, uint32_t level, double invScale, double* score, cudaStream_t s) const {
    FeatureSrc src{f.q, node, f.x, points, nodes, level, invScale, nullptr};
    launchTc(true, &src, f.hdr, 0, cap, score, s);
}

void Mlp::logitsTensor(const float* X, uint32_t n, float* z, cudaStream_t s) const {
    FeatureSrc src{nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0.0, X};
    launchTc(false, &src, nullptr, n, 0, z, s);
}

uint32_t Mlp::tensorStatus(cudaStream_t s) const {
    uint32_t v = 0;
    TBLAEQ_CUDA(cudaMemcpyAsync(&v, tcStatus_.get(), 4, cudaMemcpyDeviceToHost, s));
    TBLAEQ_CUDA(cudaStreamSynchronize(s));
    return v;
}

}  // namespace tblaeq
