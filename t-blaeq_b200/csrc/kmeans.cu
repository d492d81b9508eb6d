// Hierarchical k-means build (see kmeans.cuh).
#include "kmeans.cuh"
#include "knn.cuh"
#include "tcgen05.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <random>
#include <stdexcept>
#include <unordered_map>

namespace tblaeq {

namespace {

// ---- tensor-core assignment: layout constants ---------------------------------------------------
constexpr int kTileM = 128;                                  // points per tile = TMEM lanes
constexpr int kTileN = 128;                                  // centroids per tile = TMEM columns per buffer
constexpr int kKPad = 16;                                    // D <= 16, zero-padded; two K=8 TF32 MMAs
constexpr int kImage = kTileM * kKPad * 4;                   // one K-major TF32 operand image: 8192 B
constexpr int kPointTileBytes = 2 * kImage;                  // hi | lo
constexpr int kCentTileBytes = 2 * kImage + kTileN * 4;      // hi | lo | ||c||^2 (FP32): 16896 B
constexpr int kAssignThreads = 288;  // 8 consumer warps (two per TMEM lane quarter) + 1 producer warp
constexpr uint32_t kTmemCols = 2 * kTileN;                   // two accumulator buffers
// Shared memory requested per CTA: enough that at most two CTAs share an SM, so the two sets of
// 256 tensor-memory columns always fit and an allocation never waits.
constexpr size_t kAssignSmem = 100 * 1024;
constexpr uint32_t kSpinLimit = 1u << 22;                    // bounded mbarrier waits

constexpr uint32_t kIdesc = tc::instrDesc(tc::kFmtTf32, kTileM, kTileN);

// Byte offset of element (row r, column k) in a K-major, non-swizzled operand image: 8-row x
// 16-byte core matrices (4 values per row), the four K quarters of a row group 128 B apart
// (leading-dimension offset) and row groups 512 B apart (stride-dimension offset). One K=8 MMA
// reads two K quarters; the second MMA starts 256 B further.
__host__ __device__ constexpr uint32_t imageOffset(uint32_t r, uint32_t k) {
    return (r >> 3) * 512u + (k >> 2) * 128u + (r & 7u) * 16u + (k & 3u) * 4u;
}
constexpr uint32_t kSecondK = 256;  // byte offset of K = 8..15 within an image row group

using tc::bulkLoad;
using tc::mbarArrive;
using tc::mbarExpectTx;
using tc::mbarInit;
using tc::mmaCommit;
using tc::smemAddr;
using tc::tcFenceAfter;
using tc::tcFenceBefore;
using tc::tmemLoad32;
using tc::tmemWaitLoad;

// min(a, b, c) in one instruction (sm_100 three-input min.f32); equal to fminf(a, fminf(b, c)).
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// No swizzle, LBO = 128 B, SBO = 512 B (see imageOffset).
__device__ __forceinline__ uint64_t ummaDesc(uint32_t saddr) { return tc::smemDesc(saddr, 128, 512); }
__device__ __forceinline__ bool mbarWait(uint64_t* bar, uint32_t phase) { return tc::mbarWait(bar, phase, kSpinLimit); }
__device__ __forceinline__ void mmaTf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    tc::mma<tc::kKindTf32>(dtmem, adesc, bdesc, kIdesc, accumulate);
}

// ---- packing ----------------------------------------------------------------------------------
// v = h + l: h is v rounded to nearest-even at TF32 precision (10 fraction bits), l = v - h is
// exact in FP32 and is read by the tensor core at TF32 precision, leaving ~2^-21 |v| unrepresented.
__device__ __forceinline__ void splitTf32(float v, float& h, float& l) {
    uint32_t u = __float_as_uint(v);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0xfffu + ((u >> 13) & 1u)) & 0xffffe000u;
    h = __uint_as_float(u);
    l = v - h;
}

// Points -> per 128-point tile: hi image | lo image (rows past n stay zero: the buffer is cleared).
__global__ void packPointsKernel(const float* X, uint64_t n, int D, uint8_t* out) {
    for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < n;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint8_t* base = out + (p / kTileM) * kPointTileBytes;
        const uint32_t r = static_cast<uint32_t>(p % kTileM);
        for (int k = 0; k < kKPad; ++k) {
            float h, l;
            splitTf32(k < D ? X[p * D + k] : 0.f, h, l);
            *reinterpret_cast<float*>(base + imageOffset(r, k)) = h;
            *reinterpret_cast<float*>(base + kImage + imageOffset(r, k)) = l;
        }
    }
}

// Centroids -> per 128-centroid tile: hi image | lo image | ||c||^2. Slots past k get zero rows and
// an infinite norm, so they never win.
__global__ void packCentroidsKernel(const float* C, uint64_t k, uint64_t kPad, int D, uint8_t* out) {
    for (uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; c < kPad;
         c += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint8_t* base = out + (c / kTileN) * kCentTileBytes;
        const uint32_t r = static_cast<uint32_t>(c % kTileN);
        float nrm = INFINITY;
        if (c < k) {
            nrm = 0.f;
            for (int d = 0; d < D; ++d) nrm = fmaf(C[c * D + d], C[c * D + d], nrm);
        }
        for (int kk = 0; kk < kKPad; ++kk) {
            float h, l;
            splitTf32((c < k && kk < D) ? C[c * D + kk] : 0.f, h, l);
            *reinterpret_cast<float*>(base + imageOffset(r, kk)) = h;
            *reinterpret_cast<float*>(base + kImage + imageOffset(r, kk)) = l;
        }
        reinterpret_cast<float*>(base + 2 * kImage)[r] = nrm;
    }
}

// ---- tensor-core assignment ---------------------------------------------------------------------
// One CTA per 128-point tile, warp-specialised. The producer warp (warp 8, one lane) streams the
// centroid tiles through four shared-memory stages with bulk copies and issues the six TF32 MMAs of
// each tile into one of two tensor-memory accumulators. Eight consumer warps reduce: warps w and
// w+4 read TMEM lane quarter w (point rows 32w..32w+31), each half of the columns, and keep the two
// smallest ||c||^2 - 2 x.c (the two nearest centroids): per 32-column chunk one fused multiply-add
// and one min per value, and the top-2 update only when a lane's chunk minimum beats its current
// second best (rare once the first tiles have passed). Hand-offs are mbarriers: a stage is
// "full" when its copy lands, an accumulator "done" when its MMAs commit, and both are "free"
// again once all eight consumer warps have arrived; no CTA-wide barrier runs per tile. The two
// column halves merge through shared memory at the end, and an FP64 step then picks between the
// two candidates of every point.
constexpr int kStages = 4;
constexpr int kConsumerWarps = 8;

__device__ __forceinline__ void keepTwo(float v, uint32_t i, float& s1, uint32_t& i1, float& s2, uint32_t& i2) {
    if (v < s2) {
        if (v < s1) {
            s2 = s1;
            i2 = i1;
            s1 = v;
            i1 = i;
        } else {
            s2 = v;
            i2 = i;
        }
    }
}

__global__ void __launch_bounds__(kAssignThreads, 2)
    assignTcKernel(const uint8_t* points, const uint8_t* cents, uint64_t n, uint32_t nTiles, uint2* cand,
                   uint32_t* status) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sA = smem;
    uint8_t* sB = smem + kPointTileBytes;  // kStages stages of kCentTileBytes
    uint64_t* bars = reinterpret_cast<uint64_t*>(sB + kStages * kCentTileBytes);
    uint64_t* barA = bars;                          // A tile landed
    uint64_t* full = bars + 1;                      // [kStages] stage landed
    uint64_t* stageFree = full + kStages;           // [kStages] consumers done with a stage
    uint64_t* mmaDone = stageFree + kStages;        // [2] accumulator written
    uint64_t* accFree = mmaDone + 2;                // [2] consumers done with an accumulator
    uint32_t* sTmem = reinterpret_cast<uint32_t*>(accFree + 2);
    volatile int* sAbort = reinterpret_cast<volatile int*>(sTmem + 1);
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const uint64_t tile = blockIdx.x;

    if (tid == 0) {
        mbarInit(barA, 1);
        for (int i = 0; i < kStages; ++i) {
            mbarInit(&full[i], 1);
            mbarInit(&stageFree[i], kConsumerWarps);
        }
        for (int i = 0; i < 2; ++i) {
            mbarInit(&mmaDone[i], 1);
            mbarInit(&accFree[i], kConsumerWarps);
        }
        *sAbort = 0;
        tc::mbarInitFence();
    }
    if (warp == 0) {
        tc::tmemAlloc(sTmem, kTmemCols);
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tbase = *sTmem;

    // Producer bookkeeping (lane 0 of warp 8): what was issued, so an aborted CTA can drain it.
    uint32_t loadsIssued = 0, mmasIssued = 0;
    float s1 = INFINITY, s2 = INFINITY;
    uint32_t i1 = 0, i2 = 0;
    const int half = warp >> 2;  // consumers: which 64 columns of every tile this warp reduces

    if (warp == kConsumerWarps) {
        if (lane == 0) {
            mbarExpectTx(barA, kPointTileBytes);
            bulkLoad(sA, points + tile * kPointTileBytes, kPointTileBytes, barA);
            for (uint32_t t = 0; t < static_cast<uint32_t>(kStages) && t < nTiles; ++t) {
                mbarExpectTx(&full[t], kCentTileBytes);
                bulkLoad(sB + t * kCentTileBytes, cents + static_cast<uint64_t>(t) * kCentTileBytes, kCentTileBytes,
                         &full[t]);
                ++loadsIssued;
            }
            const uint32_t a0 = smemAddr(sA);
            bool ok = mbarWait(barA, 0);
            for (uint32_t t = 0; ok && t < nTiles; ++t) {
                const uint32_t b = t & 1u, st = t % kStages;
                // accumulator b: the consumers of tile t-2 are done with it
                if (t >= 2) ok = mbarWait(&accFree[b], ((t - 2) >> 1) & 1u);
                ok = ok && mbarWait(&full[st], (t / kStages) & 1u);
                if (!ok || *sAbort) break;
                tcFenceAfter();
                const uint32_t b0 = smemAddr(sB + st * kCentTileBytes);
                const uint32_t d = tbase + b * kTileN;
                // x.c ~ xh.ch + xh.cl + xl.ch, each as two K=8 halves
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t ko = h * kSecondK;
                    mmaTf32(d, ummaDesc(a0 + ko), ummaDesc(b0 + ko), h);
                    mmaTf32(d, ummaDesc(a0 + ko), ummaDesc(b0 + kImage + ko), 1);
                    mmaTf32(d, ummaDesc(a0 + kImage + ko), ummaDesc(b0 + ko), 1);
                }
                mmaCommit(&mmaDone[b]);
                ++mmasIssued;
                // refill the stage of tile t-1 with tile t+3 once its consumers released it
                if (t >= 1 && t + kStages - 1 < nTiles) {
                    const uint32_t ls = (t - 1) % kStages;
                    ok = mbarWait(&stageFree[ls], ((t - 1) / kStages) & 1u);
                    if (!ok) break;
                    mbarExpectTx(&full[ls], kCentTileBytes);
                    bulkLoad(sB + ls * kCentTileBytes, cents + static_cast<uint64_t>(t + kStages - 1) * kCentTileBytes,
                             kCentTileBytes, &full[ls]);
                    ++loadsIssued;
                }
            }
            if (!ok) {
                atomicOr(status, 1u);
                *sAbort = 1;
            }
        }
    } else {
        const uint32_t rowBase = static_cast<uint32_t>((warp & 3) * 32) << 16;
        for (uint32_t t = 0; t < nTiles; ++t) {
            const uint32_t b = t & 1u, st = t % kStages;
            if (!mbarWait(&mmaDone[b], (t >> 1) & 1u) || *sAbort) {
                if (lane == 0) {
                    atomicOr(status, 1u);
                    *sAbort = 1;
                }
                break;
            }
            tcFenceAfter();
            const float* cn = reinterpret_cast<const float*>(sB + st * kCentTileBytes + 2 * kImage) + half * 64;
            const uint32_t base = tbase + b * kTileN + static_cast<uint32_t>(half * 64) + rowBase;
            const uint32_t col0 = t * kTileN + static_cast<uint32_t>(half * 64);
#pragma unroll
            for (int c = 0; c < 64; c += 32) {
                uint32_t r[32];
                tmemLoad32(base + static_cast<uint32_t>(c), r);
                tmemWaitLoad();
                float m0 = INFINITY, m1 = INFINITY;
#pragma unroll
                for (int j = 0; j < 32; j += 4) {
                    // ||c||^2 - 2 x.c for four columns: two packed FMAs, two three-input minima
                    // (the same roundings as four fmaf and four fminf).
                    const float4 c4 = *reinterpret_cast<const float4*>(cn + c + j);
                    const float2 va = __ffma2_rn(make_float2(__uint_as_float(r[j]), __uint_as_float(r[j + 1])),
                                                 make_float2(-2.f, -2.f), make_float2(c4.x, c4.y));
                    const float2 vb = __ffma2_rn(make_float2(__uint_as_float(r[j + 2]), __uint_as_float(r[j + 3])),
                                                 make_float2(-2.f, -2.f), make_float2(c4.z, c4.w));
                    r[j] = __float_as_uint(va.x);
                    r[j + 1] = __float_as_uint(va.y);
                    r[j + 2] = __float_as_uint(vb.x);
                    r[j + 3] = __float_as_uint(vb.y);
                    m0 = min3f(m0, va.x, va.y);
                    m1 = min3f(m1, vb.x, vb.y);
                }
                if (fminf(m0, m1) < s2) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) keepTwo(__uint_as_float(r[j]), col0 + c + j, s1, i1, s2, i2);
                }
            }
            tcFenceBefore();
            __syncwarp();
            if (lane == 0) {
                mbarArrive(&accFree[b]);
                mbarArrive(&stageFree[st]);
            }
        }
    }
    __syncthreads();
    // An aborted CTA waits (bounded) for its own copies and MMAs still in flight before freeing.
    if (warp == kConsumerWarps && lane == 0 && *sAbort) {
        for (uint32_t t = 0; t < loadsIssued; ++t) mbarWait(&full[t % kStages], (t / kStages) & 1u);
        for (uint32_t t = 0; t < mmasIssued; ++t) mbarWait(&mmaDone[t & 1u], (t >> 1) & 1u);
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    if (warp == 0) {
        tc::tmemDealloc(tbase, kTmemCols);
    }
    // Merge the two column halves of every row through shared memory (the stages are idle now).
    float* mv = reinterpret_cast<float*>(sB);
    uint32_t* mi = reinterpret_cast<uint32_t*>(sB + 2 * kTileM * 4);
    const int row = (warp & 3) * 32 + lane;
    if (warp < kConsumerWarps && half == 1) {
        mv[2 * row] = s1;
        mv[2 * row + 1] = s2;
        mi[2 * row] = i1;
        mi[2 * row + 1] = i2;
    }
    __syncthreads();
    if (warp < kConsumerWarps && half == 0) {
        keepTwo(mv[2 * row], mi[2 * row], s1, i1, s2, i2);
        keepTwo(mv[2 * row + 1], mi[2 * row + 1], s1, i1, s2, i2);
        const uint64_t p = tile * kTileM + static_cast<uint64_t>(row);
        if (p < n && !*sAbort) cand[p] = make_uint2(i1, s2 < INFINITY ? i2 : i1);
    }
}

// FP64 choice between the two tensor-core candidates of every point (ties: the smaller index).
__global__ void refineKernel(const float* X, const uint2* cand, const double* Cd, uint64_t n, int D,
                             uint32_t* labels) {
    for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < n;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint2 c = cand[p];
        double d0 = 0.0, d1 = 0.0;
        for (int d = 0; d < D; ++d) {
            const double x = static_cast<double>(X[p * D + d]);
            const double e0 = x - Cd[static_cast<uint64_t>(c.x) * D + d];
            const double e1 = x - Cd[static_cast<uint64_t>(c.y) * D + d];
            d0 = __fma_rn(e0, e0, d0);
            d1 = __fma_rn(e1, e1, d1);
        }
        labels[p] = (d1 < d0 || (d1 == d0 && c.y < c.x)) ? c.y : c.x;
    }
}

// ---- CUDA-core assignment (FP32 or FP64) -------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) assignScalarKernel(const float* X, uint64_t n, int D, const T* C, uint64_t k,
                                                          uint32_t* labels) {
    constexpr int kChunk = 128;
    extern __shared__ __align__(16) unsigned char smemRaw[];
    T* sC = reinterpret_cast<T*>(smemRaw);
    const uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    T x[32];
    for (int d = 0; d < 32; ++d) x[d] = (p < n && d < D) ? static_cast<T>(X[p * D + d]) : T(0);
    T best = std::numeric_limits<T>::infinity();
    uint32_t bestI = 0;
    for (uint64_t c0 = 0; c0 < k; c0 += kChunk) {
        const uint64_t m = std::min<uint64_t>(kChunk, k - c0);
        __syncthreads();
        for (uint64_t i = threadIdx.x; i < m * D; i += blockDim.x) sC[i] = C[c0 * D + i];
        __syncthreads();
        for (uint64_t c = 0; c < m; ++c) {
            T dist = 0;
            for (int d = 0; d < D; ++d) {
                const T diff = x[d] - sC[c * D + d];
                if constexpr (sizeof(T) == 4) {
                    dist = __fmaf_rn(diff, diff, dist);
                } else {
                    dist = __fma_rn(diff, diff, dist);
                }
            }
            if (dist < best) {
                best = dist;
                bestI = static_cast<uint32_t>(c0 + c);
            }
        }
    }
    if (p < n) labels[p] = bestI;
}

// ---- update and objective -----------------------------------------------------------------------
__global__ void accumulateKernel(const float* X, const uint32_t* labels, uint64_t n, int D, double* sums,
                                 unsigned long long* counts) {
    for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < n;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t l = labels[p];
        atomicAdd(&counts[l], 1ull);
        for (int d = 0; d < D; ++d) atomicAdd(&sums[static_cast<uint64_t>(l) * D + d], static_cast<double>(X[p * D + d]));
    }
}

// Moves each centroid with points to their mean (FP64), keeps empty ones.
__global__ void finalizeKernel(const double* sums, const unsigned long long* counts, uint64_t k, int D, double* Cd,
                               float* C) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < k * D;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t c = i / D;
        if (counts[c] > 0) {
            const double v = sums[i] / static_cast<double>(counts[c]);
            Cd[i] = v;
            C[i] = static_cast<float>(v);
        }
    }
}

__global__ void objectiveKernel(const float* X, const uint32_t* labels, const double* Cd, uint64_t n, int D,
                                double* out) {
    __shared__ double part[256 / 32];
    double acc = 0.0;
    for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < n;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double* c = Cd + static_cast<uint64_t>(labels[p]) * D;
        for (int d = 0; d < D; ++d) {
            const double diff = static_cast<double>(X[p * D + d]) - c[d];
            acc = fma(diff, diff, acc);
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < static_cast<int>(blockDim.x / 32); ++w) s += part[w];
        atomicAdd(out, s);
    }
}

__global__ void gatherKernel(const float* X, const uint64_t* idx, uint64_t k, int D, double* Cd, float* C) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < k * D;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const float v = X[idx[i / D] * D + i % D];
        C[i] = v;
        Cd[i] = static_cast<double>(v);
    }
}

int gridFor(uint64_t work, int threads) {
    return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((work + threads - 1) / threads, 148ull * 32)));
}

// Assembles interval pIdx of the index from one level's labels, like the reference's
// Genenate_One_P_Tensor + Compute_Max_Radius: rows grouped by label (in input order within a
// label), values fine / coarse, radius = largest distance from a centroid to its members.
void assembleInterval(HostIndex& idx, uint64_t pIdx, uint64_t fineMesh, const float* fine, uint64_t nF,
                      const float* coarse, uint64_t nC, const uint32_t* labels) {
    const uint64_t D = idx.D;
    PTensor& P = idx.pTensors[pIdx];
    P.D = D;
    P.rows = nF;
    P.cols = nC;
    P.nnz = nF;
    P.isAos = 1;
    P.nnzPerCol.assign(nC, 0);
    for (uint64_t i = 0; i < nF; ++i) ++P.nnzPerCol[labels[i]];
    P.colRes.assign(nC + 1, 0);
    for (uint64_t c = 0; c < nC; ++c) P.colRes[c + 1] = P.colRes[c] + P.nnzPerCol[c];
    P.rowIds.resize(nF);
    std::iota(P.rowIds.begin(), P.rowIds.end(), uint64_t{0});
    std::vector<uint64_t> order(nF), next(P.colRes.begin(), P.colRes.end() - 1);
    for (uint64_t i = 0; i < nF; ++i) order[next[labels[i]]++] = i;
    P.vals.resize(nF * D);
    idx.radius[pIdx].assign(nC, 0.0);
    const int64_t cols = static_cast<int64_t>(nC);
    bool zeroCoord = false;
#pragma omp parallel for schedule(dynamic, 256) reduction(|| : zeroCoord)
    for (int64_t c = 0; c < cols; ++c) {
        double maxDist = 0.0;
        for (uint64_t pos = P.colRes[c]; pos < P.colRes[c + 1]; ++pos) {
            const float* fv = fine + order[pos] * D;
            double sum = 0.0;
            for (uint64_t d = 0; d < D; ++d) {
                const double cv = static_cast<double>(coarse[c * D + d]);
                const double f = static_cast<double>(fv[d]);
                if (cv == 0.0) zeroCoord = true;
                P.vals[pos * D + d] = f / cv;
                const double diff = cv - f;
                sum += diff * diff;
            }
            maxDist = std::max(maxDist, std::sqrt(sum));
        }
        idx.radius[pIdx][c] = maxDist;
    }
    if (zeroCoord) throw std::runtime_error("division by zero in P-tensor build: a centroid coordinate is 0");
    idx.maps[fineMesh] = std::move(order);
}

// ---- index assembly on the device (replaces the host loop above for builds) --------------------
// sortKeys[i] = (label << 32) | i: sorting them groups the points by label, in input order within a
// label (the order the host assembly and the reference's std::sort by label produce).
__global__ void labelKeysKernel(const uint32_t* labels, uint64_t n, uint64_t* keys, uint32_t* vals) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        keys[i] = (static_cast<uint64_t>(labels[i]) << 32) | i;
        vals[i] = static_cast<uint32_t>(i);
    }
}

// colRes from the sorted keys: colRes[c] = first position whose label is >= c, colRes[k] = n.
__global__ void colResKernel(const uint64_t* keys, uint64_t n, uint64_t k, uint64_t* colRes) {
    for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p <= n;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t prev = p == 0 ? 0 : (keys[p - 1] >> 32) + 1;  // first label not yet started
        const uint64_t cur = p == n ? k : (keys[p] >> 32);
        for (uint64_t c = prev; c <= cur && c <= k; ++c) colRes[c] = p;
    }
}

// Row `pos` of the P-tensor: the member point's coordinates divided by its centroid's (FP64
// division of the FP32 values, like the host assembly), the map entry (the member's input index),
// and the member's distance to its centroid folded into the centroid's radius (sum of squares in
// dimension order with separate multiply and add, correctly rounded square root; distances are
// non-negative, so their bit patterns order like their values and an integer maximum is exact).
__global__ void assembleRowsKernel(const uint64_t* keys, uint64_t n, int D, const float* fine, const float* coarse,
                                   double* vals, uint64_t* map, unsigned long long* radiusBits, uint32_t* zero) {
    for (uint64_t pos = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; pos < n;
         pos += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t key = keys[pos];
        const uint64_t c = key >> 32, i = key & 0xffffffffull;
        double sum = 0.0;
        bool z = false;
        for (int d = 0; d < D; ++d) {
            const double cv = static_cast<double>(coarse[c * D + d]);
            const double f = static_cast<double>(fine[i * D + d]);
            z = z || cv == 0.0;
            vals[pos * D + d] = __ddiv_rn(f, cv);
            const double diff = __dsub_rn(cv, f);
            sum = __dadd_rn(sum, __dmul_rn(diff, diff));
        }
        if (z) atomicOr(zero, 1u);
        map[pos] = i;
        atomicMax(radiusBits + c, static_cast<unsigned long long>(__double_as_longlong(__dsqrt_rn(sum))));
    }
}

// Assembles interval pIdx on the device from one level's labels (device), its points (dFine) and
// centroids (dCoarse), with the same results as assembleInterval, and copies the finished arrays
// (P values, column offsets and sizes, map, radii) into the host index. Labels and centroids stay
// on the device.
void assembleIntervalDevice(HostIndex& idx, uint64_t pIdx, uint64_t fineMesh, const float* dFine, uint64_t nF,
                            const float* dCoarse, uint64_t nC, const uint32_t* dLabels, cudaStream_t s) {
    if (nF > 0xffffffffull) throw std::invalid_argument("k-means build: a level above 2^32 points");
    const uint64_t D = idx.D;
    DeviceMem keys(nF * 8), keys2(nF * 8), vals(nF * 4), vals2(nF * 4);
    labelKeysKernel<<<gridFor(nF, 256), 256, 0, s>>>(dLabels, nF, keys.as<uint64_t>(), vals.as<uint32_t>());
    TBLAEQ_LAUNCHED();
    sortPairs(keys.as<uint64_t>(), vals.as<uint32_t>(), keys2.as<uint64_t>(), vals2.as<uint32_t>(), nF, s);
    DeviceMem colRes((nC + 1) * 8), pv(nF * D * 8), map(nF * 8), rad(nC * 8), zero(4);
    TBLAEQ_CUDA(cudaMemsetAsync(rad.get(), 0, nC * 8, s));
    TBLAEQ_CUDA(cudaMemsetAsync(zero.get(), 0, 4, s));
    colResKernel<<<gridFor(nF + 1, 256), 256, 0, s>>>(keys.as<uint64_t>(), nF, nC, colRes.as<uint64_t>());
    TBLAEQ_LAUNCHED();
    assembleRowsKernel<<<gridFor(nF, 256), 256, 0, s>>>(keys.as<uint64_t>(), nF, static_cast<int>(D), dFine, dCoarse,
                                                        pv.as<double>(), map.as<uint64_t>(),
                                                        rad.as<unsigned long long>(), zero.as<uint32_t>());
    TBLAEQ_LAUNCHED();
    PTensor& P = idx.pTensors[pIdx];
    P.D = D;
    P.rows = nF;
    P.cols = nC;
    P.nnz = nF;
    P.isAos = 1;
    P.colRes.resize(nC + 1);
    P.vals.resize(nF * D);
    idx.maps[fineMesh].resize(nF);
    idx.radius[pIdx].resize(nC);
    uint32_t z = 0;
    TBLAEQ_CUDA(cudaMemcpyAsync(P.colRes.data(), colRes.get(), (nC + 1) * 8, cudaMemcpyDeviceToHost, s));
    TBLAEQ_CUDA(cudaMemcpyAsync(P.vals.data(), pv.get(), nF * D * 8, cudaMemcpyDeviceToHost, s));
    TBLAEQ_CUDA(cudaMemcpyAsync(idx.maps[fineMesh].data(), map.get(), nF * 8, cudaMemcpyDeviceToHost, s));
    TBLAEQ_CUDA(cudaMemcpyAsync(idx.radius[pIdx].data(), rad.get(), nC * 8, cudaMemcpyDeviceToHost, s));
    TBLAEQ_CUDA(cudaMemcpyAsync(&z, zero.get(), 4, cudaMemcpyDeviceToHost, s));
    TBLAEQ_CUDA(cudaStreamSynchronize(s));
    if (z) throw std::runtime_error("division by zero in P-tensor build: a centroid coordinate is 0");
    P.nnzPerCol.resize(nC);
    for (uint64_t c = 0; c < nC; ++c) P.nnzPerCol[c] = P.colRes[c + 1] - P.colRes[c];
    P.rowIds.resize(nF);
    std::iota(P.rowIds.begin(), P.rowIds.end(), uint64_t{0});
}

}  // namespace

void kmeansRun(const float* dX, uint64_t n, uint64_t D, uint64_t k, const KmeansConfig& cfg, DeviceMem& centroids,
               DeviceMem& labels, KmeansLevelReport& report, cudaStream_t s) {
    if (n == 0 || k == 0 || k > n) throw std::invalid_argument("k-means needs 0 < k <= n");
    if (D == 0 || D > 32) throw std::invalid_argument("k-means supports 1 <= D <= 32");
    if (k > 0xffffffffull || n > (1ull << 40)) throw std::invalid_argument("k-means sizes out of range");
    int precision = cfg.precision;
    if (precision == kKmTensor && !kmeansTensorSupports(D)) precision = kKmFp32;
    report.n = n;
    report.k = k;
    report.iters = cfg.iters;
    report.objectives.clear();
    const int Di = static_cast<int>(D);

    // Initial centroids: k distinct data points, chosen with a seeded partial Fisher-Yates shuffle.
    std::vector<uint64_t> pick(k);
    {
        std::mt19937_64 rng(cfg.seed);
        std::unordered_map<uint64_t, uint64_t> swapped;
        for (uint64_t i = 0; i < k; ++i) {
            const uint64_t j = i + std::uniform_int_distribution<uint64_t>(0, n - 1 - i)(rng);
            auto vi = swapped.find(i), vj = swapped.find(j);
            const uint64_t a = vi == swapped.end() ? i : vi->second, b = vj == swapped.end() ? j : vj->second;
            pick[i] = b;
            swapped[j] = a;
        }
    }
    DeviceMem dPick = upload(pick, s);
    centroids.alloc(k * D * 4);
    DeviceMem Cd(k * D * 8), sums(k * D * 8), counts(k * 8), obj(8);
    labels.alloc(n * 4);
    gatherKernel<<<gridFor(k * D, 256), 256, 0, s>>>(dX, dPick.as<uint64_t>(), k, Di, Cd.as<double>(), centroids.as<float>());
    TBLAEQ_LAUNCHED();

    const uint64_t nTilesP = (n + kTileM - 1) / kTileM, nTilesC = (k + kTileN - 1) / kTileN;
    DeviceMem packedP, packedC, cand, status(4);
    if (precision == kKmTensor) {
        cand.alloc(n * 8);
        packedP.alloc(nTilesP * kPointTileBytes);
        packedC.alloc(nTilesC * kCentTileBytes);
        TBLAEQ_CUDA(cudaMemsetAsync(packedP.get(), 0, nTilesP * kPointTileBytes, s));
        packPointsKernel<<<gridFor(n, 256), 256, 0, s>>>(dX, n, Di, packedP.as<uint8_t>());
        TBLAEQ_LAUNCHED();
        TBLAEQ_CUDA(cudaFuncSetAttribute(assignTcKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kAssignSmem)));
    }
    TBLAEQ_CUDA(cudaMemsetAsync(status.get(), 0, 4, s));
    cudaEvent_t e0, e1;
    TBLAEQ_CUDA(cudaEventCreate(&e0));
    TBLAEQ_CUDA(cudaEventCreate(&e1));
    double assignMs = 0.0;
    for (int it = 0; it < cfg.iters; ++it) {
        TBLAEQ_CUDA(cudaEventRecord(e0, s));
        if (precision == kKmTensor) {
            packCentroidsKernel<<<gridFor(nTilesC * kTileN, 256), 256, 0, s>>>(centroids.as<float>(), k,
                                                                              nTilesC * kTileN, Di,
                                                                              packedC.as<uint8_t>());
            TBLAEQ_LAUNCHED();
            assignTcKernel<<<static_cast<unsigned>(nTilesP), kAssignThreads, kAssignSmem, s>>>(
                packedP.as<uint8_t>(), packedC.as<uint8_t>(), n, static_cast<uint32_t>(nTilesC), cand.as<uint2>(),
                status.as<uint32_t>());
            TBLAEQ_LAUNCHED();
            refineKernel<<<gridFor(n, 256), 256, 0, s>>>(dX, cand.as<uint2>(), Cd.as<double>(), n, Di,
                                                         labels.as<uint32_t>());
            TBLAEQ_LAUNCHED();
        } else if (precision == kKmFp32) {
            assignScalarKernel<float><<<static_cast<unsigned>((n + 255) / 256), 256, 128 * D * 4, s>>>(
                dX, n, Di, centroids.as<float>(), k, labels.as<uint32_t>());
            TBLAEQ_LAUNCHED();
        } else {
            assignScalarKernel<double><<<static_cast<unsigned>((n + 255) / 256), 256, 128 * D * 8, s>>>(
                dX, n, Di, Cd.as<double>(), k, labels.as<uint32_t>());
            TBLAEQ_LAUNCHED();
        }
        TBLAEQ_CUDA(cudaEventRecord(e1, s));
        TBLAEQ_CUDA(cudaMemsetAsync(sums.get(), 0, k * D * 8, s));
        TBLAEQ_CUDA(cudaMemsetAsync(counts.get(), 0, k * 8, s));
        accumulateKernel<<<gridFor(n, 256), 256, 0, s>>>(dX, labels.as<uint32_t>(), n, Di, sums.as<double>(),
                                                         counts.as<unsigned long long>());
        TBLAEQ_LAUNCHED();
        finalizeKernel<<<gridFor(k * D, 256), 256, 0, s>>>(sums.as<double>(), counts.as<unsigned long long>(), k, Di,
                                                           Cd.as<double>(), centroids.as<float>());
        TBLAEQ_LAUNCHED();
        TBLAEQ_CUDA(cudaMemsetAsync(obj.get(), 0, 8, s));
        objectiveKernel<<<gridFor(n, 256), 256, 0, s>>>(dX, labels.as<uint32_t>(), Cd.as<double>(), n, Di,
                                                        obj.as<double>());
        TBLAEQ_LAUNCHED();
        double o = 0.0;
        uint32_t st = 0;
        TBLAEQ_CUDA(cudaMemcpyAsync(&o, obj.get(), 8, cudaMemcpyDeviceToHost, s));
        TBLAEQ_CUDA(cudaMemcpyAsync(&st, status.get(), 4, cudaMemcpyDeviceToHost, s));
        TBLAEQ_CUDA(cudaStreamSynchronize(s));
        if (st) throw CudaError(cudaErrorLaunchTimeout, "k-means assignment kernel gave up waiting (status " +
                                                            std::to_string(st) + ")");
        float ms = 0.f;
        TBLAEQ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        assignMs += ms;
        report.objectives.push_back(o);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    report.objective = report.objectives.empty() ? 0.0 : report.objectives.back();
    report.assignSeconds = assignMs / 1e3;
}

HostIndex kmeansBuild(const float* hostPoints, uint64_t N, uint64_t D, uint64_t height,
                      const std::vector<uint64_t>& ratios, const KmeansConfig& cfg,
                      std::vector<KmeansLevelReport>& reports, cudaStream_t s) {
    if (height < 2) throw std::invalid_argument("k-means build: height must be >= 2");
    if (ratios.size() != height - 1) throw std::invalid_argument("k-means build: ratios size must equal height - 1");
    if (!hostPoints || N == 0 || D == 0) throw std::invalid_argument("k-means build: no points");
    HostIndex idx;
    idx.D = D;
    idx.N = N;
    idx.height = height;
    idx.intervals = height - 1;
    idx.isAos = 1;
    idx.ratios = ratios;
    idx.pTensors.resize(idx.intervals);
    idx.radius.resize(idx.intervals);
    idx.maps.resize(height);
    idx.datasetName = "Kmeans" + std::to_string(N) + "D" + std::to_string(D);
    reports.assign(idx.intervals, KmeansLevelReport{});

    DeviceMem dX(N * D * 4);
    TBLAEQ_CUDA(cudaMemcpyAsync(dX.get(), hostPoints, N * D * 4, cudaMemcpyHostToDevice, s));
    uint64_t n = N;
    for (uint64_t i = 0; i < idx.intervals; ++i) {
        const auto t0 = std::chrono::steady_clock::now();
        const uint64_t k = (ratios[i] == 0 || n / ratios[i] == 0) ? 1 : n / ratios[i];  // IndexBuilder.cu:14-19
        const uint64_t fineMesh = idx.intervals - i, pIdx = fineMesh - 1;
        idx.meshSizes.push_back(n);
        DeviceMem C, L;
        KmeansConfig c = cfg;
        c.seed = cfg.seed + i;
        kmeansRun(dX.as<float>(), n, D, k, c, C, L, reports[i], s);
        const auto ta = std::chrono::steady_clock::now();
        if (cfg.hostAssembly != kAssembleDevice) {
            std::vector<float> fine(n * D), coarse(k * D);
            std::vector<uint32_t> labels(n);
            TBLAEQ_CUDA(cudaMemcpyAsync(fine.data(), dX.get(), n * D * 4, cudaMemcpyDeviceToHost, s));
            TBLAEQ_CUDA(cudaMemcpyAsync(coarse.data(), C.get(), k * D * 4, cudaMemcpyDeviceToHost, s));
            TBLAEQ_CUDA(cudaMemcpyAsync(labels.data(), L.get(), n * 4, cudaMemcpyDeviceToHost, s));
            TBLAEQ_CUDA(cudaStreamSynchronize(s));
            assembleInterval(idx, pIdx, fineMesh, fine.data(), n, coarse.data(), k, labels.data());
        }
        if (cfg.hostAssembly != kAssembleHost) {
            // Both: the host result is kept aside and the device result must equal it byte for byte
            // (the same labels and centroids feed both; k-means itself is not bitwise repeatable,
            // its FP64 sums are atomic).
            HostIndex ref;
            const bool both = cfg.hostAssembly == kAssembleBoth;
            if (both) {
                ref.pTensors.push_back(std::move(idx.pTensors[pIdx]));
                ref.maps.push_back(std::move(idx.maps[fineMesh]));
                ref.radius.push_back(std::move(idx.radius[pIdx]));
            }
            assembleIntervalDevice(idx, pIdx, fineMesh, dX.as<float>(), n, C.as<float>(), k, L.as<uint32_t>(), s);
            if (both) {
                const PTensor& a = idx.pTensors[pIdx];
                const PTensor& b = ref.pTensors[0];
                const bool same = a.colRes == b.colRes && a.nnzPerCol == b.nnzPerCol && a.rowIds == b.rowIds &&
                                  std::memcmp(a.vals.data(), b.vals.data(), a.vals.size() * 8) == 0 &&
                                  a.vals.size() == b.vals.size() && idx.maps[fineMesh] == ref.maps[0] &&
                                  idx.radius[pIdx].size() == ref.radius[0].size() &&
                                  std::memcmp(idx.radius[pIdx].data(), ref.radius[0].data(),
                                              ref.radius[0].size() * 8) == 0;
                if (!same)
                    throw std::runtime_error("k-means build: device and host assembly differ at interval " +
                                             std::to_string(pIdx));
            }
        }
        reports[i].assembleSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - ta).count();
        if (i + 2 == height) {
            std::vector<float> coarse(k * D);
            TBLAEQ_CUDA(cudaMemcpyAsync(coarse.data(), C.get(), k * D * 4, cudaMemcpyDeviceToHost, s));
            TBLAEQ_CUDA(cudaStreamSynchronize(s));
            idx.meshSizes.push_back(k);
            idx.coarsest.rows = k;
            idx.coarsest.dim = D;
            idx.coarsest.nnz = k;
            idx.coarsest.isAos = 1;
            idx.coarsest.ids.resize(k);
            std::iota(idx.coarsest.ids.begin(), idx.coarsest.ids.end(), uint64_t{0});
            idx.coarsest.vals.assign(coarse.begin(), coarse.end());
        }
        // The centroids are the next level's data (they stay on the device).
        dX = std::move(C);
        n = k;
        reports[i].seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    idx.validate();
    return idx;
}

}  // namespace tblaeq
