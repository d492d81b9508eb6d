// extern "C" boundary (include/tblaeq.h) over the C++ facade.
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <new>
#include <string>

#include "../../include/tblaeq.h"
#include "handler.hpp"
#include "noalloc.hpp"
#include "scorer.hpp"
#include "serve.hpp"
#include "kmeans.cuh"
#include "tuning.hpp"

using namespace tblaeq;

std::atomic<uint64_t> tblaeq::gKernelLaunches{0};

struct tblaeq_handle {
    std::unique_ptr<QueryHandler> qh;
    DeviceMem stage;                            // device staging for host-side query batches
    std::vector<std::vector<uint32_t>> parent;  // parent position per mesh (lazy, decode_points)
    std::vector<std::vector<uint64_t>> posOf;   // position of each original id per mesh (lazy)
    DeviceMem kStage;                           // per-query K of KNN batches
    DeviceMem knnOff, knnIds, knnD2;            // results of KNN batches run in chunks
    std::vector<uint64_t> knnSum;               // counters summed over the last batch's chunks (empty: one run)
    uint64_t knnChunkHint = 0;                  // queries per traversal that last fitted after a split (0: none)
    bool knnHintTwoWave = true;                 // the finest-level mode that size was learnt under
    uint64_t knnChunkMax = 0;                   // caller's limit on queries per traversal (0: automatic)
    uint64_t lastKnnChunk = 0, lastKnnRuns = 0; // the last KNN batch: queries per traversal, traversals
    std::string knnSplitReason;                 // why the last split KNN batch was split
    uint64_t lastNq = 0;                        // last asynchronously enqueued batch
    unsigned lastFlags = 0;
};

namespace {

thread_local std::string gLastError;

int fail(int code, const std::string& msg) {
    gLastError = msg;
    return code;
}

template <class F>
int guarded(F&& f) {
    try {
        gLastError.clear();
        return f();
    } catch (const CudaError& e) {
        if (e.code == cudaErrorMemoryAllocation) return fail(TBLAEQ_ERR_OOM, e.what());
        if (e.code == cudaErrorLaunchTimeout) return fail(TBLAEQ_ERR_TIMEOUT, e.what());
        return fail(TBLAEQ_ERR_CUDA, e.what());
    } catch (const std::invalid_argument& e) {
        return fail(TBLAEQ_ERR_INVALID, e.what());
    } catch (const std::out_of_range& e) {
        return fail(TBLAEQ_ERR_INVALID, e.what());
    } catch (const std::bad_alloc& e) {
        return fail(TBLAEQ_ERR_OOM, std::string("host allocation failed: ") + e.what());
    } catch (const std::exception& e) {
        const std::string m = e.what();
        if (m.rfind("Cannot read", 0) == 0 || m.rfind("Truncated", 0) == 0 || m.rfind("Invalid index", 0) == 0 ||
            m.rfind("Cannot write", 0) == 0 || m.rfind("Read error", 0) == 0 || m.rfind("Short write", 0) == 0 ||
            m.rfind("Cannot stat", 0) == 0)
            return fail(TBLAEQ_ERR_IO, m);
        return fail(TBLAEQ_ERR_CUDA, m);
    } catch (...) {
        return fail(TBLAEQ_ERR_CUDA, "unknown error");
    }
}

int checkPrepared(tblaeq_handle* h) {
    if (!h || !h->qh) return fail(TBLAEQ_ERR_INVALID, "null handle");
    if (!h->qh->prepared()) return fail(TBLAEQ_ERR_STATE, "call tblaeq_prepare before querying");
    return TBLAEQ_OK;
}

}  // namespace

extern "C" {

const char* tblaeq_last_error(void) { return gLastError.c_str(); }
int tblaeq_abi_version(void) { return TBLAEQ_ABI_VERSION; }

int tblaeq_open(const char* dir, tblaeq_handle** out) {
    if (!dir || !out) return fail(TBLAEQ_ERR_INVALID, "null argument");
    *out = nullptr;
    return guarded([&]() -> int {
        if (!std::filesystem::is_directory(dir)) return fail(TBLAEQ_ERR_IO, std::string("Cannot read: ") + dir);
        auto h = std::make_unique<tblaeq_handle>();
        h->qh = std::make_unique<QueryHandler>(std::string(dir), true);
        *out = h.release();
        return TBLAEQ_OK;
    });
}

int tblaeq_generate(const tblaeq_gen_params* p, tblaeq_handle** out) {
    if (!p || !out) return fail(TBLAEQ_ERR_INVALID, "null argument");
    *out = nullptr;
    return guarded([&]() -> int {
        GenParams g;
        g.N = p->N;
        g.D = p->D;
        g.valMin = p->valMin;
        g.valMax = p->valMax;
        g.isInt = p->isInt != 0;
        g.height = p->height;
        if (p->height < 2) return fail(TBLAEQ_ERR_INVALID, "QueryHandler: height must be >= 2");
        if (!p->ratios || p->nRatios != p->height - 1)
            return fail(TBLAEQ_ERR_INVALID, "QueryHandler: ratios size must equal height - 1");
        g.ratios.assign(p->ratios, p->ratios + (p->height - 1));
        g.seed = p->seed;
        g.sigmaDivisor = p->sigmaDivisor;
        auto h = std::make_unique<tblaeq_handle>();
        h->qh = std::make_unique<QueryHandler>(g);
        *out = h.release();
        return TBLAEQ_OK;
    });
}

int tblaeq_save(const tblaeq_handle* h, const char* dir) {
    if (!h || !dir) return fail(TBLAEQ_ERR_INVALID, "null argument");
    return guarded([&]() -> int {
        h->qh->saveIndex(dir);
        return TBLAEQ_OK;
    });
}

void tblaeq_close(tblaeq_handle* h) { delete h; }

int tblaeq_info(const tblaeq_handle* h, tblaeq_index_info* out) {
    if (!h || !out) return fail(TBLAEQ_ERR_INVALID, "null argument");
    return guarded([&]() -> int {
        const HostIndex& x = h->qh->index();
        std::memset(out, 0, sizeof(*out));
        out->D = x.D;
        out->N = x.N;
        out->height = x.height;
        out->intervals = x.intervals;
        if (x.height > TBLAEQ_MAX_HEIGHT) return fail(TBLAEQ_ERR_INVALID, "index deeper than TBLAEQ_MAX_HEIGHT");
        for (uint64_t i = 0; i < x.height; ++i) out->meshSizes[i] = x.meshSizes[i];
        for (uint64_t i = 0; i < x.intervals; ++i) out->ratios[i] = x.ratios[i];
        const MemoryStats st = computeStats(x);
        out->hostBytes = st.hostTotal;
        out->deviceBytes = st.deviceTotal;
        out->prepared = h->qh->prepared() ? 1 : 0;
        if (h->qh->prepared())
            for (uint64_t i = 0; i < x.intervals; ++i) out->policy[i] = static_cast<int>(h->qh->activePolicy().levels[i]);
        return TBLAEQ_OK;
    });
}

int tblaeq_recommend(const tblaeq_handle* h, uint64_t free_bytes, int* policy_out) {
    if (!h || !policy_out) return fail(TBLAEQ_ERR_INVALID, "null argument");
    return guarded([&]() -> int {
        uint64_t fb = free_bytes;
        if (fb == 0) {
            size_t f = 0, t = 0;
            TBLAEQ_CUDA(cudaMemGetInfo(&f, &t));
            fb = f;
        }
        const IndexPolicy p = PolicyScheduler::recommend(h->qh->index(), fb);
        for (size_t i = 0; i < p.levels.size(); ++i) policy_out[i] = static_cast<int>(p.levels[i]);
        return TBLAEQ_OK;
    });
}

int tblaeq_prepare(tblaeq_handle* h, const int* policy, uint64_t n_levels) {
    if (!h) return fail(TBLAEQ_ERR_INVALID, "null handle");
    return guarded([&]() -> int {
        if (!policy) {
            h->qh->prepareForQuery();
            return TBLAEQ_OK;
        }
        if (n_levels != h->qh->index().intervals)
            return fail(TBLAEQ_ERR_INVALID, "policy must list one LevelPolicy per interval");
        IndexPolicy p;
        for (uint64_t i = 0; i < n_levels; ++i) {
            if (policy[i] < 0 || policy[i] > 3) return fail(TBLAEQ_ERR_INVALID, "LevelPolicy must be 0..3");
            p.levels.push_back(static_cast<LevelPolicy>(policy[i]));
        }
        h->qh->prepareForQuery(p);
        return TBLAEQ_OK;
    });
}

int tblaeq_level(tblaeq_handle* h, uint64_t l, const tblaeq_grid* in, int qtype, const double* lo, const double* hi,
                 const double* q, uint64_t K, tblaeq_grid* out) {
    if (int c = checkPrepared(h)) return c;
    if (!in || !out) return fail(TBLAEQ_ERR_INVALID, "null grid");
    if (qtype != TBLAEQ_RANGE && qtype != TBLAEQ_POINT) return fail(TBLAEQ_ERR_INVALID, "unknown query type");
    if (qtype == TBLAEQ_RANGE && (!lo || !hi)) return fail(TBLAEQ_ERR_INVALID, "range query needs lo and hi");
    if (qtype == TBLAEQ_POINT && !q) return fail(TBLAEQ_ERR_INVALID, "KNN query needs a point");
    return guarded([&]() -> int {
        B200Strategy s(h->qh->runtime());
        SparseGrid g{in->numRows, in->dim, in->nnz, in->ids, in->vals};
        const LevelResult r =
            s.runLevel(l, &g, qtype == TBLAEQ_RANGE ? QueryType::RANGE : QueryType::POINT, lo, hi, q, K);
        const std::unique_ptr<SparseGrid> grid(r.grid);  // the buffers stay with the handle
        out->numRows = grid->numRows;
        out->dim = grid->dim;
        out->nnz = grid->nnz;
        out->ids = grid->ids;
        out->vals = grid->vals;
        return TBLAEQ_OK;
    });
}

int tblaeq_coarsest_grid(tblaeq_handle* h, tblaeq_grid* out) {
    if (int c = checkPrepared(h)) return c;
    if (!out) return fail(TBLAEQ_ERR_INVALID, "null grid");
    Runtime& rt = h->qh->runtime();
    out->numRows = h->qh->index().coarsest.rows;
    out->dim = rt.dev->D;
    out->nnz = rt.dev->meshCount[0];
    out->ids = rt.dev->coarseIds.as<uint64_t>();
    out->vals = rt.dev->coarseVals.as<double>();
    return TBLAEQ_OK;
}

// A KNN batch too large for one traversal (high dimensions keep most clusters alive, so the
// frontier outgrows the 32-bit item space or the free device memory) runs as consecutive chunks,
// halved until each fits; the
// chunks' results are gathered into the handle's buffers in query order. Per-level counts are not
// kept for chunked batches.
static BatchOutput runKnnChunked(tblaeq_handle* h, const double* dQueries, uint64_t nq, const std::vector<uint32_t>& k,
                                 unsigned flags, uint64_t firstChunk) {
    Runtime& rt = h->qh->runtime();
    const uint64_t D = rt.dev->D;
    uint64_t sumK = 0;
    for (uint32_t v : k) sumK += v;
    if (h->knnIds.bytes() < std::max<uint64_t>(sumK, 1) * 8) {
        h->knnIds.alloc(std::max<uint64_t>(sumK, 1) * 8);
        h->knnD2.alloc(std::max<uint64_t>(sumK, 1) * 8);
    }
    if (h->knnOff.bytes() < (nq + 1) * 8) h->knnOff.alloc((nq + 1) * 8);
    std::vector<uint64_t> offs(nq + 1, 0), part;
    std::vector<uint64_t> sum(5, 0);
    uint64_t chunk = std::max<uint64_t>(1, std::min(firstChunk, nq)), i = 0, runs = 0;
    while (i < nq) {
        const uint64_t c = std::min(chunk, nq - i);
        uint64_t sk = 0;
        for (uint64_t q = i; q < i + c; ++q) sk += k[q];
        BatchOutput co;
        try {
            co = rt.engine->runKnn(dQueries + i * D, static_cast<uint32_t>(c), h->kStage.as<uint32_t>() + i, sk,
                                   flags & ~static_cast<unsigned>(TBLAEQ_WANT_LEVELS));
        } catch (const CudaError& e) {
            // Too large for the 32-bit traversal space or for the free device memory (the engine
            // released its workspace on the way out): halve the chunk.
            if (e.code != cudaErrorMemoryAllocation || c == 1) throw;
            h->knnSplitReason = std::to_string(c) + " queries: " + e.what();
            chunk = (c + 1) / 2;
            continue;
        }
        part.resize(c + 1);
        TBLAEQ_CUDA(cudaMemcpyAsync(part.data(), co.offsets, (c + 1) * 8, cudaMemcpyDeviceToHost, rt.stream));
        TBLAEQ_CUDA(cudaStreamSynchronize(rt.stream));
        if (part[c]) {
            TBLAEQ_CUDA(cudaMemcpyAsync(h->knnIds.as<uint64_t>() + offs[i], co.ids, part[c] * 8, cudaMemcpyDeviceToDevice,
                                        rt.stream));
            TBLAEQ_CUDA(cudaMemcpyAsync(h->knnD2.as<double>() + offs[i], co.dist2, part[c] * 8,
                                        cudaMemcpyDeviceToDevice, rt.stream));
        }
        for (uint64_t q = 0; q < c; ++q) offs[i + q + 1] = offs[i] + part[q + 1];
        const std::vector<uint64_t> cn = rt.engine->knnCounters();
        for (size_t t = 0; t < sum.size() && t < cn.size(); ++t) sum[t] += cn[t];
        i += c;
        ++runs;
    }
    h->knnSum = sum;
    // Later batches start at the size that fitted instead of failing at the full size first (each
    // failure costs the growth steps and the workspace reset before the split).
    h->knnChunkHint = chunk;
    h->knnHintTwoWave = rt.engine->twoWave();
    h->lastKnnChunk = chunk;
    h->lastKnnRuns = runs;
    TBLAEQ_CUDA(cudaMemcpyAsync(h->knnOff.get(), offs.data(), (nq + 1) * 8, cudaMemcpyHostToDevice, rt.stream));
    TBLAEQ_CUDA(cudaStreamSynchronize(rt.stream));
    BatchOutput o;
    o.nq = static_cast<uint32_t>(nq);
    o.total = offs[nq];
    o.offsets = h->knnOff.as<uint64_t>();
    o.ids = h->knnIds.as<uint64_t>();
    o.dist2 = h->knnD2.as<double>();
    return o;
}

static int runBatch(tblaeq_handle* h, const tblaeq_batch* b, const double* dQueries, tblaeq_batch_result* out) {
    Runtime& rt = h->qh->runtime();
    if (b->nq > 0xffffffffull) return fail(TBLAEQ_ERR_OVERFLOW, "too many queries in one batch");
    BatchOutput o;
    if (b->qtype == TBLAEQ_POINT) {
        if (b->mode != TBLAEQ_MODE_EXACT)
            return fail(TBLAEQ_ERR_INVALID, "batched KNN is exact; use tblaeq_level for the reference's STEP sets");
        std::vector<uint32_t> k(b->nq);
        uint64_t sumK = 0;
        for (uint64_t i = 0; i < b->nq; ++i) {
            const uint64_t v = b->kPerQuery ? b->kPerQuery[i] : b->K;
            if (v > 0xffffffffull) return fail(TBLAEQ_ERR_INVALID, "K too large");
            k[i] = static_cast<uint32_t>(v);
            sumK += v;
        }
        if (h->kStage.bytes() < std::max<size_t>(b->nq, 1) * 4) h->kStage.alloc(std::max<size_t>(b->nq, 1) * 4);
        if (b->nq)
            TBLAEQ_CUDA(cudaMemcpyAsync(h->kStage.get(), k.data(), b->nq * 4, cudaMemcpyHostToDevice, rt.stream));
        h->knnSum.clear();
        // A size learnt under the other finest-level mode (one pass or two waves) does not apply.
        const uint64_t hint = (h->knnHintTwoWave == rt.engine->twoWave()) ? h->knnChunkHint : 0;
        const uint64_t limit = (h->knnChunkMax && hint) ? std::min(h->knnChunkMax, hint)
                                                        : (h->knnChunkMax ? h->knnChunkMax : hint);
        if (limit && b->nq > limit) {
            o = runKnnChunked(h, dQueries, b->nq, k, b->flags, limit);
        } else {
            try {
                o = rt.engine->runKnn(dQueries, static_cast<uint32_t>(b->nq), h->kStage.as<uint32_t>(), sumK, b->flags);
                h->lastKnnChunk = b->nq;
                h->lastKnnRuns = 1;
            } catch (const CudaError& e) {
                if (e.code != cudaErrorMemoryAllocation || b->nq < 2) throw;
                h->knnSplitReason = std::to_string(b->nq) + " queries: " + e.what();
                o = runKnnChunked(h, dQueries, b->nq, k, b->flags, (b->nq + 1) / 2);
            }
        }
    } else {
        o = rt.engine->runRange(dQueries, static_cast<uint32_t>(b->nq), b->mode, b->flags);
    }
    h->lastNq = b->nq;
    h->lastFlags = b->flags;
    out->nq = b->nq;
    out->total = o.total;
    out->offsets = o.offsets;
    out->ids = o.ids;
    out->vals = o.vals;
    out->dist2 = o.dist2;
    out->levelItems = o.levelItems;
    return TBLAEQ_OK;
}

static int validateBatch(tblaeq_handle* h, const tblaeq_batch* b) {
    if (int c = checkPrepared(h)) return c;
    if (!b) return fail(TBLAEQ_ERR_INVALID, "null batch");
    if (b->mode != TBLAEQ_MODE_REF_PARITY && b->mode != TBLAEQ_MODE_EXACT) return fail(TBLAEQ_ERR_INVALID, "bad mode");
    if (b->qtype != TBLAEQ_RANGE && b->qtype != TBLAEQ_POINT) return fail(TBLAEQ_ERR_INVALID, "bad query type");
    if (b->nq > 0 && !b->queries) return fail(TBLAEQ_ERR_INVALID, "null queries");
    return TBLAEQ_OK;
}

int tblaeq_query_batch(tblaeq_handle* h, const tblaeq_batch* b, tblaeq_batch_result* out) {
    if (int c = validateBatch(h, b)) return c;
    if (!out) return fail(TBLAEQ_ERR_INVALID, "null result");
    return guarded([&]() -> int {
        const double* dq = b->queries;
        // Host queries, and device queries off a 16-byte boundary (the kernels read query rows in
        // 16-byte pairs), go through the handle's staging buffer.
        const bool misaligned = (reinterpret_cast<uintptr_t>(b->queries) & 15u) != 0;
        if (b->nq && (!b->queriesOnDevice || misaligned)) {
            Runtime& rt = h->qh->runtime();
            const uint64_t D = rt.dev->D;
            const size_t bytes = b->nq * (b->qtype == TBLAEQ_RANGE ? 2 * D : D) * 8;
            if (h->stage.bytes() < bytes) h->stage.alloc(bytes);
            TBLAEQ_CUDA(cudaMemcpyAsync(h->stage.get(), b->queries, bytes,
                                        b->queriesOnDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                        rt.stream));
            dq = h->stage.as<double>();
        }
        return runBatch(h, b, dq, out);
    });
}

int tblaeq_query_batch_host(tblaeq_handle* h, const tblaeq_batch* b, uint64_t* offsets_out, uint64_t* ids_out,
                            uint64_t ids_cap, double* dist2_out, uint64_t* total) {
    if (int c = validateBatch(h, b)) return c;
    if (!offsets_out || (!ids_out && ids_cap)) return fail(TBLAEQ_ERR_INVALID, "null output buffer");
    return guarded([&]() -> int {
        tblaeq_batch hb = *b;
        tblaeq_batch_result r{};
        int c = tblaeq_query_batch(h, &hb, &r);
        if (c) return c;
        Runtime& rt = h->qh->runtime();
        TBLAEQ_CUDA(cudaMemcpyAsync(offsets_out, r.offsets, (b->nq + 1) * 8, cudaMemcpyDeviceToHost, rt.stream));
        const uint64_t n = std::min<uint64_t>(r.total, ids_cap);
        if (n) TBLAEQ_CUDA(cudaMemcpyAsync(ids_out, r.ids, n * 8, cudaMemcpyDeviceToHost, rt.stream));
        if (n && dist2_out && r.dist2)
            TBLAEQ_CUDA(cudaMemcpyAsync(dist2_out, r.dist2, n * 8, cudaMemcpyDeviceToHost, rt.stream));
        TBLAEQ_CUDA(cudaStreamSynchronize(rt.stream));
        if (total) *total = r.total;
        if (r.total > ids_cap) return fail(TBLAEQ_ERR_OVERFLOW, "result ids exceed ids_cap");
        return TBLAEQ_OK;
    });
}

int tblaeq_query_batch_async(tblaeq_handle* h, const tblaeq_batch* b) {
    if (int c = validateBatch(h, b)) return c;
    if (!b->queriesOnDevice && b->nq) return fail(TBLAEQ_ERR_INVALID, "async batches need device queries");
    if (reinterpret_cast<uintptr_t>(b->queries) & 15u)
        return fail(TBLAEQ_ERR_INVALID, "async batches need device queries on a 16-byte boundary");
    // A KNN batch may split into chunks with host synchronisation between them: synchronous only.
    if (b->qtype != TBLAEQ_RANGE)
        return fail(TBLAEQ_ERR_INVALID, "asynchronous batches are range batches; run KNN with tblaeq_query_batch");
    return guarded([&]() -> int {
        Runtime& rt = h->qh->runtime();
        h->lastNq = b->nq;
        h->lastFlags = b->flags;
        rt.engine->enqueueRange(b->queries, static_cast<uint32_t>(b->nq), b->mode, b->flags);
        return TBLAEQ_OK;
    });
}

int tblaeq_graph_launches(tblaeq_handle* h, uint64_t* kernels, uint64_t* nodes) {
    if (int c = checkPrepared(h)) return c;
    const BatchEngine& e = *h->qh->runtime().engine;
    if (kernels) *kernels = e.graphKernels();
    if (nodes) *nodes = e.graphNodes();
    return TBLAEQ_OK;
}

uint64_t tblaeq_kernel_launches(void) { return gKernelLaunches.load(std::memory_order_relaxed); }

int tblaeq_batch_wait(tblaeq_handle* h, tblaeq_batch_result* out) {
    if (int c = checkPrepared(h)) return c;
    return guarded([&]() -> int {
        Runtime& rt = h->qh->runtime();
        const uint32_t st = rt.engine->status();
        const uint32_t over = st & (kStatusOverflowEntries | kStatusOverflowItems | kStatusOverflowSum);
        if ((st & (kStatusLookbackTimeout | kStatusWindowOverflow)) && !over)
            return fail(TBLAEQ_ERR_TIMEOUT, "traversal kernel reported status " + std::to_string(st));
        if (st) return fail(TBLAEQ_ERR_OVERFLOW, "workspace overflow; rerun with tblaeq_query_batch");
        if (out) {
            const BatchOutput o = rt.engine->output(static_cast<uint32_t>(h->lastNq), h->lastFlags);
            out->nq = h->lastNq;
            out->total = rt.engine->lastTotal(static_cast<uint32_t>(h->lastNq));
            out->offsets = o.offsets;
            out->ids = o.ids;
            out->vals = o.vals;
            out->dist2 = o.dist2;
            out->levelItems = o.levelItems;
        }
        return TBLAEQ_OK;
    });
}

int tblaeq_level_counts(tblaeq_handle* h, uint64_t* entries, uint64_t* items, int cap, uint64_t* results) {
    if (int c = checkPrepared(h)) return -c;
    int n = 0;
    const int c = guarded([&]() -> int {
        std::vector<uint64_t> e, it;
        uint64_t r = 0;
        h->qh->runtime().engine->levelCounts(e, it, r);
        n = std::min<int>(cap, static_cast<int>(e.size()));
        for (int i = 0; i < n; ++i) {
            if (entries) entries[i] = e[i];
            if (items) items[i] = it[i];
        }
        if (results) *results = r;
        return TBLAEQ_OK;
    });
    return c == TBLAEQ_OK ? n : -c;
}

int tblaeq_set_device(int device) {
    return guarded([&]() -> int {
        TBLAEQ_CUDA(cudaSetDevice(device));
        return TBLAEQ_OK;
    });
}

void* tblaeq_stream(tblaeq_handle* h) {
    if (!h || !h->qh || !h->qh->prepared()) return nullptr;
    return h->qh->runtime().stream;
}

int tblaeq_set_timing(tblaeq_handle* h, int on) {
    if (int c = checkPrepared(h)) return c;
    return guarded([&]() -> int {
        h->qh->runtime().engine->setTiming(on != 0);
        return TBLAEQ_OK;
    });
}

int tblaeq_stage_times(tblaeq_handle* h, float* ms, int cap) {
    if (!h || !h->qh || !h->qh->prepared() || !ms) return -1;
    int n = -1;
    const int c = guarded([&]() -> int {
        const std::vector<float> t = h->qh->runtime().engine->stageTimes();
        if (t.empty()) return TBLAEQ_ERR_STATE;
        n = std::min<int>(cap, static_cast<int>(t.size()));
        for (int i = 0; i < n; ++i) ms[i] = t[i];
        return TBLAEQ_OK;
    });
    return c == TBLAEQ_OK ? n : -1;
}

int tblaeq_autotune(tblaeq_handle* h, const tblaeq_batch* b, int reps, int* variants_out, float* ms_out) {
    if (int c = validateBatch(h, b)) return c;
    if (!b->queriesOnDevice || b->qtype != TBLAEQ_RANGE)
        return fail(TBLAEQ_ERR_INVALID, "autotune needs a range batch with device queries");
    return guarded([&]() -> int {
        Runtime& rt = h->qh->runtime();
        const std::vector<float> t =
            rt.engine->autotuneRange(b->queries, static_cast<uint32_t>(b->nq), b->mode, b->flags, reps);
        const std::vector<int>& v = rt.engine->variants();
        for (size_t i = 0; i < v.size(); ++i) {
            if (variants_out) variants_out[i] = v[i];
            if (ms_out) ms_out[i] = t[i];
        }
        return TBLAEQ_OK;
    });
}

int tblaeq_set_variants(tblaeq_handle* h, const int* variants, uint64_t n) {
    if (int c = checkPrepared(h)) return c;
    if (!variants) return fail(TBLAEQ_ERR_INVALID, "null variants");
    return guarded([&]() -> int {
        h->qh->runtime().engine->setVariants(std::vector<int>(variants, variants + n));
        return TBLAEQ_OK;
    });
}

int tblaeq_set_knn_probe(tblaeq_handle* h, uint32_t beam, int node_major_completion) {
    if (int c = checkPrepared(h)) return c;
    return guarded([&]() -> int {
        h->qh->runtime().engine->setKnnProbe(beam, node_major_completion != 0);
        return TBLAEQ_OK;
    });
}

int tblaeq_set_node_major(tblaeq_handle* h, int on) {
    if (int c = checkPrepared(h)) return c;
    h->qh->runtime().engine->setNodeMajor(on != 0);
    return TBLAEQ_OK;
}

int tblaeq_set_float_points(tblaeq_handle* h, int on) {
    if (int c = checkPrepared(h)) return c;
    h->qh->runtime().engine->setFloatPoints(on != 0);
    return TBLAEQ_OK;
}

int tblaeq_set_point_groups(tblaeq_handle* h, int on) {
    if (int c = checkPrepared(h)) return c;
    h->qh->runtime().engine->setPointGroups(on != 0);
    h->qh->runtime().engine->setKnnGroups(on != 0);
    return TBLAEQ_OK;
}

int tblaeq_group_counts(tblaeq_handle* h, uint64_t* out3) {
    if (int c = checkPrepared(h)) return c;
    if (!out3) return fail(TBLAEQ_ERR_INVALID, "null output");
    return guarded([&]() -> int {
        const std::vector<uint64_t> v = h->qh->runtime().engine->groupCounts();
        for (int i = 0; i < 3; ++i) out3[i] = v[i];
        return TBLAEQ_OK;
    });
}

int tblaeq_set_launch_shapes(tblaeq_handle* h, const int* variants, const int* grid_percent, uint64_t n) {
    if (int c = checkPrepared(h)) return c;
    if (!variants || !grid_percent) return fail(TBLAEQ_ERR_INVALID, "null launch shapes");
    return guarded([&]() -> int {
        h->qh->runtime().engine->setLaunchShapes(std::vector<int>(variants, variants + n),
                                                 std::vector<int>(grid_percent, grid_percent + n));
        return TBLAEQ_OK;
    });
}

int tblaeq_get_launch_shapes(tblaeq_handle* h, int* variants, int* grid_percent, uint64_t cap) {
    if (int c = checkPrepared(h)) return c;
    if (!variants || !grid_percent) return fail(TBLAEQ_ERR_INVALID, "null output");
    const BatchEngine& e = *h->qh->runtime().engine;
    if (cap < e.variants().size()) return fail(TBLAEQ_ERR_INVALID, "output smaller than the index height");
    for (size_t i = 0; i < e.variants().size(); ++i) {
        variants[i] = e.variants()[i];
        grid_percent[i] = e.gridPercents()[i];
    }
    return TBLAEQ_OK;
}

int tblaeq_tuning_key(tblaeq_handle* h, int mode, uint64_t nq, char* buf, uint64_t cap) {
    if (!h || !h->qh) return fail(TBLAEQ_ERR_INVALID, "null handle");
    if (!buf) return fail(TBLAEQ_ERR_INVALID, "null buffer");
    return guarded([&]() -> int {
        int dev = 0;
        TBLAEQ_CUDA(cudaGetDevice(&dev));
        cudaDeviceProp prop{};
        TBLAEQ_CUDA(cudaGetDeviceProperties(&prop, dev));
        const HostIndex& x = h->qh->index();
        uint64_t bucket = 1;
        while (bucket < nq) bucket <<= 1;
        std::string key = std::string(prop.name) + "/" + std::to_string(prop.multiProcessorCount) + "sm|N=" +
                          std::to_string(x.N) + "|D=" + std::to_string(x.D) + "|H=" + std::to_string(x.height) +
                          "|ratios=";
        for (size_t i = 0; i < x.ratios.size(); ++i) key += (i ? "," : "") + std::to_string(x.ratios[i]);
        key += "|mode=" + std::to_string(mode) + "|nq=" + std::to_string(bucket);
        for (char& c : key)
            if (c == '\t' || c == '\n' || c == '\r') c = ' ';
        if (key.size() + 1 > cap) return fail(TBLAEQ_ERR_INVALID, "key buffer too small");
        std::memcpy(buf, key.c_str(), key.size() + 1);
        return TBLAEQ_OK;
    });
}

int tblaeq_tuning_store(const char* path, const char* key, const int* variants, const int* grid_percent, uint64_t n) {
    if (!path || !key || !variants || !grid_percent) return fail(TBLAEQ_ERR_INVALID, "null argument");
    return guarded([&]() -> int {
        LaunchShapes s;
        s.variants.assign(variants, variants + n);
        s.gridPercent.assign(grid_percent, grid_percent + n);
        tuningStore(path, key, s);
        return TBLAEQ_OK;
    });
}

int tblaeq_tuning_lookup(const char* path, const char* key, int* variants, int* grid_percent, uint64_t cap,
                         uint64_t* n) {
    if (!path || !key || !n) return fail(TBLAEQ_ERR_INVALID, "null argument");
    return guarded([&]() -> int {
        *n = 0;
        LaunchShapes s;
        if (!tuningLookup(path, key, s)) return TBLAEQ_OK;
        if (cap < s.variants.size() || !variants || !grid_percent)
            return fail(TBLAEQ_ERR_INVALID, "output smaller than the cached entry");
        for (size_t i = 0; i < s.variants.size(); ++i) {
            variants[i] = s.variants[i];
            grid_percent[i] = s.gridPercent[i];
        }
        *n = s.variants.size();
        return TBLAEQ_OK;
    });
}

int tblaeq_set_two_wave(tblaeq_handle* h, int on) {
    if (int c = checkPrepared(h)) return c;
    h->qh->runtime().engine->setTwoWave(on != 0);
    return TBLAEQ_OK;
}

int tblaeq_set_knn_wave1(tblaeq_handle* h, double scale) {
    if (int c = checkPrepared(h)) return c;
    if (!(scale > 0.0) || scale > 1e6) return fail(TBLAEQ_ERR_INVALID, "wave-1 scale must be in (0, 1e6]");
    h->qh->runtime().engine->setWaveScale(scale);
    return TBLAEQ_OK;
}

int tblaeq_set_knn_refine(tblaeq_handle* h, uint32_t stride) {
    if (int c = checkPrepared(h)) return c;
    h->qh->runtime().engine->setKnnRefine(stride, h->qh->runtime().engine->knnRefineStages());
    return TBLAEQ_OK;
}

int tblaeq_set_knn_refine_stages(tblaeq_handle* h, uint32_t stages) {
    if (int c = checkPrepared(h)) return c;
    if (stages < 1 || stages > kMaxRefineStages) return fail(TBLAEQ_ERR_INVALID, "refine stages must be in [1, 4]");
    auto& e = *h->qh->runtime().engine;
    e.setKnnRefine(e.knnRefine(), stages);
    return TBLAEQ_OK;
}

int tblaeq_set_knn_chunk(tblaeq_handle* h, uint64_t max_queries) {
    if (int c = checkPrepared(h)) return c;
    h->knnChunkMax = max_queries;
    if (max_queries == 0) h->knnChunkHint = 0;
    return TBLAEQ_OK;
}

int tblaeq_knn_split_reason(tblaeq_handle* h, char* buf, uint64_t cap) {
    if (int c = checkPrepared(h)) return c;
    if (!buf || cap == 0) return fail(TBLAEQ_ERR_INVALID, "null output");
    const size_t n = std::min<size_t>(cap - 1, h->knnSplitReason.size());
    std::memcpy(buf, h->knnSplitReason.data(), n);
    buf[n] = '\0';
    return TBLAEQ_OK;
}

int tblaeq_last_batch_runs(tblaeq_handle* h, uint64_t* runs) {
    if (int c = checkPrepared(h)) return c;
    if (!runs) return fail(TBLAEQ_ERR_INVALID, "null output");
    *runs = h->qh->runtime().engine->lastRuns();
    return TBLAEQ_OK;
}

int tblaeq_knn_batch_info(tblaeq_handle* h, uint64_t* out2) {
    if (int c = checkPrepared(h)) return c;
    if (!out2) return fail(TBLAEQ_ERR_INVALID, "null output");
    out2[0] = h->lastKnnChunk;
    out2[1] = h->lastKnnRuns;
    return TBLAEQ_OK;
}

int tblaeq_knn_counters(tblaeq_handle* h, uint64_t* out5) {
    if (int c = checkPrepared(h)) return c;
    if (!out5) return fail(TBLAEQ_ERR_INVALID, "null output");
    return guarded([&]() -> int {
        const std::vector<uint64_t> v = h->knnSum.empty() ? h->qh->runtime().engine->knnCounters() : h->knnSum;
        for (int i = 0; i < 5; ++i) out5[i] = v[i];
        return TBLAEQ_OK;
    });
}

int tblaeq_scorer_train(tblaeq_handle* h, const double* points, uint64_t nq, const uint32_t* k_per_query, uint64_t K,
                        uint64_t max_samples, int epochs, float lr, uint64_t seed, float* loss_out) {
    if (int c = checkPrepared(h)) return c;
    if (!points || nq == 0 || nq > 0xffffffffull || epochs < 1 || max_samples == 0)
        return fail(TBLAEQ_ERR_INVALID, "scorer training needs queries, epochs >= 1 and samples > 0");
    return guarded([&]() -> int {
        Runtime& rt = h->qh->runtime();
        std::vector<uint32_t> k(nq);
        for (uint64_t i = 0; i < nq; ++i) k[i] = static_cast<uint32_t>(k_per_query ? k_per_query[i] : K);
        ScorerTrainConfig cfg;
        cfg.maxSamples = max_samples;
        cfg.epochs = epochs;
        cfg.lr = lr;
        cfg.seed = seed;
        const std::vector<float> losses = trainScorer(rt, points, static_cast<uint32_t>(nq), k, cfg);
        if (loss_out) std::copy(losses.begin(), losses.end(), loss_out);
        enableScorer(rt, true);
        return TBLAEQ_OK;
    });
}

int tblaeq_scorer_stats(tblaeq_handle* h, uint64_t* samples, uint64_t* positives) {
    if (int c = checkPrepared(h)) return c;
    Runtime& rt = h->qh->runtime();
    if (samples) *samples = rt.scorerSamples;
    if (positives) *positives = rt.scorerPositives;
    return TBLAEQ_OK;
}

namespace {
constexpr char kScorerMagic[8] = {'T', 'B', 'L', 'Q', 'S', 'C', 'R', '1'};
}

int tblaeq_scorer_save(tblaeq_handle* h, const char* path) {
    if (int c = checkPrepared(h)) return c;
    if (!path) return fail(TBLAEQ_ERR_INVALID, "null path");
    return guarded([&]() -> int {
        Runtime& rt = h->qh->runtime();
        if (!rt.scorer) return fail(TBLAEQ_ERR_STATE, "no scorer to save (train or load one first)");
        const std::vector<float> p = rt.scorer->getParams();
        FILE* f = std::fopen(path, "wb");
        if (!f) return fail(TBLAEQ_ERR_IO, std::string("Cannot write ") + path);
        const uint64_t head[5] = {static_cast<uint64_t>(rt.scorer->shape().D),
                                  static_cast<uint64_t>(rt.scorer->shape().levels), p.size(), rt.scorerSamples,
                                  rt.scorerPositives};
        bool ok = std::fwrite(kScorerMagic, 1, 8, f) == 8 && std::fwrite(head, 8, 5, f) == 5 &&
                  std::fwrite(&rt.scorerInvScale, 8, 1, f) == 1 && std::fwrite(p.data(), 4, p.size(), f) == p.size();
        ok = (std::fclose(f) == 0) && ok;
        return ok ? TBLAEQ_OK : fail(TBLAEQ_ERR_IO, std::string("Short write ") + path);
    });
}

int tblaeq_scorer_load(tblaeq_handle* h, const char* path) {
    if (int c = checkPrepared(h)) return c;
    if (!path) return fail(TBLAEQ_ERR_INVALID, "null path");
    return guarded([&]() -> int {
        Runtime& rt = h->qh->runtime();
        FILE* f = std::fopen(path, "rb");
        if (!f) return fail(TBLAEQ_ERR_IO, std::string("Cannot read ") + path);
        char magic[8];
        uint64_t head[5];
        double inv = 0.0;
        bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kScorerMagic, 8) == 0 &&
                  std::fread(head, 8, 5, f) == 5 && std::fread(&inv, 8, 1, f) == 1;
        Mlp& m = ensureScorer(rt);
        ok = ok && head[0] == static_cast<uint64_t>(m.shape().D) && head[1] == static_cast<uint64_t>(m.shape().levels) &&
             head[2] == m.shape().params();
        std::vector<float> p(ok ? head[2] : 0);
        ok = ok && std::fread(p.data(), 4, p.size(), f) == p.size();
        std::fclose(f);
        if (!ok) return fail(TBLAEQ_ERR_IO, std::string("Invalid index: scorer file ") + path +
                                                " is truncated or was trained for another index shape");
        m.setParams(p, rt.stream);
        rt.scorerInvScale = inv;
        rt.scorerSamples = head[3];
        rt.scorerPositives = head[4];
        enableScorer(rt, true);
        TBLAEQ_CUDA(cudaStreamSynchronize(rt.stream));
        return TBLAEQ_OK;
    });
}

int tblaeq_scorer_enable(tblaeq_handle* h, int on) {
    if (int c = checkPrepared(h)) return c;
    return guarded([&]() -> int {
        enableScorer(h->qh->runtime(), on != 0);
        return TBLAEQ_OK;
    });
}

int tblaeq_scorer_get_params(tblaeq_handle* h, float* out, uint64_t cap, uint64_t* n) {
    if (int c = checkPrepared(h)) return c;
    return guarded([&]() -> int {
        const std::vector<float> p = ensureScorer(h->qh->runtime()).getParams();
        if (n) *n = p.size();
        if (out) std::copy(p.begin(), p.begin() + std::min<uint64_t>(cap, p.size()), out);
        return TBLAEQ_OK;
    });
}

int tblaeq_scorer_set_params(tblaeq_handle* h, const float* params, uint64_t n) {
    if (int c = checkPrepared(h)) return c;
    if (!params) return fail(TBLAEQ_ERR_INVALID, "null parameters");
    return guarded([&]() -> int {
        Runtime& rt = h->qh->runtime();
        ensureScorer(rt).setParams(std::vector<float>(params, params + n), rt.stream);
        return TBLAEQ_OK;
    });
}

int tblaeq_scorer_loss_grad(tblaeq_handle* h, const float* X, const float* y, uint64_t n, float* grad_out,
                            float* loss_out) {
    if (int c = checkPrepared(h)) return c;
    if (!X || !y || !grad_out || n == 0 || n > 0xffffffffull) return fail(TBLAEQ_ERR_INVALID, "bad samples");
    return guarded([&]() -> int {
        Runtime& rt = h->qh->runtime();
        Mlp& m = ensureScorer(rt);
        const int in = m.shape().in();
        DeviceMem dX(n * in * 4), dy(n * 4), dg(m.shape().params() * 4);
        TBLAEQ_CUDA(cudaMemcpyAsync(dX.get(), X, n * in * 4, cudaMemcpyHostToDevice, rt.stream));
        TBLAEQ_CUDA(cudaMemcpyAsync(dy.get(), y, n * 4, cudaMemcpyHostToDevice, rt.stream));
        const float loss = m.lossAndGrad(dX.as<float>(), dy.as<float>(), static_cast<uint32_t>(n), dg.as<float>(), rt.stream);
        TBLAEQ_CUDA(cudaMemcpyAsync(grad_out, dg.get(), m.shape().params() * 4, cudaMemcpyDeviceToHost, rt.stream));
        TBLAEQ_CUDA(cudaStreamSynchronize(rt.stream));
        if (loss_out) *loss_out = loss;
        return TBLAEQ_OK;
    });
}

static int scorerLogits(tblaeq_handle* h, const float* X, uint64_t n, float* z_out, bool tensor) {
    if (int c = checkPrepared(h)) return c;
    if (!X || !z_out || n > 0xffffffffull) return fail(TBLAEQ_ERR_INVALID, "bad samples");
    return guarded([&]() -> int {
        Runtime& rt = h->qh->runtime();
        Mlp& m = ensureScorer(rt);
        const int in = m.shape().in();
        DeviceMem dX(std::max<uint64_t>(n, 1) * in * 4), dz(std::max<uint64_t>(n, 1) * 4);
        TBLAEQ_CUDA(cudaMemcpyAsync(dX.get(), X, n * in * 4, cudaMemcpyHostToDevice, rt.stream));
        if (tensor)
            m.logitsTensor(dX.as<float>(), static_cast<uint32_t>(n), dz.as<float>(), rt.stream);
        else
            m.logits(dX.as<float>(), static_cast<uint32_t>(n), dz.as<float>(), rt.stream);
        TBLAEQ_CUDA(cudaMemcpyAsync(z_out, dz.get(), n * 4, cudaMemcpyDeviceToHost, rt.stream));
        TBLAEQ_CUDA(cudaStreamSynchronize(rt.stream));
        if (tensor && m.tensorStatus(rt.stream)) return fail(TBLAEQ_ERR_TIMEOUT, "tensor-core scorer gave up waiting");
        return TBLAEQ_OK;
    });
}

int tblaeq_scorer_logits(tblaeq_handle* h, const float* X, uint64_t n, float* z_out) {
    return scorerLogits(h, X, n, z_out, false);
}

int tblaeq_scorer_logits_tensor(tblaeq_handle* h, const float* X, uint64_t n, float* z_out) {
    return scorerLogits(h, X, n, z_out, true);
}

int tblaeq_host_array(const tblaeq_handle* h, int which, uint64_t l, const void** ptr, uint64_t* count) {
    if (!h || !ptr || !count) return fail(TBLAEQ_ERR_INVALID, "null argument");
    const HostIndex& x = h->qh->index();
    switch (which) {
        case 0:
            if (l >= x.intervals) break;
            *ptr = x.pTensors[l].vals.data();
            *count = x.pTensors[l].vals.size();
            return TBLAEQ_OK;
        case 1:
            if (l >= x.intervals) break;
            *ptr = x.pTensors[l].colRes.data();
            *count = x.pTensors[l].colRes.size();
            return TBLAEQ_OK;
        case 2:
            if (l >= x.intervals) break;
            *ptr = x.radius[l].data();
            *count = x.radius[l].size();
            return TBLAEQ_OK;
        case 3:
            if (l == 0 || l >= x.height) break;
            *ptr = x.maps[l].data();
            *count = x.maps[l].size();
            return TBLAEQ_OK;
        case 4:
            *ptr = x.coarsest.ids.data();
            *count = x.coarsest.ids.size();
            return TBLAEQ_OK;
        case 5:
            *ptr = x.coarsest.vals.data();
            *count = x.coarsest.vals.size();
            return TBLAEQ_OK;
        default:
            break;
    }
    return fail(TBLAEQ_ERR_INVALID, "no such host array");
}

int tblaeq_decode_points(tblaeq_handle* h, const uint64_t* positions, uint64_t n, double* coords_out,
                         uint64_t* ids_out) {
    if (!h || (n && (!positions || !coords_out))) return fail(TBLAEQ_ERR_INVALID, "null argument");
    return guarded([&]() -> int {
        const HostIndex& x = h->qh->index();
        const uint64_t H = x.height, D = x.D;
        if (h->parent.empty()) {
            h->posOf.resize(H);
            for (uint64_t m = 0; m + 1 < H; ++m) {
                const uint64_t cnt = x.meshCount(m);
                h->posOf[m].resize(cnt);
                for (uint64_t s = 0; s < cnt; ++s) h->posOf[m][m == 0 ? x.coarsest.ids[s] : x.maps[m][s]] = s;
            }
            h->parent.resize(H);
            for (uint64_t m = 1; m < H; ++m) {
                const PTensor& P = x.pTensors[m - 1];
                h->parent[m].resize(P.rows);
                for (uint64_t o = 0; o < P.cols; ++o)
                    for (uint64_t j = P.colRes[o]; j < P.colRes[o + 1]; ++j)
                        h->parent[m][j] = static_cast<uint32_t>(h->posOf[m - 1][o]);
            }
        }
        const uint64_t nLeaf = x.meshCount(H - 1);
        std::vector<uint64_t> chain(H);
        std::vector<double> v(D);
        for (uint64_t i = 0; i < n; ++i) {
            if (positions[i] >= nLeaf) return fail(TBLAEQ_ERR_INVALID, "position out of range");
            chain[H - 1] = positions[i];
            for (uint64_t m = H - 1; m > 0; --m) chain[m - 1] = h->parent[m][chain[m]];
            for (uint64_t d = 0; d < D; ++d) v[d] = x.coarsest.vals[chain[0] * D + d];
            for (uint64_t m = 1; m < H; ++m)
                for (uint64_t d = 0; d < D; ++d) v[d] = x.pTensors[m - 1].vals[chain[m] * D + d] * v[d];
            for (uint64_t d = 0; d < D; ++d) coords_out[i * D + d] = v[d];
            if (ids_out) ids_out[i] = x.maps[H - 1][positions[i]];
        }
        return TBLAEQ_OK;
    });
}

int tblaeq_level_range_noalloc(tblaeq_handle* h, uint64_t l, const tblaeq_grid* in, const double* lo,
                               const double* hi, uint64_t* out_ids, double* out_vals, uint64_t out_cap,
                               uint64_t* out_n) {
    if (!h || !h->qh) return fail(TBLAEQ_ERR_INVALID, "null handle");
    if (!in || !lo || !hi || !out_n || (out_cap && (!out_ids || !out_vals)))
        return fail(TBLAEQ_ERR_INVALID, "null argument");
    // A grid of another dimension would make the first expand read nnz * D doubles from a buffer
    // holding nnz * dim: reject it before any launch (and before the state check), as tblaeq_level does.
    if (in->dim != h->qh->index().D)
        return fail(TBLAEQ_ERR_INVALID, "grid dimension mismatch: grid has " + std::to_string(in->dim) +
                                            ", index has " + std::to_string(h->qh->index().D));
    if (int c = checkPrepared(h)) return c;
    return guarded([&]() -> int {
        try {
            *out_n = runLevelRangeNoAlloc(h->qh->runtime(), l, in->ids, in->vals, in->nnz, lo, hi, out_ids, out_vals,
                                          out_cap);
        } catch (const NoAllocOverflow& e) {
            return fail(TBLAEQ_ERR_OVERFLOW, e.what());
        }
        return TBLAEQ_OK;
    });
}

uint64_t tblaeq_live_device_bytes(void) { return liveDeviceBytes(); }

int tblaeq_debug_split_above(tblaeq_handle* h, uint64_t limit) {
    if (int c = checkPrepared(h)) return c;
    h->qh->runtime().engine->setSplitLimit(limit ? limit : 0xffffffffull);
    h->knnChunkHint = 0;  // a size learnt under another limit does not carry over
    return TBLAEQ_OK;
}

void tblaeq_debug_lookback_timeout(uint64_t withhold_tile, uint64_t spin_limit) {
    const bool off = withhold_tile >= 0xffffffffull || spin_limit == 0;
    setLookbackTestHook(off ? 0xffffffffu : static_cast<uint32_t>(withhold_tile),
                        off ? 0u : static_cast<uint32_t>(std::min<uint64_t>(spin_limit, 0xffffffffull)));
}

void tblaeq_debug_fail_alloc_after(uint64_t n) {
    if (n == 0) {
        setAllocHook(nullptr);
        return;
    }
    auto counter = std::make_shared<uint64_t>(n);
    setAllocHook([counter](size_t) { return --(*counter) > 0; });
}

}  // extern "C"

struct tblaeq_server {
    std::unique_ptr<tblaeq::Server> server;
};

extern "C" {

int tblaeq_serve_start(tblaeq_handle* h, const tblaeq_serve_config* cfg, tblaeq_server** out) {
    if (int c = checkPrepared(h)) return c;
    if (!out) return fail(TBLAEQ_ERR_INVALID, "null output");
    return guarded([&]() -> int {
        ServeConfig sc;
        if (cfg) {
            if (cfg->max_batch) sc.maxBatch = cfg->max_batch;
            sc.memoryBudget = cfg->memory_budget;
            if (cfg->mode != TBLAEQ_MODE_REF_PARITY && cfg->mode != TBLAEQ_MODE_EXACT)
                return fail(TBLAEQ_ERR_INVALID, "bad mode");
            sc.mode = cfg->mode;
            sc.learned = cfg->learned != 0;
            if (cfg->lanes) sc.lanes = cfg->lanes;
            sc.levels = cfg->levels != 0;
        }
        auto s = std::make_unique<tblaeq_server>();
        s->server = std::make_unique<Server>(h->qh->runtime(), sc);
        *out = s.release();
        return TBLAEQ_OK;
    });
}

int tblaeq_serve_submit(tblaeq_server* s, int qtype, const double* query, uint64_t K, uint64_t* ticket) {
    if (!s || !s->server) return fail(TBLAEQ_ERR_INVALID, "null server");
    if (K > 0xffffffffull) return fail(TBLAEQ_ERR_INVALID, "K too large");
    return guarded([&]() -> int {
        const uint64_t t = s->server->submit(qtype, query, static_cast<uint32_t>(K), Server::Clock::now());
        if (ticket) *ticket = t;
        return TBLAEQ_OK;
    });
}

int tblaeq_serve_replay(tblaeq_server* s, uint64_t n, const int* qtypes, const double* queries,
                        const uint64_t* offsets, const uint32_t* K, const double* arrival_us, uint64_t* tickets) {
    if (!s || !s->server) return fail(TBLAEQ_ERR_INVALID, "null server");
    if (n && (!qtypes || !queries || !offsets || !arrival_us)) return fail(TBLAEQ_ERR_INVALID, "null argument");
    return guarded([&]() -> int {
        const std::vector<uint64_t> t = s->server->replay(n, qtypes, queries, offsets, K, arrival_us);
        if (tickets) std::copy(t.begin(), t.end(), tickets);
        return TBLAEQ_OK;
    });
}

static int servePoll(tblaeq_server* s, uint64_t ticket, int wait_ms, uint64_t* ids_out, double* dist2_out,
                     uint64_t cap, uint64_t* n_out, double* latency_us, uint32_t* levels_out, uint64_t levels_cap,
                     uint64_t* n_levels) {
    if (!s || !s->server) return fail(TBLAEQ_ERR_INVALID, "null server");
    return guarded([&]() -> int {
        Server::Result r;
        if (!s->server->poll(ticket, r, wait_ms)) return fail(TBLAEQ_ERR_TIMEOUT, "request not done yet");
        if (latency_us) *latency_us = r.latencyUs;
        if (n_out) *n_out = r.ids.size();
        if (n_levels) *n_levels = r.levels.size();
        if (r.status != 0) return fail(r.status, r.error);
        if (r.ids.size() > cap) {
            // Keep the result for a call with a larger buffer.
            const uint64_t need = r.ids.size();
            s->server->repost(ticket, std::move(r));
            if (n_out) *n_out = need;
            return fail(TBLAEQ_ERR_OVERFLOW, "result larger than cap");
        }
        if (ids_out && !r.ids.empty()) std::copy(r.ids.begin(), r.ids.end(), ids_out);
        if (dist2_out && !r.dist2.empty()) std::copy(r.dist2.begin(), r.dist2.end(), dist2_out);
        if (levels_out)
            std::copy_n(r.levels.begin(), std::min<uint64_t>(levels_cap, r.levels.size()), levels_out);
        return TBLAEQ_OK;
    });
}

int tblaeq_serve_poll(tblaeq_server* s, uint64_t ticket, int wait_ms, uint64_t* ids_out, double* dist2_out,
                      uint64_t cap, uint64_t* n_out, double* latency_us) {
    return servePoll(s, ticket, wait_ms, ids_out, dist2_out, cap, n_out, latency_us, nullptr, 0, nullptr);
}

int tblaeq_serve_poll_levels(tblaeq_server* s, uint64_t ticket, int wait_ms, uint64_t* ids_out, double* dist2_out,
                             uint64_t cap, uint64_t* n_out, double* latency_us, uint32_t* levels_out,
                             uint64_t levels_cap, uint64_t* n_levels) {
    return servePoll(s, ticket, wait_ms, ids_out, dist2_out, cap, n_out, latency_us, levels_out, levels_cap,
                     n_levels);
}

int tblaeq_serve_wait_idle(tblaeq_server* s, int wait_ms) {
    if (!s || !s->server) return fail(TBLAEQ_ERR_INVALID, "null server");
    return guarded([&]() -> int {
        return s->server->waitIdle(wait_ms) ? TBLAEQ_OK : fail(TBLAEQ_ERR_TIMEOUT, "requests still in flight");
    });
}

int tblaeq_serve_stats(tblaeq_server* s, int reset, tblaeq_serve_metrics* out) {
    if (!s || !s->server || !out) return fail(TBLAEQ_ERR_INVALID, "null argument");
    return guarded([&]() -> int {
        const ServeStats st = s->server->stats(reset != 0);
        out->submitted = st.submitted;
        out->completed = st.completed;
        out->failed = st.failed;
        out->batches = st.batches;
        out->max_batch = st.maxBatch;
        out->mean_batch = st.meanBatch;
        out->p50_us = st.p50Us;
        out->p99_us = st.p99Us;
        out->mean_us = st.meanUs;
        out->max_us = st.maxUs;
        out->span_s = st.spanS;
        return TBLAEQ_OK;
    });
}

int tblaeq_serve_stop(tblaeq_server* s) {
    if (!s) return fail(TBLAEQ_ERR_INVALID, "null server");
    return guarded([&]() -> int {
        if (s->server) s->server->stop();
        delete s;
        return TBLAEQ_OK;
    });
}

}  // extern "C"

extern "C" {

static KmeansConfig kmeansConfigOf(const tblaeq_build_config* cfg) {
    KmeansConfig c;
    if (cfg) {
        if (cfg->iters > 0) c.iters = cfg->iters;
        c.seed = cfg->seed;
        c.precision = cfg->precision;
        c.hostAssembly = cfg->host_assembly;
    }
    return c;
}

int tblaeq_kmeans_build(const float* points, uint64_t N, uint64_t D, uint64_t height, const uint64_t* ratios,
                        const tblaeq_build_config* cfg, tblaeq_handle** out, tblaeq_build_report* report) {
    if (!points || !out || (height > 1 && !ratios)) return fail(TBLAEQ_ERR_INVALID, "null argument");
    if (cfg && (cfg->precision < 0 || cfg->precision > 2)) return fail(TBLAEQ_ERR_INVALID, "bad precision");
    if (cfg && (cfg->host_assembly < 0 || cfg->host_assembly > 2)) return fail(TBLAEQ_ERR_INVALID, "bad host_assembly");
    *out = nullptr;
    return guarded([&]() -> int {
        const KmeansConfig c = kmeansConfigOf(cfg);
        std::vector<uint64_t> r(ratios, ratios + (height > 1 ? height - 1 : 0));
        std::vector<KmeansLevelReport> reps;
        cudaStream_t s = nullptr;
        TBLAEQ_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        HostIndex idx;
        try {
            idx = kmeansBuild(points, N, D, height, r, c, reps, s);
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
        if (report) {
            for (size_t i = 0; i < reps.size(); ++i) {
                report[i].n = reps[i].n;
                report[i].k = reps[i].k;
                report[i].iters = reps[i].iters;
                report[i].objective = reps[i].objective;
                report[i].assign_seconds = reps[i].assignSeconds;
                report[i].assemble_seconds = reps[i].assembleSeconds;
                report[i].seconds = reps[i].seconds;
            }
        }
        auto h = std::make_unique<tblaeq_handle>();
        h->qh = std::make_unique<QueryHandler>(std::move(idx));
        *out = h.release();
        return TBLAEQ_OK;
    });
}

int tblaeq_load_points_text(const char* path, double* points_out, uint64_t cap, uint64_t* n, uint64_t* d) {
    if (!path || !n || !d) return fail(TBLAEQ_ERR_INVALID, "null argument");
    return guarded([&]() -> int {
        uint64_t rows = 0, dim = 0;
        try {
            loadPointsText(path, rows, dim, nullptr);
            *n = rows;
            *d = dim;
            if (!points_out) return TBLAEQ_OK;
            if (cap < rows * dim) return fail(TBLAEQ_ERR_INVALID, "points buffer smaller than N * D");
            std::vector<double> pts;
            loadPointsText(path, rows, dim, &pts);
            std::copy(pts.begin(), pts.end(), points_out);
        } catch (const std::bad_alloc&) {
            throw;
        } catch (const std::exception& e) {
            return fail(TBLAEQ_ERR_IO, e.what());
        }
        return TBLAEQ_OK;
    });
}

int tblaeq_kmeans(const float* points, uint64_t n, uint64_t D, uint64_t k, const tblaeq_build_config* cfg,
                  float* centroids_out, uint32_t* labels_out, double* objectives_out) {
    if (!points) return fail(TBLAEQ_ERR_INVALID, "null points");
    if (cfg && (cfg->precision < 0 || cfg->precision > 2)) return fail(TBLAEQ_ERR_INVALID, "bad precision");
    return guarded([&]() -> int {
        const KmeansConfig c = kmeansConfigOf(cfg);
        cudaStream_t s = nullptr;
        TBLAEQ_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            DeviceMem dX(n * D * 4), C, L;
            TBLAEQ_CUDA(cudaMemcpyAsync(dX.get(), points, n * D * 4, cudaMemcpyHostToDevice, s));
            KmeansLevelReport rep;
            kmeansRun(dX.as<float>(), n, D, k, c, C, L, rep, s);
            if (centroids_out) TBLAEQ_CUDA(cudaMemcpyAsync(centroids_out, C.get(), k * D * 4, cudaMemcpyDeviceToHost, s));
            if (labels_out) TBLAEQ_CUDA(cudaMemcpyAsync(labels_out, L.get(), n * 4, cudaMemcpyDeviceToHost, s));
            TBLAEQ_CUDA(cudaStreamSynchronize(s));
            if (objectives_out) std::copy(rep.objectives.begin(), rep.objectives.end(), objectives_out);
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
        return TBLAEQ_OK;
    });
}

}  // extern "C"
