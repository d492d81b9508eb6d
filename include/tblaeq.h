/* T-BLAEQ on B200: C ABI of the query hot path.
 *
 * Plain C types only (no torch or C++ types). Every entry point returns a tblaeq_status; on a
 * non-zero status tblaeq_last_error() returns a thread-local description. Device pointers are
 * marked "device"; everything else is host memory.
 *
 * Each declaration names the reference interface it replaces (paths inside Mgepahmge/T-BLAEQ).
 * Threading: a handle serves one thread at a time (the reference is not thread-safe either,
 * src/HTTPServer.cu:445,498,525); use one handle per serving thread.
 */
#ifndef TBLAEQ_H
#define TBLAEQ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: tblaeq_serve_config gained `levels` (and tblaeq_serve_poll_levels was added).
 * 3: tblaeq_build_config gained `host_assembly`, tblaeq_build_report `assemble_seconds`. */
#define TBLAEQ_ABI_VERSION 3

typedef struct tblaeq_handle tblaeq_handle; /* QueryHandler: host index + device state */

enum tblaeq_status {
    TBLAEQ_OK = 0,
    TBLAEQ_ERR_INVALID = 1,   /* bad argument (reference: std::invalid_argument) */
    TBLAEQ_ERR_IO = 2,        /* index file missing / truncated (reference: std::runtime_error) */
    TBLAEQ_ERR_CUDA = 3,      /* CUDA runtime error (reference: CUDA_CHECK -> exit, src/Query/check.cuh:15-25) */
    TBLAEQ_ERR_OOM = 4,       /* device allocation failed */
    TBLAEQ_ERR_OVERFLOW = 5,  /* batch exceeds the 32-bit traversal capacities; split it */
    TBLAEQ_ERR_TIMEOUT = 6,   /* a kernel's bounded wait gave up (reported status, context intact) */
    TBLAEQ_ERR_STATE = 7,     /* call order violated (e.g. query before prepare) */
    TBLAEQ_ERR_TYPE = 8       /* query type mismatch (reference: QueryResult.errorCode = 1) */
};

/* QueryType of src/Data_Structures/File.cuh:39-43 (same enumerator values). */
enum tblaeq_qtype { TBLAEQ_POINT = 0, TBLAEQ_RANGE = 1 };
/* LevelPolicy of src/core/MemoryPolicy.cuh:51. */
enum tblaeq_policy { TBLAEQ_L0 = 0, TBLAEQ_L1 = 1, TBLAEQ_L2 = 2, TBLAEQ_L3 = 3 };
/* Result semantics: the reference's candidate sets, or exact answers. */
enum tblaeq_mode { TBLAEQ_MODE_REF_PARITY = 0, TBLAEQ_MODE_EXACT = 1 };
/* Batch flags. */
enum tblaeq_batch_flags { TBLAEQ_WANT_VALS = 1, TBLAEQ_WANT_LEVELS = 2, TBLAEQ_USE_GRAPH = 4 };

typedef struct {
    uint64_t N, D;
    double valMin, valMax;
    int isInt;
    uint64_t height;
    const uint64_t* ratios; /* nRatios entries, finest first; nRatios must equal height-1 */
    uint64_t nRatios;
    uint64_t seed;
    double sigmaDivisor;
} tblaeq_gen_params;

#define TBLAEQ_MAX_HEIGHT 16
typedef struct {
    uint64_t D, N, height, intervals;
    uint64_t meshSizes[TBLAEQ_MAX_HEIGHT]; /* finest -> coarsest, like metadata.bin */
    uint64_t ratios[TBLAEQ_MAX_HEIGHT];
    uint64_t hostBytes, deviceBytes;       /* MemoryStats totals (src/core/IndexData.cu:141-194) */
    int prepared;
    int policy[TBLAEQ_MAX_HEIGHT];         /* active LevelPolicy per interval once prepared */
} tblaeq_index_info;

/* A grid of one query at one level: ids (original mesh ids) and AOS coordinates.
 * Mirrors SparseGrid (src/Data_Structures/Data_Structures.cuh:134-229); both pointers device. */
typedef struct {
    uint64_t numRows, dim, nnz;
    const uint64_t* ids;
    const double* vals;
} tblaeq_grid;

typedef struct {
    int qtype;              /* tblaeq_qtype */
    int mode;               /* tblaeq_mode */
    uint64_t nq;
    const double* queries;  /* RANGE: nq rows lo[D] hi[D]; POINT: nq rows point[D] */
    int queriesOnDevice;    /* 1: `queries` is a device pointer (off a 16-byte boundary: staged by a copy;
                               tblaeq_query_batch_async rejects it) */
    uint64_t K;             /* KNN: neighbours per query (when kPerQuery is NULL) */
    unsigned flags;         /* tblaeq_batch_flags */
    const uint32_t* kPerQuery; /* KNN: optional host array of nq neighbour counts */
} tblaeq_batch;

typedef struct {
    uint64_t nq, total;
    const uint64_t* offsets;    /* device, nq+1: results of query i are [offsets[i], offsets[i+1]) */
    const uint64_t* ids;        /* device, total: original dataset ids */
    const double* vals;         /* device, total*D (TBLAEQ_WANT_VALS) or NULL */
    const double* dist2;        /* device, total (KNN) or NULL */
    const uint32_t* levelItems; /* device, intervals*nq: reference levelFineMeshSize per level (WANT_LEVELS) */
} tblaeq_batch_result;

const char* tblaeq_last_error(void);
int tblaeq_abi_version(void);

/* QueryHandler(indexPath, true) -> IndexSerializer::load (src/core/QueryHandler.cu:126-137,
 * src/core/IndexSerializer.cu:34-67). Reads the reference's on-disk layout byte for byte. */
int tblaeq_open(const char* index_dir, tblaeq_handle** out);

/* QueryHandler(N, D, valMin, valMax, isInt, height, ratios, seed, sigmaDivisor)
 * (src/core/QueryHandler.cu:101-124 -> IndexBuilder::buildRandom, src/core/IndexBuilder.cu:153-234).
 * Produces the same index files, byte for byte, as the reference's --gen-index. */
int tblaeq_generate(const tblaeq_gen_params* params, tblaeq_handle** out);

/* QueryHandler::saveIndex (src/core/QueryHandler.cu:139-145). */
int tblaeq_save(const tblaeq_handle* h, const char* dir);

/* ~QueryHandler. Frees host and device state. NULL is accepted. */
void tblaeq_close(tblaeq_handle* h);

/* getSize / getDim / getMemoryStats / getActivePolicy (src/core/QueryHandler.cuh:160-240). */
int tblaeq_info(const tblaeq_handle* h, tblaeq_index_info* out);

/* PolicyScheduler::recommend (src/core/MemoryPolicy.cu:100-177). free_bytes = 0 queries the
 * device (cudaMemGetInfo); otherwise the given budget is used (fake budgets for tests).
 * Writes `intervals` LevelPolicy values to policy_out. */
int tblaeq_recommend(const tblaeq_handle* h, uint64_t free_bytes, int* policy_out);

/* prepareForQuery() / prepareForQuery(IndexPolicy) (src/core/QueryHandler.cu:160-182).
 * policy = NULL selects the recommendation; otherwise n_levels must equal intervals.
 * Uploads the index, derives the per-node arrays and allocates all query workspaces. */
int tblaeq_prepare(tblaeq_handle* h, const int* policy, uint64_t n_levels);

/* IQueryStrategy::runLevel (src/core/strategies/IQueryStrategy.cuh:104-105), B200 strategy:
 * prune `in` at interval l with the reference predicate (range: RangePruning.cu:5-25 with the
 * level's max radius; KNN: KNN.cu:9-24 bound + STEP, L0Strategy.cu:133-154), compact the survivors
 * in order, expand them through P_l (SpMSpV.cuh:47-67) and remap ids with Map_{l+1}
 * (Refactor.cu:10-16). lo/hi/q are host arrays of D values. `out` points at device buffers owned
 * by the handle (the reference's L0 ownsIds = ownsVals = false): valid until the next call for
 * the same level. */
int tblaeq_level(tblaeq_handle* h, uint64_t l, const tblaeq_grid* in, int qtype, const double* lo,
                 const double* hi, const double* q, uint64_t K, tblaeq_grid* out);

/* The coarsest mesh as a device grid (QueryEngine::runSingleQuery's coarsestView,
 * src/core/QueryEngine.cu:66-70). */
int tblaeq_coarsest_grid(tblaeq_handle* h, tblaeq_grid* out);

/* Batched traversal of many queries in one pass over the hierarchy (replaces the one-query loop
 * of QueryEngine::run, src/core/QueryEngine.cu:109-252). Result pointers are device memory owned
 * by the handle, valid until the next batch call. KNN batches are exact (mode must be
 * TBLAEQ_MODE_EXACT): each query's K nearest points by FP64 squared distance, ties broken by
 * smaller id, ascending; the reference's per-level KNN candidate sets come from tblaeq_level. */
int tblaeq_query_batch(tblaeq_handle* h, const tblaeq_batch* batch, tblaeq_batch_result* out);

/* Same as tblaeq_query_batch with host buffers on both sides: queries are copied to the device,
 * and offsets (nq+1), ids (up to ids_cap) and, for KNN, dist2 are copied back. *total receives
 * the number of results; if it exceeds ids_cap nothing past ids_cap is written and
 * TBLAEQ_ERR_OVERFLOW is returned. */
int tblaeq_query_batch_host(tblaeq_handle* h, const tblaeq_batch* batch, uint64_t* offsets_out, uint64_t* ids_out,
                            uint64_t ids_cap, double* dist2_out, uint64_t* total);

/* Enqueue a range batch on the handle's stream and return without waiting (no host
 * synchronisation, so it can be timed with events or overlapped; KNN batches, which may run as
 * chunks with host synchronisation between them, go through tblaeq_query_batch). `queries` must be
 * device memory that stays valid
 * until tblaeq_batch_wait returns, and a synchronous tblaeq_query_batch with the same nq, mode and
 * flags must have run first (it sizes the workspaces). With TBLAEQ_USE_GRAPH the launches are
 * captured once into a CUDA graph and replayed. */
int tblaeq_query_batch_async(tblaeq_handle* h, const tblaeq_batch* batch);

/* Nodes of the CUDA graph that TBLAEQ_USE_GRAPH replays: *kernels = kernel launches per replay,
 * *nodes = all nodes (kernels, memsets, copies, event records). Both 0 when no graph is held (no
 * graph batch yet, or a setting or workspace growth since dropped it). */
int tblaeq_graph_launches(tblaeq_handle* h, uint64_t* kernels, uint64_t* nodes);

/* Kernel launches this library has issued in the process so far (index build, scorer training
 * and queries; a launch captured into a CUDA graph counts once, at capture, and graph replays are
 * not counted: tblaeq_graph_launches gives the kernels per replay). */
uint64_t tblaeq_kernel_launches(void);

/* Wait for the last enqueued batch, check its device status (workspace overflow ->
 * TBLAEQ_ERR_OVERFLOW: rerun it with tblaeq_query_batch) and describe its results. */
int tblaeq_batch_wait(tblaeq_handle* h, tblaeq_batch_result* out);

/* Frontier entries and work items (children) per level of the last batch: entries[0], items[0]
 * describe the root frontier (one entry per query), entries[m+1], items[m+1] the survivors of
 * mesh m and their children; results[0] = number of results. Returns the number of levels written. */
int tblaeq_level_counts(tblaeq_handle* h, uint64_t* entries, uint64_t* items, int cap, uint64_t* results);

/* Select the CUDA device used by this library on the calling thread (cudaSetDevice); call before
 * tblaeq_prepare. */
int tblaeq_set_device(int device);

/* The CUDA stream (cudaStream_t) every launch of this handle goes to. */
void* tblaeq_stream(tblaeq_handle* h);

/* Record CUDA events between the launch stages of every batch (1 = on). */
int tblaeq_set_timing(tblaeq_handle* h, int on);

/* Elapsed milliseconds per stage of the last batch: [0] workspace reset + root frontier,
 * [1..height] one per mesh expand (the last one is the finest level), [height+1] result offsets.
 * Returns the number of stages written (at most cap), or -1 when timing is off. */
int tblaeq_stage_times(tblaeq_handle* h, float* ms, int cap);

/* Autotuner: times every launch shape (expand-kernel variant -- registers or a cp.async
 * shared-memory ring -- times persistent-grid size, see tblaeq_set_launch_shapes) on this batch for
 * every level and keeps the fastest per level (device queries, range batches). variants_out
 * (height entries) receives the variants chosen, ms_out (height entries, may be NULL) the median
 * milliseconds of each chosen level; tblaeq_get_launch_shapes returns the grid sizes too. */
int tblaeq_autotune(tblaeq_handle* h, const tblaeq_batch* batch, int reps, int* variants_out, float* ms_out);

/* Set the expand-kernel variant per level (0 = direct, 1 = staged), e.g. from a tuning cache. */
int tblaeq_set_variants(tblaeq_handle* h, const int* variants, uint64_t n);

/* Exact range batches test their inner levels node-major (1, the default: one warp per node and 32
 * of the queries holding it) or entry-major (0: one work item per query and child). Same results;
 * node-major returns each query's ids in no particular order. No counterpart in the reference. */
int tblaeq_set_node_major(tblaeq_handle* h, int on);

/* Exact range batches: the finest level decides each point from a float copy of the decoded points
 * (4·D bytes a point instead of the 8·D of its P row) and takes the FP64 test only for a point with
 * a coordinate within float rounding of a face of the box, so the results are the same either way
 * (on = default; for D = 4, 8, 16 with the last interval device-resident). No counterpart in the
 * reference, whose final filter reads every surviving point's doubles. */
int tblaeq_set_float_points(tblaeq_handle* h, int on);

/* Exact range batches with float points: every finest cluster's points are kept in point groups
 * of at most 32 (a median split along the widest dimension, repeated; the rows of a cluster are
 * reordered within the cluster's own range when the index is prepared), each with the box of its
 * points. The finest level first keeps the groups whose box meets the query box and then tests
 * only their points (on = default; off = every point of every surviving cluster). Same results.
 * Batches that ask for per-level counts (TBLAEQ_WANT_LEVELS) test every point: those counts are
 * the points of the surviving clusters. The same switch governs exact KNN batches, whose
 * node-major point pass skips every group whose box lies beyond the query's bound. No counterpart
 * in the reference. */
int tblaeq_set_point_groups(tblaeq_handle* h, int on);
/* The last range batch's point groups: out3[0] groups tested, out3[1] (query, group) pairs kept,
 * out3[2] points tested; zeros when it tested no groups. With groups, tblaeq_level_counts'
 * children of the finest clusters are their groups. */
int tblaeq_group_counts(tblaeq_handle* h, uint64_t* out3);

/* ---- Launch shapes and the tuning cache (no counterpart in the reference, whose kernel shapes are
 * compile-time constants: kCompact* in src/core/strategies/L0Strategy.cu:18-21, UNROLL_FACTOR in
 * src/Kernel/SpMSpV.cuh:24) ----
 * A launch shape per expand launch (one per mesh, `height` of them): the kernel variant (0 = direct,
 * 1 = staged) and the persistent grid as a percentage (1..100) of the kernel's full occupancy.
 * tblaeq_autotune searches variant x grid {100, 75, 50, 25}% per level on the live batch. */
int tblaeq_set_launch_shapes(tblaeq_handle* h, const int* variants, const int* grid_percent, uint64_t n);
int tblaeq_get_launch_shapes(tblaeq_handle* h, int* variants, int* grid_percent, uint64_t cap);

/* The tuning-cache key of this handle for a range batch of nq queries in `mode`: the GPU model and
 * SM count, the index shape (N, D, height, ratios), the mode and nq rounded up to a power of two.
 * Written NUL-terminated into buf (cap bytes; TBLAEQ_ERR_INVALID when too small). */
int tblaeq_tuning_key(tblaeq_handle* h, int mode, uint64_t nq, char* buf, uint64_t cap);

/* The tuning cache is a versioned text file ("tblaeq-tuning-cache 1", then one line per key).
 * tblaeq_tuning_store adds or replaces the key's shapes (n levels); tblaeq_tuning_lookup copies them
 * out (*n = levels; *n = 0 when the file or the key is missing, TBLAEQ_ERR_INVALID when cap < levels). */
int tblaeq_tuning_store(const char* path, const char* key, const int* variants, const int* grid_percent, uint64_t n);
int tblaeq_tuning_lookup(const char* path, const char* key, int* variants, int* grid_percent, uint64_t cap,
                         uint64_t* n);

/* ---- Exact KNN tuning and the learned frontier scorer (no counterpart in the reference) ----
 * Exact KNN batches end with a two-wave finest level: each query's surviving finest clusters are
 * ranked, the best few are expanded first so the K-th distance is bounded by real points, and only
 * the clusters that bound cannot exclude are expanded next. The ranking is the clusters' lower
 * bound, or the learned scorer (a 2x64 MLP over query || centroid || radius || level one-hot, BF16
 * weights, FP32 accumulation) once trained. Exactness never depends on the ranking. */

/* 1 (default) = two-wave finest level, 0 = one pass over every surviving cluster. */
int tblaeq_set_two_wave(tblaeq_handle* h, int on);

/* Exact KNN batches with the two-wave finest level: `beam` (0..32, default 32) is the probe's beam
 * -- at every level above the clusters each query keeps its `beam` entries of smallest lower bound,
 * and wave 1 ranks only the clusters under them (0: every surviving cluster is ranked) -- and
 * node_major_completion (default 1) selects how the points within wave 1's bound are found: the
 * hierarchy walked again node-major (one warp per node and 32 of its queries; each cluster's points
 * read once per 32 of its queries), or 0: every remaining frontier entry expanded query by query
 * (the beam is then not applied: that wave only covers the frontier). Exactness never depends on
 * either. No counterpart in the reference. */
int tblaeq_set_knn_probe(tblaeq_handle* h, uint32_t beam, int node_major_completion);

/* Wave 1 of a two-wave KNN batch reads every point of each query's ceil(scale * K / leaf) + 1
 * best-ranked finest clusters (at least 2, at most 32; leaf = the index's points per finest cluster)
 * and takes the K-th distance among them as the bound the rest of the batch prunes with. A larger
 * wave 1 costs more rows up front and tightens the bound (default scale 16). Same results for every
 * scale. No counterpart in the reference (its KNN keeps the STEP candidate set). */
int tblaeq_set_knn_wave1(tblaeq_handle* h, double scale);

/* The node-major KNN completion (after wave 1) first tests every stride²-th and then every
 * stride-th point of the clusters it listed; with wave 1's points they are real points, so each
 * query's K-th distance among them bounds its K-th neighbour distance, and each later pass (the
 * full point pass last) skips every cluster whose sphere lies beyond the bound so far (fewer points
 * tested and far fewer candidates kept). stride 0 or 1: off; default 16. Same results for every
 * stride. No counterpart in the reference. */
int tblaeq_set_knn_refine(tblaeq_handle* h, uint32_t stride);
/* How many refinement stages run (1..4; default 2): strides stride^stages, ..., stride. */
int tblaeq_set_knn_refine_stages(tblaeq_handle* h, uint32_t stages);

/* Queries per traversal of a KNN batch. A batch whose workspace exceeds the 32-bit traversal space or
 * the free device memory runs as consecutive traversals of a halved size; later batches start at the
 * size that fitted. max_queries > 0 caps every traversal at that many queries; 0 restores the
 * automatic choice (and forgets the size learnt). No counterpart in the reference, which runs one
 * query at a time. */
int tblaeq_set_knn_chunk(tblaeq_handle* h, uint64_t max_queries);
/* Traversals the last synchronous batch (range or KNN, the last chunk of a split one) ran: 1, plus
 * one rerun after every workspace growth. */
int tblaeq_last_batch_runs(tblaeq_handle* h, uint64_t* runs);
/* The last KNN batch: out2[0] = queries per traversal, out2[1] = traversals. */
int tblaeq_knn_batch_info(tblaeq_handle* h, uint64_t* out2);
/* Why a KNN batch of this handle was last split: the traversal size that did not fit and the
 * error it met (empty if none was split), NUL-terminated into buf (cap bytes). */
int tblaeq_knn_split_reason(tblaeq_handle* h, char* buf, uint64_t cap);

/* Counters of the last KNN batch (summed over its chunks when it ran in several): [0] final-frontier
 * clusters, [1] wave-1 candidates,
 * [2] wave-2 candidates, [3] points whose rows wave 1 loaded and tested (the single pass, when
 * two-wave is off), [4] points whose rows wave 2 loaded and tested. */
int tblaeq_knn_counters(tblaeq_handle* h, uint64_t* out5);

/* Trains the scorer on traces of exact KNN over the given training queries (host points, nq x D;
 * per-query K or uniform K), sampling up to max_samples (query, cluster) examples; runs `epochs`
 * of Adam with learning rate lr. loss_out (epochs entries, may be NULL) receives the mean loss of
 * each epoch. Leaves the scorer enabled. */
int tblaeq_scorer_train(tblaeq_handle* h, const double* points, uint64_t nq, const uint32_t* k_per_query, uint64_t K,
                        uint64_t max_samples, int epochs, float lr, uint64_t seed, float* loss_out);

/* Enable (1) or disable (0) the trained scorer for KNN ranking. */
int tblaeq_scorer_enable(tblaeq_handle* h, int on);

/* Scorer parameters as FP32 (layout W1[in][64] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3 with
 * in = 2D + 1 + (height-1)): *n receives the count; get copies up to cap values. */
int tblaeq_scorer_get_params(tblaeq_handle* h, float* out, uint64_t cap, uint64_t* n);
int tblaeq_scorer_set_params(tblaeq_handle* h, const float* params, uint64_t n);

/* Mean binary cross-entropy of host samples X (n x in) / labels y under the current parameters
 * (BF16 forward, FP32 accumulation) and its gradient (params-sized) -- for gradient checks. */
int tblaeq_scorer_loss_grad(tblaeq_handle* h, const float* X, const float* y, uint64_t n, float* grad_out,
                            float* loss_out);

/* Logits of host samples X (n x in): CUDA-core forward (BF16 weights, FP32 activations). */
int tblaeq_scorer_logits(tblaeq_handle* h, const float* X, uint64_t n, float* z_out);

/* The same logits through the kernel that scores KNN frontiers: tcgen05 BF16 MMAs with FP32
 * accumulation, so X and the hidden layer are rounded to BF16. TBLAEQ_ERR_TIMEOUT if the kernel
 * gave up waiting for its MMAs. No counterpart in the reference (it ranks frontiers by bound). */
int tblaeq_scorer_logits_tensor(tblaeq_handle* h, const float* X, uint64_t n, float* z_out);

/* The last training's sample count and how many of the traced (query, cluster) pairs were
 * positives (the cluster holds one of the query's K nearest points). */
int tblaeq_scorer_stats(tblaeq_handle* h, uint64_t* samples, uint64_t* positives);

/* Saves the trained scorer (parameters, feature scale, training counts) to a file, or loads one
 * (checked against the index's dimension and height) and enables it. */
int tblaeq_scorer_save(tblaeq_handle* h, const char* path);
int tblaeq_scorer_load(tblaeq_handle* h, const char* path);

/* Host copies of the index arrays (read-only, owned by the handle), for tools and tests:
 * which = 0: P-tensor values of interval l (rows*D doubles), 1: colRes of interval l (cols+1),
 * 2: max radius of interval l (cols), 3: Map of mesh l (meshSizes), 4: coarsest ids, 5: coarsest vals. */
int tblaeq_host_array(const tblaeq_handle* h, int which, uint64_t l, const void** ptr, uint64_t* count);

/* Decoded coordinates (the reference's rebuilt values, P products down the hierarchy) of the
 * finest points at the given sorted positions, with their original dataset ids. Host only; used
 * to draw query workloads centred on data points. */
int tblaeq_decode_points(tblaeq_handle* h, const uint64_t* positions, uint64_t n, double* coords_out,
                         uint64_t* ids_out);

/* Allocation-free per-level range step. No counterpart in the reference: it exists for callers
 * that cannot allocate device memory while they query (a process that reserved its whole memory
 * budget at start-up, or one whose rules forbid allocation between start-up and shutdown).
 * Same result as tblaeq_level for a range query -- the grid of interval l after pruning, in the
 * reference's order -- written into the caller's device buffers out_ids (out_cap entries) and
 * out_vals (out_cap * D doubles); *out_n receives the number of entries.
 * It calls no cudaMalloc/cudaFree and no allocating library routine: its scratch is one fixed
 * array in device memory (about 2.4 MB), held by every GPU that loads the library until exit.
 * Limits: in->nnz <= 16384, out_cap <= 1048576, D <= 16; larger requests fail with
 * TBLAEQ_ERR_INVALID, outputs that do not fit with TBLAEQ_ERR_OVERFLOW.
 * The first call on a device looks up the array's device address; make that first call before
 * any stream capture. All calls on a device share the array: calls whose work overlaps on the
 * GPU (other streams or handles on the same device) race and must be serialised by the caller. */
int tblaeq_level_range_noalloc(tblaeq_handle* h, uint64_t l, const tblaeq_grid* in, const double* lo,
                               const double* hi, uint64_t* out_ids, double* out_vals, uint64_t out_cap,
                               uint64_t* out_n);

/* Number of device bytes currently allocated by the library (leak checks). */
uint64_t tblaeq_live_device_bytes(void);

/* Test hook: make the n-th device allocation from now on fail (n = 0 disables). */
void tblaeq_debug_fail_alloc_after(uint64_t n);

/* Test hook for failure detection (no counterpart in the reference, whose kernels never wait on
 * one another): from now on, range and per-level plugin traversals (tblaeq_query_batch of range
 * queries, tblaeq_level, tblaeq_level_range_noalloc) leave work tile `withhold_tile` of every
 * expand launch unpublished, and their look-back waits give up after `spin_limit` polls. The wait
 * runs out, the kernel sets its timeout status and returns, later launches of the batch skip their
 * work, and the call fails with TBLAEQ_ERR_TIMEOUT with the CUDA context intact. withhold_tile =
 * UINT64_MAX or spin_limit = 0 switches the hook off. Process-wide; KNN batches are never affected;
 * launches already captured in a CUDA graph keep the setting they were captured with. */
void tblaeq_debug_lookback_timeout(uint64_t withhold_tile, uint64_t spin_limit);

/* Test hook: treat traversal workspaces above `limit` frontier entries or work items as too large
 * (0 restores the 32-bit limit), so that small indexes exercise the chunked KNN batches. */
int tblaeq_debug_split_above(tblaeq_handle* h, uint64_t limit);

/* ---- Index build -------------------------------------------------------------------------------
 * Replaces IndexBuilder::build (src/core/IndexBuilder.cu:44-151: cuVS k-means per level, then
 * Genenate_One_P_Tensor / Compute_Max_Radius, src/Setup/Setup.cuh:87-171): Lloyd's k-means per
 * level on the GPU, k = floor(n / ratio) centroids sampled from the data (seeded), `iters`
 * iterations, then the same P-tensor / map / radius assembly (rows grouped by label in input
 * order), done on the device: labels and centroids never leave it, only the finished index
 * arrays are copied to the host index. precision: 0 = tensor cores (tcgen05; TF32 hi/lo split
 * operands, FP32 accumulation; D <= 16, larger D uses 1), 1 = FP32 CUDA cores, 2 = FP64 CUDA cores
 * (the precision reference). Centroid sums accumulate in FP64; objectives are sum ||x - c(x)||^2 in
 * FP64. */
typedef struct {
    int iters;         /* Lloyd iterations per level (0: 20) */
    uint64_t seed;
    int precision;
    int host_assembly; /* 0: on the device; 1: on the host from downloaded labels and centroids, as the
                          reference does; 2: both from the same labels and centroids, the device
                          result kept and checked byte for byte against the host's (an error if they
                          differ) */
} tblaeq_build_config;

typedef struct {
    uint64_t n, k;          /* points and centroids of the level */
    int iters;
    double objective;       /* after the last iteration */
    double assign_seconds;  /* device time of the assignment passes */
    double assemble_seconds; /* the level's index assembly (P-tensor, map, radii) */
    double seconds;         /* the whole level, including the index assembly */
} tblaeq_build_report;

/* Builds an index over host FP32 points (N x D) with `height` levels and `ratios` (finest first, as
 * in the reference). *out receives an unprepared handle (like tblaeq_open); report (height - 1
 * entries, finest level first, may be NULL). */
int tblaeq_kmeans_build(const float* points, uint64_t N, uint64_t D, uint64_t height, const uint64_t* ratios,
                        const tblaeq_build_config* cfg, tblaeq_handle** out, tblaeq_build_report* report);

/* One level of k-means on the current device (no index): centroids_out (k x D) and labels_out (n)
 * may be NULL; objectives_out receives one FP64 objective per iteration. */
int tblaeq_kmeans(const float* points, uint64_t n, uint64_t D, uint64_t k, const tblaeq_build_config* cfg,
                  float* centroids_out, uint32_t* labels_out, double* objectives_out);

/* Dataset text file (reference loadFromFile, src/Data_Structures/File.cu:8-50): a header "N D",
 * then N rows of D values. With points_out == NULL only the header is read into *n and *d; with a
 * buffer of cap >= N * D doubles the rows are parsed into it, row-major. TBLAEQ_ERR_IO carries the
 * reference's message (cannot open, empty file, invalid header, dimension mismatch at row r, row
 * count mismatch); TBLAEQ_ERR_INVALID when cap is too small. */
int tblaeq_load_points_text(const char* path, double* points_out, uint64_t cap, uint64_t* n, uint64_t* d);

/* ---- Serving loop ------------------------------------------------------------------------------
 * Replaces the reference's one-query-at-a-time request loop behind its HTTP front end
 * (src/HTTPServer.cu:414-550; the HTTP layer itself is not part of this library). A server owns two
 * lanes (range and KNN), each a worker thread with its own device workspace and CUDA stream; each
 * lane batches continuously (requests that arrive while its batch is on the GPU form the next
 * batch), with slots per batch bounded by max_batch and by the lane's device-memory budget.
 * Requests are exact (KNN always; range in `mode`). The handle must stay open and prepared while a
 * server runs; other calls on the same handle may run concurrently from one other thread. */
typedef struct tblaeq_server tblaeq_server;

typedef struct {
    uint32_t max_batch;      /* requests per batch and lane (0: 4096) */
    uint64_t memory_budget;  /* traversal workspace bytes per lane (0: a quarter of free memory) */
    int mode;                /* tblaeq_mode for range requests */
    int learned;             /* rank KNN frontiers with the trained scorer, when one exists */
    int lanes;               /* 2 (range and KNN lanes, default when 0) or 1 (one lane, arrival order) */
    int levels;              /* 1: record each request's per-level child counts (tblaeq_serve_poll_levels) */
} tblaeq_serve_config;

typedef struct {
    uint64_t submitted, completed, failed, batches, max_batch;
    double mean_batch;
    double p50_us, p99_us, mean_us, max_us; /* arrival to result, per request */
    double span_s;                          /* first arrival to last completion */
} tblaeq_serve_metrics;

int tblaeq_serve_start(tblaeq_handle* h, const tblaeq_serve_config* cfg, tblaeq_server** out);
/* qtype TBLAEQ_POINT: query = point[D], K neighbours; TBLAEQ_RANGE: query = lo[D] hi[D]. */
int tblaeq_serve_submit(tblaeq_server* s, int qtype, const double* query, uint64_t K, uint64_t* ticket);
/* Submits n requests from the calling thread, request i at arrival_us[i] microseconds after the
 * call (a replayed arrival schedule); its query starts at queries + offsets[i]. */
int tblaeq_serve_replay(tblaeq_server* s, uint64_t n, const int* qtypes, const double* queries,
                        const uint64_t* offsets, const uint32_t* K, const double* arrival_us, uint64_t* tickets);
/* Waits up to wait_ms for the ticket's result. TBLAEQ_OK: *n_out ids (and squared distances for
 * KNN) copied, ticket released. TBLAEQ_ERR_TIMEOUT: not done yet. TBLAEQ_ERR_OVERFLOW: cap < *n_out,
 * the result stays. A failed request returns its error code and message and is released. */
int tblaeq_serve_poll(tblaeq_server* s, uint64_t ticket, int wait_ms, uint64_t* ids_out, double* dist2_out,
                      uint64_t cap, uint64_t* n_out, double* latency_us);
/* As tblaeq_serve_poll, and the request's generated-children count per level (the reference's
 * QueryResult::levelFineMeshSize of a single query, src/core/QueryEngine.cu:65-81; one value per
 * interval, coarsest first) into levels_out when the server records them (config `levels`);
 * *n_levels receives their count (0 otherwise; at most levels_cap are copied). Serves the HTTP
 * front end's `level_pruned_sizes` (src/HTTPServer.cu:466-468). */
int tblaeq_serve_poll_levels(tblaeq_server* s, uint64_t ticket, int wait_ms, uint64_t* ids_out, double* dist2_out,
                             uint64_t cap, uint64_t* n_out, double* latency_us, uint32_t* levels_out,
                             uint64_t levels_cap, uint64_t* n_levels);
/* TBLAEQ_OK once every submitted request has completed, TBLAEQ_ERR_TIMEOUT after wait_ms. */
int tblaeq_serve_wait_idle(tblaeq_server* s, int wait_ms);
int tblaeq_serve_stats(tblaeq_server* s, int reset, tblaeq_serve_metrics* out);
/* Drains the queued requests, joins the workers and frees the server (its results go with it). */
int tblaeq_serve_stop(tblaeq_server* s);

#ifdef __cplusplus
}
#endif
#endif /* TBLAEQ_H */
