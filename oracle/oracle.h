/* Test infrastructure: CPU oracle for the T-BLAEQ query path.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this library, and only
 * as a checker or as the timed CPU baseline -- never as part of the product path.
 *
 * It restates, in plain C++, the reference's per-query traversal (ref-parity mode) and the exact
 * semantics the B200 path implements (exact mode), plus an FP64 brute-force scan:
 *   - ref-parity: src/core/QueryEngine.cu:63-107 driving src/core/strategies/L0Strategy.cu:50-191
 *     (range mask RangePruning.cu:5-25, KNN bound KNN.cu:9-24 + STEP L0Strategy.cu:133-154,
 *     order-preserving compaction GridCompact.cuh:41-100, expansion SpMSpV.cuh:47-67 /
 *     SpMSpV.cu:200-254, id remap Refactor.cu:10-16);
 *   - exact: the same traversal with subtree radii and leaf counts, followed by an exact filter
 *     (range: lo <= x <= hi on every dimension; KNN: the K smallest squared distances, ties
 *     broken by smaller id);
 *   - brute force: the exact predicates over every decoded finest point.
 *
 * Pinning: the index generator and serializer are pinned byte-for-byte against files written by
 * the reference binary built from source (oracle/Makefile); the ref-parity traversal is pinned
 * against the reference CUDA build's candidate sets (oracle/ref_harness.cu) on the GPU box and
 * against the committed fixtures in tests/golden/.
 */
#ifndef TBLAEQ_ORACLE_H
#define TBLAEQ_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Read-only view of an index in the reference's host layout (src/core/IndexData.cuh:89-110).
 * Mesh m runs from 0 (coarsest) to height-1 (finest points); interval l links mesh l (columns)
 * to mesh l+1 (rows). */
typedef struct {
    uint64_t D, height, intervals;
    const uint64_t* meshCount;        /* [height] node count of mesh m */
    const uint64_t* const* colRes;    /* [intervals] -> cols+1 column offsets */
    const double* const* pvals;       /* [intervals] -> rows*D ratios (AOS) */
    const double* const* radius;      /* [intervals] -> cols max child radius, by original id */
    const uint64_t* const* maps;      /* [height] -> sort-to-original map of mesh m (maps[0] unused) */
    const uint64_t* coarseIds;        /* [meshCount[0]] */
    const double* coarseVals;         /* [meshCount[0]*D] */
} oracle_index;

/* Per-query result set owned by the oracle (release with oracle_free_results). */
typedef struct {
    uint64_t nq, intervals;
    uint64_t* offsets;      /* [nq+1] */
    uint64_t* ids;          /* [offsets[nq]] */
    double* dist2;          /* [offsets[nq]] for KNN results, else NULL */
    uint64_t* levelSizes;   /* [nq*intervals] grid size after each level (reference levelFineMeshSize) */
} oracle_results;

enum { ORACLE_RANGE = 0, ORACLE_KNN = 1 };

/* Reference traversal (ref-parity). queries: RANGE -> nq rows of lo[D] then hi[D];
 * KNN -> nq rows of point[D]. use_fma selects fma(diff,diff,acc) accumulation (the reference's
 * nvcc default contraction) versus a separately rounded multiply and add.
 * sorted_ids != 0 sorts each query's ids ascending; otherwise they keep the reference order. */
int oracle_ref_query(const oracle_index* idx, int qtype, uint64_t nq, const double* queries, uint64_t K,
                     int use_fma, int sorted_ids, int threads, oracle_results* out);

/* Exact traversal: subtree radii / leaf counts (from oracle_subtree) + exact final filter. */
int oracle_exact_query(const oracle_index* idx, const double* const* subRadius, const uint64_t* const* leafCount,
                       int qtype, uint64_t nq, const double* queries, uint64_t K, int threads,
                       oracle_results* out);

/* Decoded coordinates of every node of mesh m, by position (mesh 0: coarsest list order; mesh m>=1:
 * sorted position = row of P_{m-1}). out: meshCount[m]*D doubles. */
int oracle_decode_mesh(const oracle_index* idx, uint64_t m, double* out);

/* Subtree radius (largest distance from a node's decoded centre to a decoded finest point below it,
 * inflated by the conservative slack documented in oracle.cpp) and leaf count for every node of
 * mesh m < height-1, indexed by ORIGINAL id like the reference's radius arrays. */
int oracle_subtree(const oracle_index* idx, double* const* subRadius, uint64_t* const* leafCount);

/* FP64 brute force over decoded finest points (points[n*D], ids[n]). */
int oracle_brute_query(const double* points, const uint64_t* ids, uint64_t n, uint64_t D, int qtype, uint64_t nq,
                       const double* queries, uint64_t K, int threads, oracle_results* out);

void oracle_free_results(oracle_results* r);

/* Correctly rounded-down square root (reference uses __dsqrt_rd, KNN.cu:21). */
double oracle_sqrt_rd(double x);

#ifdef __cplusplus
}
#endif
#endif
