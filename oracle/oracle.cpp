// Test infrastructure: CPU oracle for the T-BLAEQ query path (see oracle.h for what each entry
// point restates and how it is pinned). Built with -ffp-contract=off so every multiply and add
// below is rounded exactly as written; fused multiply-adds appear only as explicit std::fma.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <vector>

#include <omp.h>

namespace {

// Conservative slack for subtree radii: R_stored = R * (1 + kRelSlack) + kAbsSlack. Rounding errors
// of the box distance, the centre-to-point distance and the decoded coordinates are all below
// 1e-14 relative for coordinates of the magnitudes these indexes hold, so this slack only ever
// adds candidates; it never drops a true result.
constexpr double kRelSlack = 1e-9;
constexpr double kAbsSlack = 1e-12;

struct Grid {
    std::vector<uint64_t> ids;
    std::vector<double> vals;
};

inline double accumulate_sq(double acc, double diff, int use_fma) {
    return use_fma ? std::fma(diff, diff, acc) : acc + diff * diff;
}

// Squared distance from x to the axis-aligned box [lo, hi] (RangePruning.cu:7-20).
inline double box_dist2(const double* x, const double* lo, const double* hi, uint64_t D, int use_fma) {
    double dist = 0.0;
    for (uint64_t d = 0; d < D; ++d) {
        double diff = 0.0;
        const double cv = x[d];
        if (cv < lo[d]) {
            diff = lo[d] - cv;
        } else if (cv > hi[d]) {
            diff = cv - hi[d];
        }
        dist = accumulate_sq(dist, diff, use_fma);
    }
    return dist;
}

// Squared distance between a query point and x (KNN.cu:14-19).
inline double point_dist2(const double* q, const double* x, uint64_t D, int use_fma) {
    double dist = 0.0;
    for (uint64_t d = 0; d < D; ++d) {
        const double diff = q[d] - x[d];
        dist = accumulate_sq(dist, diff, use_fma);
    }
    return dist;
}

// Position of a mesh-m node given its original id (inverse of the sort-to-original map).
std::vector<uint64_t> inverse_map(const oracle_index* idx, uint64_t m) {
    const uint64_t n = idx->meshCount[m];
    std::vector<uint64_t> inv(n);
    if (m == 0) {
        for (uint64_t i = 0; i < n; ++i) inv[idx->coarseIds[i]] = i;
    } else {
        for (uint64_t s = 0; s < n; ++s) inv[idx->maps[m][s]] = s;
    }
    return inv;
}

// One traversal of one query. radius[l] / counts[l] are indexed by original id of mesh l.
// exact_filter != 0 applies the exact final predicate to the finest grid.
struct TraversalConfig {
    const double* const* radius;
    const uint64_t* const* counts;   // STEP child counts (reference: nnzPerCol; exact: leaf counts)
    int use_fma;
    int exact;
};

void traverse_one(const oracle_index* idx, const TraversalConfig& cfg, int qtype, const double* query, uint64_t K,
                  std::vector<uint64_t>& outIds, std::vector<double>& outD2, uint64_t* levelSizes) {
    const uint64_t D = idx->D;
    Grid cur;
    const uint64_t n0 = idx->meshCount[0];
    cur.ids.assign(idx->coarseIds, idx->coarseIds + n0);
    cur.vals.assign(idx->coarseVals, idx->coarseVals + n0 * D);
    const double* lo = query;
    const double* hi = query + D;

    for (uint64_t l = 0; l < idx->intervals; ++l) {
        const uint64_t p = cur.ids.size();
        const double* r = cfg.radius[l];
        std::vector<char> mask(p, 0);
        if (qtype == ORACLE_RANGE) {
            for (uint64_t i = 0; i < p; ++i) {
                const double dist = box_dist2(&cur.vals[i * D], lo, hi, D, cfg.use_fma);
                const double rr = r[cur.ids[i]];
                mask[i] = dist <= rr * rr;
            }
        } else {
            // Lower bound per centroid, sorted ascending (ties by position: a total order), then
            // the STEP selection of L0Strategy.cu:133-154.
            struct Cl {
                double distance;
                uint64_t label;
            };
            std::vector<Cl> cl(p);
            for (uint64_t i = 0; i < p; ++i) {
                const double dist = point_dist2(query, &cur.vals[i * D], D, cfg.use_fma);
                const double s = cfg.exact ? std::sqrt(dist) : oracle_sqrt_rd(dist);
                cl[i] = {s - r[cur.ids[i]], i};
            }
            std::sort(cl.begin(), cl.end(), [](const Cl& a, const Cl& b) {
                return a.distance < b.distance || (a.distance == b.distance && a.label < b.label);
            });
            uint64_t count = 0;
            double curDist = 0.0;
            for (uint64_t i = 0; i < p; ++i) {
                const uint64_t g = cur.ids[cl[i].label];
                if (count >= K) {
                    if (cl[i].distance > curDist) break;
                    count += cfg.counts[l][g];
                    mask[cl[i].label] = 1;
                } else {
                    count += cfg.counts[l][g];
                    curDist = std::max(curDist, cl[i].distance + 2.0 * r[g]);
                    mask[cl[i].label] = 1;
                }
            }
        }
        // Order-preserving compaction, then expansion through P_l and the map of mesh l+1.
        Grid next;
        const uint64_t* colRes = idx->colRes[l];
        const double* P = idx->pvals[l];
        const uint64_t* map = idx->maps[l + 1];
        for (uint64_t i = 0; i < p; ++i) {
            if (!mask[i]) continue;
            const uint64_t c = cur.ids[i];
            const double* x = &cur.vals[i * D];
            for (uint64_t j = colRes[c]; j < colRes[c + 1]; ++j) {
                next.ids.push_back(map[j]);
                for (uint64_t d = 0; d < D; ++d) next.vals.push_back(P[j * D + d] * x[d]);
            }
        }
        if (levelSizes) levelSizes[l] = next.ids.size();
        cur = std::move(next);
    }

    outIds.clear();
    outD2.clear();
    const uint64_t n = cur.ids.size();
    if (!cfg.exact) {
        outIds = cur.ids;
        return;
    }
    if (qtype == ORACLE_RANGE) {
        for (uint64_t i = 0; i < n; ++i) {
            const double* x = &cur.vals[i * D];
            bool in = true;
            for (uint64_t d = 0; d < D; ++d) in = in && (lo[d] <= x[d]) && (x[d] <= hi[d]);
            if (in) outIds.push_back(cur.ids[i]);
        }
        std::sort(outIds.begin(), outIds.end());
    } else {
        std::vector<std::pair<double, uint64_t>> c(n);
        for (uint64_t i = 0; i < n; ++i) c[i] = {point_dist2(query, &cur.vals[i * D], D, 1), cur.ids[i]};
        const uint64_t k = std::min<uint64_t>(K, n);
        std::partial_sort(c.begin(), c.begin() + k, c.end());
        for (uint64_t i = 0; i < k; ++i) {
            outIds.push_back(c[i].second);
            outD2.push_back(c[i].first);
        }
    }
}

void pack_results(std::vector<std::vector<uint64_t>>& ids, std::vector<std::vector<double>>& d2, uint64_t intervals,
                  std::vector<uint64_t>& levels, bool withD2, oracle_results* out) {
    const uint64_t nq = ids.size();
    out->nq = nq;
    out->intervals = intervals;
    out->offsets = static_cast<uint64_t*>(std::malloc((nq + 1) * 8));
    out->offsets[0] = 0;
    for (uint64_t q = 0; q < nq; ++q) out->offsets[q + 1] = out->offsets[q] + ids[q].size();
    const uint64_t total = out->offsets[nq];
    out->ids = static_cast<uint64_t*>(std::malloc(std::max<uint64_t>(total, 1) * 8));
    out->dist2 = withD2 ? static_cast<double*>(std::malloc(std::max<uint64_t>(total, 1) * 8)) : nullptr;
    for (uint64_t q = 0; q < nq; ++q) {
        if (!ids[q].empty()) std::memcpy(out->ids + out->offsets[q], ids[q].data(), ids[q].size() * 8);
        if (withD2 && !d2[q].empty()) std::memcpy(out->dist2 + out->offsets[q], d2[q].data(), d2[q].size() * 8);
    }
    out->levelSizes = static_cast<uint64_t*>(std::malloc(std::max<uint64_t>(nq * intervals, 1) * 8));
    if (nq > 0 && intervals > 0) std::memcpy(out->levelSizes, levels.data(), nq * intervals * 8);
}

int run_traversals(const oracle_index* idx, const TraversalConfig& cfg, int qtype, uint64_t nq, const double* queries,
                   uint64_t K, int sorted_ids, int threads, oracle_results* out) {
    const uint64_t D = idx->D;
    const uint64_t stride = (qtype == ORACLE_RANGE) ? 2 * D : D;
    std::vector<std::vector<uint64_t>> ids(nq);
    std::vector<std::vector<double>> d2(nq);
    std::vector<uint64_t> levels(nq * idx->intervals, 0);
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
    for (int64_t q = 0; q < static_cast<int64_t>(nq); ++q) {
        traverse_one(idx, cfg, qtype, queries + q * stride, K, ids[q], d2[q], &levels[q * idx->intervals]);
        if (sorted_ids && !(cfg.exact && qtype == ORACLE_KNN)) std::sort(ids[q].begin(), ids[q].end());
    }
    pack_results(ids, d2, idx->intervals, levels, cfg.exact && qtype == ORACLE_KNN, out);
    return 0;
}

}  // namespace

extern "C" {

double oracle_sqrt_rd(double x) {
    // RN square root, stepped down one ulp when it lies above the exact root. fma(s, s, -x) is
    // the correctly rounded s*s - x, whose sign is the sign of the exact difference.
    double s = std::sqrt(x);
    if (s > 0.0 && std::fma(s, s, -x) > 0.0) s = std::nextafter(s, 0.0);
    return s;
}

int oracle_ref_query(const oracle_index* idx, int qtype, uint64_t nq, const double* queries, uint64_t K, int use_fma,
                     int sorted_ids, int threads, oracle_results* out) {
    std::vector<const uint64_t*> counts(idx->intervals);
    std::vector<std::vector<uint64_t>> owned(idx->intervals);
    for (uint64_t l = 0; l < idx->intervals; ++l) {
        const uint64_t cols = idx->meshCount[l];
        owned[l].resize(cols);
        for (uint64_t c = 0; c < cols; ++c) owned[l][c] = idx->colRes[l][c + 1] - idx->colRes[l][c];
        counts[l] = owned[l].data();
    }
    TraversalConfig cfg{idx->radius, counts.data(), use_fma, 0};
    return run_traversals(idx, cfg, qtype, nq, queries, K, sorted_ids, threads, out);
}

int oracle_exact_query(const oracle_index* idx, const double* const* subRadius, const uint64_t* const* leafCount,
                       int qtype, uint64_t nq, const double* queries, uint64_t K, int threads, oracle_results* out) {
    TraversalConfig cfg{subRadius, leafCount, 1, 1};
    return run_traversals(idx, cfg, qtype, nq, queries, K, 1, threads, out);
}

int oracle_decode_mesh(const oracle_index* idx, uint64_t m, double* out) {
    const uint64_t D = idx->D;
    std::vector<double> cur(idx->coarseVals, idx->coarseVals + idx->meshCount[0] * D);
    for (uint64_t l = 0; l < m; ++l) {
        const std::vector<uint64_t> inv = inverse_map(idx, l);
        const uint64_t cols = idx->meshCount[l];
        std::vector<double> next(idx->meshCount[l + 1] * D);
        for (uint64_t c = 0; c < cols; ++c) {
            const double* x = &cur[inv[c] * D];
            for (uint64_t j = idx->colRes[l][c]; j < idx->colRes[l][c + 1]; ++j)
                for (uint64_t d = 0; d < D; ++d) next[j * D + d] = idx->pvals[l][j * D + d] * x[d];
        }
        cur.swap(next);
    }
    std::memcpy(out, cur.data(), cur.size() * 8);
    return 0;
}

int oracle_subtree(const oracle_index* idx, double* const* subRadius, uint64_t* const* leafCount) {
    const uint64_t D = idx->D;
    const uint64_t H = idx->height;
    // Decoded coordinates of every mesh, by position.
    std::vector<std::vector<double>> dec(H);
    for (uint64_t m = 0; m < H; ++m) {
        dec[m].resize(idx->meshCount[m] * D);
        oracle_decode_mesh(idx, m, dec[m].data());
    }
    // parentPos[m][s]: position in mesh m-1 of the parent of the node at position s of mesh m.
    std::vector<std::vector<uint64_t>> parentPos(H);
    for (uint64_t m = 1; m < H; ++m) {
        const std::vector<uint64_t> inv = inverse_map(idx, m - 1);
        parentPos[m].resize(idx->meshCount[m]);
        for (uint64_t c = 0; c < idx->meshCount[m - 1]; ++c)
            for (uint64_t j = idx->colRes[m - 1][c]; j < idx->colRes[m - 1][c + 1]; ++j) parentPos[m][j] = inv[c];
    }
    std::vector<std::vector<double>> R(H - 1);
    std::vector<std::vector<uint64_t>> cnt(H - 1);
    for (uint64_t m = 0; m + 1 < H; ++m) {
        R[m].assign(idx->meshCount[m], 0.0);
        cnt[m].assign(idx->meshCount[m], 0);
    }
    const uint64_t nLeaf = idx->meshCount[H - 1];
    for (uint64_t s = 0; s < nLeaf; ++s) {
        const double* x = &dec[H - 1][s * D];
        uint64_t pos = s;
        for (uint64_t m = H - 1; m > 0; --m) {
            pos = parentPos[m][pos];
            const double* c = &dec[m - 1][pos * D];
            double sum = 0.0;
            for (uint64_t d = 0; d < D; ++d) {
                const double diff = c[d] - x[d];
                sum += diff * diff;
            }
            R[m - 1][pos] = std::max(R[m - 1][pos], std::sqrt(sum));
            cnt[m - 1][pos] += 1;
        }
    }
    for (uint64_t m = 0; m + 1 < H; ++m) {
        const uint64_t n = idx->meshCount[m];
        for (uint64_t pos = 0; pos < n; ++pos) {
            const uint64_t orig = (m == 0) ? idx->coarseIds[pos] : idx->maps[m][pos];
            subRadius[m][orig] = R[m][pos] * (1.0 + kRelSlack) + kAbsSlack;
            leafCount[m][orig] = cnt[m][pos];
        }
    }
    return 0;
}

int oracle_brute_query(const double* points, const uint64_t* ids, uint64_t n, uint64_t D, int qtype, uint64_t nq,
                       const double* queries, uint64_t K, int threads, oracle_results* out) {
    const uint64_t stride = (qtype == ORACLE_RANGE) ? 2 * D : D;
    std::vector<std::vector<uint64_t>> res(nq);
    std::vector<std::vector<double>> d2(nq);
    std::vector<uint64_t> levels;
    if (threads <= 0) threads = omp_get_max_threads();
    constexpr uint64_t kTile = 64;  // queries per tile: one pass over the points serves 64 queries
    const uint64_t nTiles = (nq + kTile - 1) / kTile;
    if (qtype == ORACLE_RANGE) {
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
        for (int64_t t = 0; t < static_cast<int64_t>(nTiles); ++t) {
            const uint64_t q0 = t * kTile, q1 = std::min(nq, q0 + kTile);
            for (uint64_t i = 0; i < n; ++i) {
                const double* x = points + i * D;
                for (uint64_t q = q0; q < q1; ++q) {
                    const double* lo = queries + q * stride;
                    const double* hi = lo + D;
                    bool in = true;
                    for (uint64_t d = 0; d < D && in; ++d) in = (lo[d] <= x[d]) && (x[d] <= hi[d]);
                    if (in) res[q].push_back(ids[i]);
                }
            }
            for (uint64_t q = q0; q < q1; ++q) std::sort(res[q].begin(), res[q].end());
        }
    } else {
        // Bounded max-heap per query of (dist2, id) pairs: the K smallest under (dist2, id) order.
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
        for (int64_t t = 0; t < static_cast<int64_t>(nTiles); ++t) {
            const uint64_t q0 = t * kTile, q1 = std::min(nq, q0 + kTile);
            std::vector<std::vector<std::pair<double, uint64_t>>> heaps(q1 - q0);
            for (uint64_t i = 0; i < n; ++i) {
                const double* x = points + i * D;
                for (uint64_t q = q0; q < q1; ++q) {
                    const double dd = point_dist2(queries + q * stride, x, D, 1);
                    auto& h = heaps[q - q0];
                    const std::pair<double, uint64_t> e{dd, ids[i]};
                    if (h.size() < K) {
                        h.push_back(e);
                        std::push_heap(h.begin(), h.end());
                    } else if (K && e < h.front()) {
                        std::pop_heap(h.begin(), h.end());
                        h.back() = e;
                        std::push_heap(h.begin(), h.end());
                    }
                }
            }
            for (uint64_t q = q0; q < q1; ++q) {
                auto& h = heaps[q - q0];
                std::sort_heap(h.begin(), h.end());
                for (auto& e : h) {
                    res[q].push_back(e.second);
                    d2[q].push_back(e.first);
                }
            }
        }
    }
    pack_results(res, d2, 0, levels, qtype == ORACLE_KNN, out);
    return 0;
}

void oracle_free_results(oracle_results* r) {
    if (!r) return;
    std::free(r->offsets);
    std::free(r->ids);
    std::free(r->dist2);
    std::free(r->levelSizes);
    r->offsets = r->ids = r->levelSizes = nullptr;
    r->dist2 = nullptr;
}

}  // extern "C"
