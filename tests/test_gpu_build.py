"""GPU k-means index build (the reference's IndexBuilder::build) through the C ABI.

* one assignment pass on the tensor cores (tcgen05, TF32 hi/lo split, FP32 accumulation) labels
  the points like the FP64 CUDA-core reference (>= 99.5%, the rest are near-ties), and after
  several Lloyd iterations the objective is within 1e-3 of the FP64 build from the same start;
* a whole built index matches the FP64 build's per-level objectives within 1e-3, validates, round
  trips through the reference's on-disk layout, and answers exact range and KNN queries exactly
  like the FP64 brute force over its own decoded points.
"""
import numpy as np
import pytest

from conftest import oracle_from_handler

pytestmark = pytest.mark.gpu


def _mixture(n, D, seed, nclusters=None):
    """80% of the points in Gaussian clusters (sigma 0.01, centres uniform in [0,1]^D), 20% uniform."""
    rng = np.random.default_rng(seed)
    ncl = nclusters or max(1, n // 400)
    centres = rng.uniform(0, 1, (ncl, D))
    m = int(n * 0.8)
    X = np.concatenate([centres[rng.integers(0, ncl, m)] + rng.normal(0, 0.01, (m, D)),
                        rng.uniform(0, 1, (n - m, D))])
    return np.ascontiguousarray(rng.permutation(X).astype(np.float32))


@pytest.mark.parametrize("D", [16, 8, 3])
def test_tensor_assignment_matches_fp64(tb, cuda, D):
    X = _mixture(60000, D, 1 + D)
    k = 600
    _, L64, o64 = tb.kmeans(X, k, iters=1, seed=5, precision=tb.KmeansPrecision.FP64)
    _, Lt, ot = tb.kmeans(X, k, iters=1, seed=5, precision=tb.KmeansPrecision.TENSOR)
    assert np.mean(Lt == L64) >= 0.995
    assert abs(ot[-1] - o64[-1]) <= 1e-4 * o64[-1]
    _, _, o64 = tb.kmeans(X, k, iters=8, seed=5, precision=tb.KmeansPrecision.FP64)
    _, _, ot = tb.kmeans(X, k, iters=8, seed=5, precision=tb.KmeansPrecision.TENSOR)
    assert abs(ot[-1] - o64[-1]) <= 1e-3 * o64[-1]
    assert np.all(np.diff(ot) <= 1e-5 * ot[0])  # Lloyd never increases the objective (up to near-ties)


def test_kmeans_edges(tb, cuda):
    X = _mixture(1000, 16, 3)
    C, L, o = tb.kmeans(X, 1000, iters=2, seed=1)  # k = n: every point its own centroid
    assert o[-1] <= 1e-9
    C, L, o = tb.kmeans(X, 1, iters=2, seed=1)      # k = 1: the mean
    assert np.allclose(C[0], X.astype(np.float64).mean(0), atol=1e-6)
    with pytest.raises(tb.TblaeqError):
        tb.kmeans(X, 1001, iters=1)
    C, L, o = tb.kmeans(X[:, :20 % 16 + 1], 10, iters=2, seed=1)
    assert L.max() < 10


def test_built_index_objective_and_exact_queries(tb, oracle_mod, tmp_path, cuda):
    X = _mixture(200000, 16, 7, nclusters=500)
    h, rep = tb.QueryHandler.build(X, height=4, ratios=(100, 50, 20), iters=10, seed=11)
    h64, rep64 = tb.QueryHandler.build(X, height=4, ratios=(100, 50, 20), iters=10, seed=11,
                                       precision=tb.KmeansPrecision.FP64)
    assert [r["k"] for r in rep] == [2000, 40, 2]
    # The first level starts from the same sample; upper levels cluster slightly different data.
    assert abs(rep[0]["objective"] - rep64[0]["objective"]) <= 1e-3 * rep64[0]["objective"]
    for r, r64 in zip(rep[1:], rep64[1:]):
        assert abs(r["objective"] - r64["objective"]) <= 2e-2 * r64["objective"]
    info = h.info()
    assert info["N"] == 200000 and info["meshSizes"][:4] == [200000, 2000, 40, 2]
    o = oracle_from_handler(oracle_mod, h, tmp_path / "built")
    pts, ids = oracle_mod.decoded_points(o)
    assert np.allclose(pts[np.argsort(ids)], X.astype(np.float64), atol=1e-5)
    h.prepare_for_query(tb.LevelPolicy.L0)
    rng = np.random.default_rng(3)
    c = pts[rng.integers(0, len(pts), 200)]
    hw = np.exp(rng.uniform(np.log(0.002), np.log(0.05), c.shape))
    boxes = np.ascontiguousarray(np.concatenate([c - hw, c + hw], 1))
    r = h.query_batch(tb.QueryType.RANGE, boxes, tb.Mode.EXACT)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, boxes)
    offs, got = r.offsets.numpy(), r.ids.numpy()
    assert np.array_equal(offs, b.offsets)
    for q in range(len(boxes)):
        assert np.array_equal(np.sort(got[offs[q]:offs[q + 1]]), b.query(q)), q
    P = np.ascontiguousarray(pts[rng.integers(0, len(pts), 100)] + rng.normal(0, 0.01, (100, 16)))
    rk = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=10)
    bk = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, P, K=10)
    assert np.array_equal(rk.ids.numpy(), bk.ids) and np.array_equal(rk.dist2.numpy(), bk.dist2)


def test_device_assembly_writes_the_host_assembly_bytes(tb, tmp_path, cuda):
    """The P-tensors, maps and radii assembled on the device (labels and centroids never leave it)
    are byte-identical to the host assembly (the reference's Genenate_One_P_Tensor /
    Compute_Max_Radius order of work) from the same labels and centroids: the build's `both` mode
    assembles every level both ways and fails on any difference. (Two separate builds are not
    compared: k-means itself is not bitwise repeatable, its FP64 sums are atomic.)"""
    X = _mixture(300000, 8, 13, nclusters=700)
    h, rep = tb.QueryHandler.build(X, height=4, ratios=(50, 20, 10), iters=4, seed=3, host_assembly=2)
    assert [r["k"] for r in rep] == [6000, 300, 30]
    assert all(r["assemble_seconds"] > 0 for r in rep)
    hd, _ = tb.QueryHandler.build(X, height=4, ratios=(50, 20, 10), iters=4, seed=3)
    info = hd.info()
    assert info["meshSizes"][:4] == [300000, 6000, 300, 30]
    h.save_index(str(tmp_path / "both"))
