"""GPU parity of the KNN path through the C ABI.

* the per-level plugin (IQueryStrategy::runLevel, KNN): device lower bounds (sqrt rounded down, like
  __dsqrt_rd in the reference), device sort and STEP; every level's grid equals the reference
  traversal's (oracle, pinned to the reference CUDA build), in the reference's order;
* batched exact KNN: the K nearest points by FP64 squared distance with id tie-break, identical
  ids and bit-identical squared distances to the FP64 brute force, for uniform and per-query K.
"""
import numpy as np
import pytest

from conftest import oracle_from_handler

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(tb, oracle_mod, tmp_path_factory, cuda):
    h = tb.QueryHandler.generate(200000, 5, 1.0, 100.0, False, 4, (40, 20, 10), 31, 2.2)
    h.prepare_for_query(tb.LevelPolicy.L0)
    o = oracle_from_handler(oracle_mod, h, tmp_path_factory.mktemp("idx"))
    pts, ids = oracle_mod.decoded_points(o)
    return h, o, pts, ids


def _points(pts, n, seed, noise=0.5):
    rng = np.random.default_rng(seed)
    return np.ascontiguousarray(pts[rng.integers(0, len(pts), n)] + rng.normal(0, noise, (n, pts.shape[1])))


def test_plugin_knn_levels_match_reference(tb, env, oracle_mod):
    h, o, pts, ids = env
    P = _points(pts, 10, 1)
    for K in (1, 10, 50):
        ref = oracle_mod.ref_query(o, oracle_mod.KNN, P, K=K, sorted_ids=False)
        for q in range(len(P)):
            grid = h.coarsest_grid()
            sizes = []
            for l in range(3):
                grid = h.run_level(l, grid, tb.QueryType.POINT, point=P[q], K=K)
                sizes.append(grid.nnz)
            got, _ = h.grid_arrays(grid)
            assert sizes == list(ref.level_sizes[q]), (K, q)
            assert np.array_equal(got, ref.query(q)), (K, q)


def test_plugin_knn_large_grid_sort(tb, oracle_mod, tmp_path, cuda):
    """A level whose grid exceeds one sort tile exercises the merge passes of the device sort."""
    h = tb.QueryHandler.generate(300000, 3, 1.0, 100.0, False, 3, (5, 3), 9, 3.0)
    h.prepare_for_query(tb.LevelPolicy.L0)
    o = oracle_from_handler(oracle_mod, h, tmp_path)
    pts, _ = oracle_mod.decoded_points(o)
    P = _points(pts, 3, 2)
    ref = oracle_mod.ref_query(o, oracle_mod.KNN, P, K=20, sorted_ids=False)
    for q in range(3):
        grid = h.coarsest_grid()
        assert grid.nnz > 2048 * 4
        for l in range(2):
            grid = h.run_level(l, grid, tb.QueryType.POINT, point=P[q], K=20)
        got, _ = h.grid_arrays(grid)
        assert np.array_equal(got, ref.query(q))


@pytest.mark.parametrize("K", [1, 10, 100])
def test_batched_exact_knn_equals_brute_force(tb, env, oracle_mod, K):
    h, o, pts, ids = env
    P = _points(pts, 200, 3 + K)
    r = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=K)
    offs, got, d2 = r.offsets.numpy(), r.ids.numpy(), r.dist2.numpy()
    b = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, P, K=K)
    assert np.array_equal(offs, b.offsets)
    assert np.array_equal(got, b.ids)
    assert np.array_equal(d2, b.dist2)


def test_batched_knn_per_query_k_and_edges(tb, env, oracle_mod):
    h, o, pts, ids = env
    P = _points(pts, 64, 7)
    P[0] = pts.max(0) + 50.0   # far outside the data
    P[1] = pts[123]            # exactly on a data point
    Ks = np.array([1, 2, 5, 20, 100, 0, 256, 3] * 8, dtype=np.uint32)
    r = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=Ks)
    offs, got, d2 = r.offsets.numpy(), r.ids.numpy(), r.dist2.numpy()
    for q in range(len(P)):
        b = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, P[q:q + 1], K=int(Ks[q]))
        assert np.array_equal(got[offs[q]:offs[q + 1]], b.ids), q
        assert np.array_equal(d2[offs[q]:offs[q + 1]], b.dist2), q
    assert offs[6] - offs[5] == 0          # K = 0
    assert got[offs[1]] == ids[123] and d2[offs[1]] == 0.0


def test_batched_knn_same_alone_and_in_batch(tb, env):
    h, o, pts, ids = env
    P = _points(pts, 32, 11)
    r = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=16)
    offs, got = r.offsets.numpy(), r.ids.numpy()
    for q in range(0, 32, 5):
        o1, i1, d1 = h.query_batch_host(tb.QueryType.POINT, P[q:q + 1], tb.Mode.EXACT, K=16)
        assert np.array_equal(i1, got[offs[q]:offs[q + 1]])


def test_knn_ref_parity_batch_is_rejected(tb, env):
    h, o, pts, ids = env
    with pytest.raises(tb.TblaeqError) as e:
        h.query_batch(tb.QueryType.POINT, pts[:2], tb.Mode.REF_PARITY, K=5)
    assert e.value.code == 1


def test_knn_first_batch_grows_every_buffer(tb, oracle_mod, cuda):
    """A fresh engine whose first KNN batch overflows the wave-2 result buffer grows it and reruns
    (wave-2 results have their own header; growth must read it, not double blindly)."""
    h = tb.QueryHandler.generate(100000, 8, 1.0, 100.0, False, 3, (100, 20), 57, 2.5)
    h.prepare_for_query(tb.LevelPolicy.L0)
    pts, ids = h.decode_points(np.arange(100000))
    P = _points(pts, 2000, 11, noise=1.0)
    r = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=20)
    c = h.knn_counters()
    assert c["wave2"] > 0
    b = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, P[:64], K=20)
    off = r.offsets.numpy()
    assert np.array_equal(off[:65], b.offsets)
    assert np.array_equal(r.ids.numpy()[:off[64]], b.ids)
    assert np.array_equal(r.dist2.numpy()[:off[64]], b.dist2)


def test_knn_batch_split_into_chunks(tb, env, oracle_mod):
    """A KNN batch whose workspace exceeds the traversal limit runs as chunks with the same results
    as one traversal (the limit is lowered here so a small index needs several chunks)."""
    h, o, pts, ids = env
    P = _points(pts, 400, 21)
    Kq = np.where(np.arange(400) % 2 == 0, 20, 100).astype(np.uint32)
    whole = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=Kq)
    w_off, w_ids, w_d2 = whole.offsets.numpy(), whole.ids.numpy(), whole.dist2.numpy()
    lib = tb.lib()
    assert lib.tblaeq_debug_split_above(h._h, 1 << 18) == 0
    try:
        r = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=Kq)
        assert np.array_equal(r.offsets.numpy(), w_off)
        assert np.array_equal(r.ids.numpy(), w_ids)
        assert np.array_equal(r.dist2.numpy(), w_d2)
        # (Counters are not compared: which clusters survive depends on when concurrent tau
        # tightenings land, while the results do not.)
        assert lib.tblaeq_debug_split_above(h._h, 50) == 0
        with pytest.raises(tb.TblaeqError):
            h.query_batch(tb.QueryType.POINT, P[:1], tb.Mode.EXACT, K=20)
    finally:
        lib.tblaeq_debug_split_above(h._h, 0)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, P[:50], K=20)
    r2 = h.query_batch(tb.QueryType.POINT, P[:50], tb.Mode.EXACT, K=20)
    assert np.array_equal(r2.ids.numpy(), b.ids) and np.array_equal(r2.dist2.numpy(), b.dist2)


@pytest.mark.parametrize("beam,completion", [(0, False), (32, False), (0, True), (32, True), (2, True)])
def test_probe_and_node_major_completion_stay_exact(tb, env, oracle_mod, beam, completion):
    """Every combination of the probe's beam (0: wave 1 ranks every surviving cluster) and the
    completion after wave 1 (node-major walk with the clusters' points read once per 32 queries, or
    the query-major wave 2) returns the FP64 brute force's ids and bit-identical squared distances."""
    h, o, pts, ids = env
    P = _points(pts, 300, 41)
    Kq = np.where(np.arange(300) % 3 == 0, 50, 10).astype(np.uint32)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, P[Kq == 10], K=10)
    b50 = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, P[Kq == 50], K=50)
    h.set_knn_probe(beam, completion)
    try:
        for _ in range(2):  # the first batch may grow the workspaces and rerun
            r = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=Kq)
            offs, got, d2 = r.offsets.numpy(), r.ids.numpy(), r.dist2.numpy()
            for bb, sel in ((b, np.nonzero(Kq == 10)[0]), (b50, np.nonzero(Kq == 50)[0])):
                for j, q in enumerate(sel):
                    assert np.array_equal(got[offs[q]:offs[q + 1]], bb.query(j)), (beam, completion, q)
                    assert np.array_equal(d2[offs[q]:offs[q + 1]], bb.dist2[bb.offsets[j]:bb.offsets[j + 1]])
        c = h.knn_counters()
        assert c["rows"] > 0
    finally:
        h.set_knn_probe(32, True)


@pytest.mark.parametrize("fail_at", [3, 8, 20])
def test_knn_batch_splits_when_an_allocation_fails(tb, oracle_mod, cuda, fail_at):
    """An allocation that fails while a KNN batch grows its workspace (the fail_at-th device
    allocation from the batch's start) leaves no buffer behind a stale capacity: the engine releases
    its workspace, the batch reruns as smaller traversals with the brute force's results, later
    batches start at the size that fitted, and closing the handle returns every byte."""
    lib = tb.lib()
    before = lib.tblaeq_live_device_bytes()
    h = tb.QueryHandler.generate(100000, 6, 1.0, 100.0, False, 4, (40, 20, 10), 77, 2.5)
    h.prepare_for_query(tb.LevelPolicy.L0)
    pts, ids = h.decode_points(np.arange(100000))
    P = _points(pts, 256, 5, noise=0.5)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, P, K=10)
    lib.tblaeq_debug_fail_alloc_after(fail_at)
    try:
        r = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=10)
    finally:
        lib.tblaeq_debug_fail_alloc_after(0)
    assert np.array_equal(r.offsets.numpy(), b.offsets)
    assert np.array_equal(r.ids.numpy(), b.ids) and np.array_equal(r.dist2.numpy(), b.dist2)
    info = h.knn_batch_info()
    r2 = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=10)
    assert np.array_equal(r2.ids.numpy(), b.ids)
    if info["traversals"] > 1:  # the failure hit the batch's growth: the next batch starts split
        assert h.knn_batch_info()["chunk"] == info["chunk"] < 256
    h.set_knn_chunk(0)
    r3 = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=10)
    assert np.array_equal(r3.ids.numpy(), b.ids) and {k: v for k, v in h.knn_batch_info().items() if k in ("chunk", "traversals")} == {"chunk": 256, "traversals": 1}
    h.set_knn_chunk(64)
    r4 = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=10)
    assert np.array_equal(r4.ids.numpy(), b.ids) and {k: v for k, v in h.knn_batch_info().items() if k in ("chunk", "traversals")} == {"chunk": 64, "traversals": 4}
    h.close()
    assert lib.tblaeq_live_device_bytes() == before


@pytest.mark.parametrize("scale", [0.5, 4.0, 64.0])
def test_wave_one_width_keeps_results(tb, env, oracle_mod, scale):
    """Wave 1's width (how many best-ranked clusters per query it reads before the bound is set)
    changes the work, never the results."""
    h, o, pts, ids = env
    P = _points(pts, 200, 51)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, P, K=30)
    h.set_knn_wave1(scale)
    try:
        r = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=30)
        assert np.array_equal(r.ids.numpy(), b.ids) and np.array_equal(r.dist2.numpy(), b.dist2)
    finally:
        h.set_knn_wave1(16.0)


@pytest.mark.parametrize("stride", [0, 3, 8])
def test_bound_refinement_keeps_results(tb, env, oracle_mod, stride):
    """The completion's bound refinement (a pass over every stride-th point of the listed clusters
    before the full point pass) changes the work, never the results."""
    h, o, pts, ids = env
    P = _points(pts, 250, 71)
    Kq = np.where(np.arange(250) % 2 == 0, 5, 40).astype(np.uint32)
    h.set_knn_refine(stride)
    try:
        r = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=Kq)
        offs, got, d2 = r.offsets.numpy(), r.ids.numpy(), r.dist2.numpy()
        for kv in (5, 40):
            sel = np.nonzero(Kq == kv)[0]
            b = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, P[sel], K=kv)
            for j, q in enumerate(sel):
                assert np.array_equal(got[offs[q]:offs[q + 1]], b.query(j)), (stride, q)
                assert np.array_equal(d2[offs[q]:offs[q + 1]], b.dist2[b.offsets[j]:b.offsets[j + 1]]), (stride, q)
    finally:
        h.set_knn_refine(16)


@pytest.mark.parametrize("D,ratios", [(8, (40, 20, 10)), (16, (40, 20, 10))])
def test_knn_point_groups_keep_results(tb, oracle_mod, cuda, D, ratios):
    """The completion's point pass over point groups (a group whose box lies beyond the query's
    bound is skipped; the decoded points are kept in group order) returns the FP64 brute force's
    ids and bit-identical squared distances, with the groups on and off and with and without the
    bound refinement."""
    h = tb.QueryHandler.generate(150000, D, 1.0, 100.0, False, 4, ratios, 90 + D, 2.5)
    h.prepare_for_query(tb.LevelPolicy.L0)
    N = h.info()["N"]
    pts, ids = h.decode_points(np.arange(N))
    P = _points(pts, 200, 91 + D, noise=1.0)
    Kq = np.where(np.arange(200) % 2 == 0, 10, 60).astype(np.uint32)
    bs = {kv: oracle_mod.brute_query(pts, ids, oracle_mod.KNN, P[Kq == kv], K=kv) for kv in (10, 60)}
    rows = {}
    try:
        for groups in (True, False):
            for stride in (16, 0):
                h.set_point_groups(groups)
                h.set_knn_refine(stride)
                r = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=Kq)
                offs, got, d2 = r.offsets.numpy(), r.ids.numpy(), r.dist2.numpy()
                for kv, b in bs.items():
                    for j, q in enumerate(np.nonzero(Kq == kv)[0]):
                        assert np.array_equal(got[offs[q]:offs[q + 1]], b.query(j)), (groups, stride, q)
                        assert np.array_equal(d2[offs[q]:offs[q + 1]], b.dist2[b.offsets[j]:b.offsets[j + 1]])
                rows[(groups, stride)] = h.knn_counters()["rows"]
    finally:
        h.set_point_groups(True)
        h.set_knn_refine(16)
    assert rows[(True, 16)] <= rows[(False, 16)]
