"""GPU parity of the range path through the C ABI against the CPU oracle.

* exact mode (batched and one query at a time) == FP64 brute force, bit-exact id sets;
* ref-parity mode == the oracle's restatement of the reference traversal: same candidate ids and
  the same per-level grid sizes (the reference's levelFineMeshSize);
* the per-level plugin (IQueryStrategy::runLevel) returns the reference's grid, in the reference's
  order, level by level;
* edge cases: empty boxes, boxes outside the data, a box holding every point, tiny and large
  batches (workspace growth), other dimensions (specialised and generic kernels).
"""
import ctypes

import numpy as np
import pytest

from conftest import ids_by_query, oracle_from_handler

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(tb, oracle_mod, tmp_path_factory, cuda):
    h = tb.QueryHandler.generate(200000, 5, 1.0, 100.0, False, 4, (40, 20, 10), 11, 2.2)
    h.prepare_for_query(tb.LevelPolicy.L0)
    o = oracle_from_handler(oracle_mod, h, tmp_path_factory.mktemp("idx"))
    pts, ids = oracle_mod.decoded_points(o)
    return h, o, pts, ids


def _boxes(pts, n, seed, lo_frac=0.005, hi_frac=0.15):
    rng = np.random.default_rng(seed)
    ext = pts.max(0) - pts.min(0)
    c = pts[rng.integers(0, len(pts), n)]
    hw = np.exp(rng.uniform(np.log(lo_frac), np.log(hi_frac), c.shape)) * ext
    return np.ascontiguousarray(np.concatenate([c - hw, c + hw], 1))


def _batch_ids(tb, h, Q, mode, flags=0):
    r = h.query_batch(tb.QueryType.RANGE, Q, mode, flags=flags)
    offs = r.offsets.numpy()
    ids = r.ids.numpy() if r.total else np.zeros(0, np.uint64)
    return r, offs, ids


def test_exact_batch_equals_brute_force(tb, env, oracle_mod):
    h, o, pts, ids = env
    Q = _boxes(pts, 300, 1)
    r, offs, got = _batch_ids(tb, h, Q, tb.Mode.EXACT)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, Q)
    assert np.array_equal(offs, b.offsets)
    for q, g in enumerate(ids_by_query(offs, got)):
        assert np.array_equal(g, b.query(q)), q
    assert b.offsets[-1] > 200


def test_exact_single_queries_equal_batch(tb, env):
    """Each query's result is the same alone and inside a batch."""
    h, o, pts, ids = env
    Q = _boxes(pts, 40, 2)
    r, offs, got = _batch_ids(tb, h, Q, tb.Mode.EXACT)
    batch = ids_by_query(offs, got)
    for q in range(len(Q)):
        o1, i1, _ = h.query_batch_host(tb.QueryType.RANGE, Q[q:q + 1], tb.Mode.EXACT)
        assert np.array_equal(np.sort(i1), batch[q])


def test_ref_parity_batch_equals_oracle(tb, env, oracle_mod):
    h, o, pts, ids = env
    Q = _boxes(pts, 200, 3)
    r, offs, got = _batch_ids(tb, h, Q, tb.Mode.REF_PARITY, flags=tb.WANT_LEVELS)
    ref = oracle_mod.ref_query(o, oracle_mod.RANGE, Q, sorted_ids=False)
    assert np.array_equal(offs, ref.offsets)
    # Same order as the reference (survivor order, then column order), not only the same set.
    assert np.array_equal(got, ref.ids)
    levels = r.level_items.numpy().T.astype(np.uint64)
    assert np.array_equal(levels, ref.level_sizes)


def test_plugin_levels_match_reference_order(tb, env, oracle_mod):
    """IQueryStrategy::runLevel on the device: grid after every level equals the reference's."""
    h, o, pts, ids = env
    Q = _boxes(pts, 12, 4)
    ref = oracle_mod.ref_query(o, oracle_mod.RANGE, Q, sorted_ids=False)
    D = 5
    for q in range(len(Q)):
        grid = h.coarsest_grid()
        sizes = []
        for l in range(3):
            grid = h.run_level(l, grid, tb.QueryType.RANGE, lo=Q[q, :D], hi=Q[q, D:])
            sizes.append(grid.nnz)
        got_ids, got_vals = h.grid_arrays(grid)
        assert np.array_equal(got_ids, ref.query(q)), q
        assert sizes == list(ref.level_sizes[q])
        # vals are the decoded coordinates of those ids
        pos = np.argsort(o.maps[3])
        assert np.array_equal(got_vals, pts[pos[got_ids.astype(np.int64)]])


def test_query_batch_host_matches_device(tb, env):
    h, o, pts, ids = env
    Q = _boxes(pts, 64, 5)
    r, offs, got = _batch_ids(tb, h, Q, tb.Mode.EXACT)
    hoffs, hids, _ = h.query_batch_host(tb.QueryType.RANGE, Q, tb.Mode.EXACT)
    assert np.array_equal(hoffs, offs) and np.array_equal(hids, got)


def test_edge_boxes(tb, env, oracle_mod):
    h, o, pts, ids = env
    D = 5
    lo, hi = pts.min(0), pts.max(0)
    Q = np.stack([
        np.concatenate([hi, lo]),                       # inverted box: empty
        np.concatenate([hi + 10, hi + 20]),             # outside the data
        np.concatenate([lo - 1, hi + 1]),               # every point
        np.concatenate([pts[17], pts[17]]),             # a single point (degenerate box)
        np.concatenate([lo - 50, lo - 40]),
    ])
    r, offs, got = _batch_ids(tb, h, Q, tb.Mode.EXACT)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, Q)
    assert np.array_equal(offs, b.offsets)
    per = ids_by_query(offs, got)
    assert len(per[0]) == 0 and len(per[1]) == 0 and len(per[4]) == 0
    assert len(per[2]) == len(pts)
    assert np.array_equal(per[2], np.arange(len(pts), dtype=np.uint64))
    assert ids[17] in per[3]


def test_empty_batch_and_single(tb, env):
    h, o, pts, ids = env
    r = h.query_batch(tb.QueryType.RANGE, np.zeros((0, 10)), tb.Mode.EXACT)
    assert r.total == 0 and r.offsets.numpy().tolist() == [0]


def test_large_results_force_workspace_growth(tb, env, oracle_mod):
    h, o, pts, ids = env
    Q = _boxes(pts, 48, 6, lo_frac=0.3, hi_frac=0.6)
    r, offs, got = _batch_ids(tb, h, Q, tb.Mode.REF_PARITY)
    ref = oracle_mod.ref_query(o, oracle_mod.RANGE, Q, sorted_ids=False)
    assert ref.offsets[-1] > 2_000_000
    assert np.array_equal(offs, ref.offsets) and np.array_equal(got, ref.ids)


@pytest.mark.parametrize("D,ratios", [(2, (16, 8, 4)), (3, (10, 10, 10)), (5, (40, 20, 10)), (6, (30, 10, 5)),
                                      (8, (100, 50, 20)), (16, (50, 20, 10)),
                                      # 40-100 children per node at the two finest levels: many
                                      # 32-item rounds lie in one entry and take the coalesced
                                      # single-entry tests (box prefilter and point test)
                                      (4, (100, 20, 10)), (4, (40, 40, 10)), (16, (40, 40, 10))])
def test_other_dimensions(tb, oracle_mod, tmp_path, cuda, D, ratios):
    """Both kernel variants (rows read straight into registers, or staged through shared memory by
    warp-wide chunk copies) give the oracle's results at every level, for even and odd D."""
    h = tb.QueryHandler.generate(60000 if D != 8 else 200000, D, 1.0, 100.0, False, 4, ratios, 5 + D, 3.0)
    h.prepare_for_query(tb.LevelPolicy.L0)
    o = oracle_from_handler(oracle_mod, h, tmp_path)
    pts, ids = oracle_mod.decoded_points(o)
    Q = _boxes(pts, 80, 7 + D, 0.02, 0.3)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, Q)
    ref = oracle_mod.ref_query(o, oracle_mod.RANGE, Q, sorted_ids=False)
    for variant in (0, 1):
        h.set_variants([variant] * 4)
        r, offs, got = _batch_ids(tb, h, Q, tb.Mode.EXACT)
        assert np.array_equal(offs, b.offsets), variant
        assert all(np.array_equal(g, b.query(q)) for q, g in enumerate(ids_by_query(offs, got))), variant
        r2, offs2, got2 = _batch_ids(tb, h, Q, tb.Mode.REF_PARITY)
        assert np.array_equal(got2, ref.ids), variant


def test_height_three_and_truncated_plan(tb, oracle_mod, tmp_path, cuda):
    h = tb.QueryHandler.generate(5000, 4, 1.0, 100.0, True, 3, (7, 9), 11, 1.5)
    h.prepare_for_query(tb.LevelPolicy.L0)
    o = oracle_from_handler(oracle_mod, h, tmp_path)
    pts, ids = oracle_mod.decoded_points(o)
    Q = _boxes(pts, 50, 8, 0.05, 0.4)
    r, offs, got = _batch_ids(tb, h, Q, tb.Mode.EXACT)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, Q)
    assert np.array_equal(offs, b.offsets)


def test_allocation_failure_surfaces_cleanly(tb, cuda):
    lib = tb.lib()
    h = tb.QueryHandler.generate(20000, 3, 1.0, 100.0, False, 4, (10, 10, 10), 1, 3.0)
    before = lib.tblaeq_live_device_bytes()
    lib.tblaeq_debug_fail_alloc_after(5)
    try:
        with pytest.raises(tb.TblaeqError) as e:
            h.prepare_for_query(tb.LevelPolicy.L0)
        assert e.value.code == 4
    finally:
        lib.tblaeq_debug_fail_alloc_after(0)
    assert lib.tblaeq_live_device_bytes() == before
    h.prepare_for_query(tb.LevelPolicy.L0)  # a later prepare succeeds
    h.close()
    assert lib.tblaeq_live_device_bytes() == before


@pytest.mark.parametrize("policy", [("L0", "L0", "L2"), ("L3", "L3", "L3"), ("L2", "L3", "L1")])
def test_streamed_levels_equal_resident(tb, oracle_mod, tmp_path, cuda, policy):
    """Intervals under L2 / L3 read their P rows (L3: and their maps) from page-locked host memory
    mapped into the device address space (the float copy and the point groups stay on the device
    when they fit). Results equal the resident index's: exact range (ids and coordinates) and KNN
    against the FP64 brute force, ref-parity range against the oracle's restatement of the
    reference, in the reference's order."""
    h = tb.QueryHandler.generate(200000, 8, 1.0, 100.0, False, 4, (100, 50, 20), 9, 3.0)
    h.prepare_for_query([tb.LevelPolicy[p] for p in policy])
    assert [p.name for p in h.info()["policy"]] == list(policy)
    o = oracle_from_handler(oracle_mod, h, tmp_path)
    pts, ids = oracle_mod.decoded_points(o)
    Q = _boxes(pts, 120, 21)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, Q)
    ref = oracle_mod.ref_query(o, oracle_mod.RANGE, Q, sorted_ids=False)
    for variant in (0, 1):
        h.set_variants([variant] * 4)
        r, offs, got = _batch_ids(tb, h, Q, tb.Mode.EXACT)
        assert np.array_equal(offs, b.offsets), variant
        assert all(np.array_equal(g, b.query(q)) for q, g in enumerate(ids_by_query(offs, got))), variant
        r2, offs2, got2 = _batch_ids(tb, h, Q, tb.Mode.REF_PARITY)
        assert np.array_equal(offs2, ref.offsets) and np.array_equal(got2, ref.ids), variant
        rv = h.query_batch(tb.QueryType.RANGE, Q, tb.Mode.EXACT, flags=tb.WANT_VALS)
        rows = {int(i): k for k, i in enumerate(ids)}
        assert np.array_equal(rv.vals.numpy(), pts[[rows[int(i)] for i in rv.ids.numpy()]]), variant
    rng = np.random.default_rng(4)
    P = np.ascontiguousarray(pts[rng.integers(0, len(pts), 60)] + rng.normal(0, 0.5, (60, 8)))
    rk = h.query_batch(tb.QueryType.POINT, P, tb.Mode.EXACT, K=15)
    bk = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, P, K=15)
    assert np.array_equal(rk.ids.numpy(), bk.ids) and np.array_equal(rk.dist2.numpy(), bk.dist2)


def test_lookback_timeout_is_reported_and_the_handle_recovers(tb, env, oracle_mod):
    """Failure detection without a fault: a work tile that never publishes its counts makes its
    successors' look-back waits run out (bounded spins). The kernel sets its timeout status and
    returns, the later launches of the batch skip their work, and the call fails with
    TBLAEQ_ERR_TIMEOUT. The CUDA context stays usable: the next batch on the same handle is exact."""
    h, o, pts, ids = env
    lib = tb.lib()
    Q = _boxes(pts, 300, 9)  # 300 queries x 25 coarsest nodes: 30 work tiles at the first level
    lo, hi = pts.min(0) - 1.0, pts.max(0) + 1.0  # every cluster survives
    grid = h.run_level(0, h.coarsest_grid(), tb.QueryType.RANGE, lo=lo, hi=hi)  # 250 nodes of mesh 1
    n_mesh1 = grid.nnz
    lib.tblaeq_debug_lookback_timeout(1, 2000)
    try:
        with pytest.raises(tb.TblaeqError) as e:
            h.query_batch(tb.QueryType.RANGE, Q, tb.Mode.EXACT)
        assert e.value.code == 6, e.value
        with pytest.raises(tb.TblaeqError) as e:
            h.run_level(1, grid, tb.QueryType.RANGE, lo=lo, hi=hi)  # 5,000 children: 20 work tiles
        assert e.value.code == 6, e.value
    finally:
        lib.tblaeq_debug_lookback_timeout(2**64 - 1, 0)
    r, offs, got = _batch_ids(tb, h, Q, tb.Mode.EXACT)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, Q)
    assert np.array_equal(offs, b.offsets)
    for q, g in enumerate(ids_by_query(offs, got)):
        assert np.array_equal(g, b.query(q)), q
    assert n_mesh1 == h.info()["meshSizes"][2]
    g2 = h.run_level(1, grid, tb.QueryType.RANGE, lo=lo, hi=hi)
    assert g2.nnz == h.info()["meshSizes"][1]


def test_autotuned_launch_shapes_keep_results_and_round_trip(tb, env, oracle_mod, tmp_path):
    """Every launch shape the autotuner searches (variant x persistent grid size) returns the same
    exact results; the chosen shapes go to the tuning cache and come back on the next lookup."""
    import torch
    h, o, pts, ids = env
    Q = _boxes(pts, 256, 21)
    dQ = torch.from_numpy(Q).cuda()
    b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, Q)
    H = h.info()["height"]
    for v, g in ((0, 25), (1, 50), (0, 75), (1, 100)):
        h.set_launch_shapes([v] * H, [g] * H)
        r, offs, got = _batch_ids(tb, h, dQ, tb.Mode.EXACT)
        assert np.array_equal(offs, b.offsets), (v, g)
        assert all(np.array_equal(a, c) for a, c in zip(ids_by_query(offs, got), [b.query(q) for q in range(len(Q))]))
    cache = str(tmp_path / "tuning.txt")
    v1, g1, ms, src = h.autotune_cached(dQ, cache, tb.Mode.EXACT, reps=2)
    assert src == "tuned" and len(v1) == len(g1) == H and all(x in (25, 50, 75, 100) for x in g1)
    h.set_launch_shapes([0] * H, [100] * H)
    v2, g2, _, src2 = h.autotune_cached(dQ, cache, tb.Mode.EXACT, reps=2)
    assert src2 == "cache" and (v2, g2) == (v1, g1) and h.launch_shapes() == (v1, g1)
    h.set_launch_shapes([0] * H, [100] * H)


@pytest.mark.parametrize("flags", [0, 2, 1])  # plain, WANT_LEVELS, WANT_VALS
def test_node_major_levels_equal_entry_major(tb, env, oracle_mod, flags):
    """Node-major inner levels (one warp per node and 32 of its queries) keep exactly the children the
    entry-major kernel keeps: identical per-level frontier sizes and per-query level counts, and the
    same exact results (as sets; node-major leaves each query's ids in no particular order)."""
    h, o, pts, ids = env
    Q = _boxes(pts, 700, 31, hi_frac=0.3)  # a workspace that grows: several growth steps
    b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, Q)
    out = {}
    H = h.info()["height"]
    for nm in (False, True):
        h.set_launch_shapes([2 if nm else 0] * H, [100] * H)  # variant 2: node-major inner levels
        r = h.query_batch(tb.QueryType.RANGE, Q, tb.Mode.EXACT, flags=flags)
        offs, got = r.offsets.numpy(), r.ids.numpy()
        lv = r.level_items.numpy().copy() if r.level_items is not None else None
        vals = r.vals.numpy().copy() if r.vals is not None else None
        out[nm] = (offs.copy(), ids_by_query(offs, got), h.level_counts(), lv, vals, got.copy())
        assert np.array_equal(offs, b.offsets)
        assert all(np.array_equal(g, b.query(q)) for q, g in enumerate(out[nm][1]))
    assert out[False][2] == out[True][2]  # same frontier entries and children at every level
    if flags == 2:
        assert np.array_equal(out[False][3], out[True][3])
    if flags == 1:
        # Each id keeps its own coordinates.
        for nm in (False, True):
            o_, _, _, _, vals, got = out[nm]
            order = np.argsort(got)
            rows = dict(zip(ids.tolist(), range(len(ids))))
            assert np.array_equal(vals[order], pts[[rows[int(i)] for i in got[order]]])
    # Mixed: node-major at one level only, entry-major below it.
    h.set_launch_shapes([0, 2] + [0] * (H - 2), [100] * H)
    r = h.query_batch(tb.QueryType.RANGE, Q, tb.Mode.EXACT, flags=flags)
    assert np.array_equal(r.offsets.numpy(), b.offsets)
    assert all(np.array_equal(g, b.query(q)) for q, g in enumerate(ids_by_query(r.offsets.numpy(), r.ids.numpy())))
    h.set_node_major(False)  # node-major disabled: the variant launches entry-major
    r = h.query_batch(tb.QueryType.RANGE, Q, tb.Mode.EXACT, flags=flags)
    assert np.array_equal(r.ids.numpy(), out[False][5])
    h.set_node_major(True)
    h.set_launch_shapes([0] * H, [100] * H)


@pytest.mark.parametrize("D,ratios", [(4, (100, 20, 10)), (8, (100, 50, 20)), (16, (40, 40, 10))])
def test_float_points_decide_exactly_at_box_faces(tb, oracle_mod, tmp_path, cuda, D, ratios):
    """The finest level decides points from their float copies and takes the FP64 test only near a
    face. Boxes whose faces lie exactly on decoded coordinates, one double ulp beside them or one
    float ulp beside them give the FP64 brute force's results, with the float copies on and off."""
    h = tb.QueryHandler.generate(60000 if D != 8 else 200000, D, 1.0, 100.0, False, 4, ratios, 5 + D, 3.0)
    h.prepare_for_query(tb.LevelPolicy.L0)
    o = oracle_from_handler(oracle_mod, h, tmp_path)
    pts, ids = oracle_mod.decoded_points(o)
    rng = np.random.default_rng(100 + D)
    n = 480
    c = pts[rng.integers(0, len(pts), n)]
    hw = np.exp(rng.uniform(np.log(0.01), np.log(0.2), c.shape)) * (pts.max(0) - pts.min(0))
    lo, hi = c - hw, c + hw
    g = n // 6
    fulp = np.spacing(np.abs(c).astype(np.float32)).astype(np.float64)
    lo[0 * g:1 * g] = c[0 * g:1 * g]                                # the centre on every lower face
    hi[1 * g:2 * g] = c[1 * g:2 * g]                                # ... on every upper face
    lo[2 * g:3 * g] = np.nextafter(c[2 * g:3 * g], np.inf)          # one double ulp above it: out
    hi[3 * g:4 * g] = np.nextafter(c[3 * g:4 * g], -np.inf)         # one double ulp below it: out
    lo[4 * g:5 * g] = c[4 * g:5 * g] - fulp[4 * g:5 * g] / 2        # half a float ulp below it
    hi[5 * g:6 * g] = c[5 * g:6 * g] + fulp[5 * g:6 * g] / 2        # half a float ulp above it
    Q = np.ascontiguousarray(np.concatenate([lo, hi], 1))
    b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, Q)
    try:
        for on in (True, False):
            h.set_float_points(on)
            r, offs, got = _batch_ids(tb, h, Q, tb.Mode.EXACT)
            assert np.array_equal(offs, b.offsets), on
            assert all(np.array_equal(gq, b.query(q)) for q, gq in enumerate(ids_by_query(offs, got))), on
    finally:
        h.set_float_points(True)
    sizes = np.diff(b.offsets.astype(np.int64))
    assert np.all(sizes[:2 * g] >= 1) and np.all(sizes[2 * g:4 * g] >= 0)


@pytest.mark.parametrize("D,ratios", [(4, (100, 20, 10)), (8, (100, 50, 20)), (16, (40, 40, 10))])
def test_point_groups_keep_results(tb, oracle_mod, tmp_path, cuda, D, ratios):
    """Testing the finest clusters' point groups (at most 32 points, with their boxes) before their
    points changes which points are tested, never the results: ids equal the FP64 brute force with
    groups on and off, entry-major and node-major, and so do the coordinates (WANT_VALS: every id
    keeps its own point). Far fewer points are tested with the groups."""
    h = tb.QueryHandler.generate(60000 if D != 8 else 200000, D, 1.0, 100.0, False, 4, ratios, 15 + D, 3.0)
    h.prepare_for_query(tb.LevelPolicy.L0)
    o = oracle_from_handler(oracle_mod, h, tmp_path)
    pts, ids = oracle_mod.decoded_points(o)
    Q = _boxes(pts, 300, 60 + D, 0.005, 0.2)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, Q)
    rows = {int(i): k for k, i in enumerate(ids)}
    H = h.info()["height"]
    tested = {}
    try:
        for groups in (True, False):
            h.set_point_groups(groups)
            for shapes in ([0] * H, [0, 2, 2, 0][:H]):
                h.set_launch_shapes(shapes, [100] * H)
                r = h.query_batch(tb.QueryType.RANGE, Q, tb.Mode.EXACT, flags=tb.WANT_VALS)
                offs, got, vals = r.offsets.numpy(), r.ids.numpy(), r.vals.numpy()
                assert np.array_equal(offs, b.offsets), (groups, shapes)
                assert all(np.array_equal(g, b.query(q)) for q, g in enumerate(ids_by_query(offs, got))), (groups, shapes)
                assert np.array_equal(vals, pts[[rows[int(i)] for i in got]]), (groups, shapes)
                c = h.group_counts()
                if groups:
                    assert 0 < c["kept"] <= c["groups"] and c["points"] > 0
                    tested[groups] = c["points"]
                else:
                    assert c == {"groups": 0, "kept": 0, "points": 0}
                    tested[groups] = h.level_counts()[1][H - 1]
        # Per-level counts are the points of the surviving clusters: the batch tests every point.
        h.set_point_groups(True)
        h.set_launch_shapes([0] * H, [100] * H)
        r = h.query_batch(tb.QueryType.RANGE, Q, tb.Mode.EXACT, flags=tb.WANT_LEVELS)
        assert h.group_counts()["groups"] == 0
        ref = oracle_mod.exact_query(o, oracle_mod.RANGE, Q)
        assert np.array_equal(r.offsets.numpy(), ref.offsets)
    finally:
        h.set_point_groups(True)
        h.set_launch_shapes([0] * H, [100] * H)
    assert tested[True] < tested[False]
