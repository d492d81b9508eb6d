"""Serving loop through the C ABI: continuous batching of mixed range and KNN requests.

* every request's result in the mix equals the same request run alone (exact mode: identical id
  sets; KNN: identical ids and squared distances), and a sample equals the FP64 brute force;
* requests that arrive while a batch is on the GPU are batched together (mean batch > 1 under a
  burst), while a one-slot, one-lane server serves them one at a time with the same results;
* the learned ranking, when trained, is used by the server's KNN lane and changes no result;
* stop() drains the queue; bad requests are rejected on the host.
"""
import numpy as np
import pytest

from conftest import oracle_from_handler

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(tb, oracle_mod, tmp_path_factory, cuda):
    h = tb.QueryHandler.generate(300000, 6, 1.0, 100.0, False, 4, (60, 30, 15), 77, 2.5)
    h.prepare_for_query(tb.LevelPolicy.L0)
    o = oracle_from_handler(oracle_mod, h, tmp_path_factory.mktemp("idx"))
    pts, ids = oracle_mod.decoded_points(o)
    return h, pts, ids


def _mix(pts, n, seed):
    """n requests, half range boxes and half KNN points, as rows padded to 2D values."""
    rng = np.random.default_rng(seed)
    D = pts.shape[1]
    ext = pts.max(0) - pts.min(0)
    qt = rng.integers(0, 2, n).astype(np.int32)  # 0 = KNN, 1 = range
    rows = np.zeros((n, 2 * D))
    K = np.zeros(n, np.uint32)
    c = pts[rng.integers(0, len(pts), n)]
    hw = np.exp(rng.uniform(np.log(0.001), np.log(0.05), (n, D))) * ext
    rows[qt == 1] = np.concatenate([c - hw, c + hw], 1)[qt == 1]
    rows[qt == 0, :D] = (c + rng.normal(0, 0.01, (n, D)) * ext)[qt == 0]
    K[qt == 0] = np.floor(np.exp(rng.uniform(0, np.log(256), (qt == 0).sum()))).astype(np.uint32)
    return qt, rows, K


def _alone(tb, h, qt, row, k, D):
    if qt == 1:
        r = h.query_batch(tb.QueryType.RANGE, row[None, :2 * D], tb.Mode.EXACT)
        return np.sort(r.ids.numpy()), None
    r = h.query_batch(tb.QueryType.POINT, row[None, :D], tb.Mode.EXACT, K=int(k))
    return r.ids.numpy(), r.dist2.numpy()


def _check_same(tb, h, srv, tickets, qt, rows, K, D, sample=None):
    for i in (range(len(tickets)) if sample is None else sample):
        got = srv.poll(int(tickets[i]), 60000)
        assert got is not None, i
        ids, d2, lat = got
        ref_ids, ref_d2 = _alone(tb, h, qt[i], rows[i], K[i], D)
        if qt[i] == 1:
            assert np.array_equal(np.sort(ids), ref_ids), i
        else:
            assert np.array_equal(ids, ref_ids), i
            assert np.array_equal(d2, ref_d2), i
        assert lat > 0


def test_mix_equals_alone_and_brute_force(tb, env, oracle_mod):
    h, pts, ids = env
    D = pts.shape[1]
    qt, rows, K = _mix(pts, 600, 1)
    at = np.sort(np.random.default_rng(2).uniform(0, 20000, len(qt)))  # a 20 ms burst
    with tb.Server(h, max_batch=256) as srv:
        tickets = srv.replay(qt, rows, K, at)
        assert srv.wait_idle(120000)
        st = srv.stats()
        assert st["completed"] == len(qt) and st["failed"] == 0
        assert st["mean_batch"] > 1.0 and st["max_batch"] <= 256
        assert 0 < st["p50_us"] <= st["p99_us"] <= st["max_us"]
        # every result equals the request alone; a sample against the brute force too
        results = {}
        for i in range(len(qt)):
            results[i] = srv.poll(int(tickets[i]), 0)
    for i in range(len(qt)):
        got_ids, got_d2, _ = results[i]
        ref_ids, ref_d2 = _alone(tb, h, qt[i], rows[i], K[i], D)
        if qt[i] == 1:
            assert np.array_equal(np.sort(got_ids), ref_ids), i
        else:
            assert np.array_equal(got_ids, ref_ids) and np.array_equal(got_d2, ref_d2), i
    for i in range(0, len(qt), 37):
        if qt[i] == 1:
            b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, rows[i:i + 1])
            assert np.array_equal(np.sort(results[i][0]), b.query(0)), i
        else:
            b = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, rows[i:i + 1, :D], K=int(K[i]))
            assert np.array_equal(results[i][0], b.ids) and np.array_equal(results[i][1], b.dist2), i


def test_one_slot_server_serves_one_at_a_time(tb, env):
    h, pts, ids = env
    D = pts.shape[1]
    qt, rows, K = _mix(pts, 60, 3)
    with tb.Server(h, max_batch=1, lanes=1) as srv:
        tickets = [srv.submit(tb.QueryType(int(qt[i])), rows[i, :2 * D] if qt[i] == 1 else rows[i, :D], int(K[i]))
                   for i in range(len(qt))]
        assert srv.wait_idle(120000)
        st = srv.stats(reset=True)
        assert st["max_batch"] == 1 and st["batches"] == len(qt)
        _check_same(tb, h, srv, tickets, qt, rows, K, D)
        assert srv.stats()["completed"] == 0  # reset


def test_learned_lane_keeps_results(tb, env):
    h, pts, ids = env
    D = pts.shape[1]
    rng = np.random.default_rng(5)
    T = pts[rng.integers(0, len(pts), 800)] + rng.normal(0, 0.5, (800, D))
    h.scorer_train(T, K=20, max_samples=50000, epochs=3, seed=3)
    h.scorer_enable(False)
    qt, rows, K = _mix(pts, 200, 7)
    qt[:] = 0
    rows[:, :D] = pts[rng.integers(0, len(pts), 200)] + rng.normal(0, 0.5, (200, D))
    K[:] = np.maximum(K, 1)
    with tb.Server(h, learned=True) as srv:
        tickets = srv.replay(qt, rows, K, np.zeros(len(qt)))
        assert srv.wait_idle(120000)
        _check_same(tb, h, srv, tickets, qt, rows, K, D, sample=range(0, 200, 3))


def test_stop_drains_and_bad_requests(tb, env):
    h, pts, ids = env
    D = pts.shape[1]
    qt, rows, K = _mix(pts, 300, 9)
    srv = tb.Server(h, max_batch=64)
    srv.replay(qt, rows, K, np.zeros(len(qt)))
    with pytest.raises(tb.TblaeqError):
        srv.submit(7, rows[0], 1)
    with pytest.raises(tb.TblaeqError):
        srv.poll(10 ** 9, 0)
    srv.stop()  # drains what was queued, then frees the server
    srv.stop()
