"""HTTP front end (the reference's src/HTTPServer.cu routes) over the real serving loop on the GPU.

* concurrent /query requests (range and KNN, from many client threads) are batched by the serving
  loop, and each response's `result` equals the same query run alone through the library (exact
  mode: the same id set for range, the same ids in distance order for KNN); a sample equals the
  FP64 brute force; a range response's `level_pruned_sizes` equals the per-level child counts of
  the query alone;
* /build-index builds an index from a dataset text file on the GPU and saves it in the cache,
  /datasets lists it, and /query on it answers like the brute force over its decoded points.
"""
import json
import threading
import urllib.error
import urllib.request
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from conftest import oracle_from_handler

pytestmark = pytest.mark.gpu


def _post(url, path, obj):
    req = urllib.request.Request(url + path, data=json.dumps(obj).encode(),
                                 headers={"Content-Type": "application/json"}, method="POST")
    try:
        with urllib.request.urlopen(req, timeout=300) as r:
            return r.status, json.loads(r.read())
    except urllib.error.HTTPError as e:
        return e.code, json.loads(e.read())


@pytest.fixture(scope="module")
def site(tb, oracle_mod, tmp_path_factory, cuda):
    import importlib
    http = importlib.import_module("tblaeq_b200.http_server")
    root = tmp_path_factory.mktemp("cache")
    h = tb.QueryHandler.generate(200000, 5, 1.0, 100.0, False, 4, (50, 20, 10), 21, 2.5)
    h.save_index(str(root / "synth"))
    h.prepare_for_query(tb.LevelPolicy.L0)
    o = oracle_from_handler(oracle_mod, h, tmp_path_factory.mktemp("o"))
    pts, ids = oracle_mod.decoded_points(o)
    manager = http.IndexManager(str(root))
    httpd = http.make_server(http.QueryService(manager), "127.0.0.1", 0)
    t = threading.Thread(target=httpd.serve_forever, daemon=True)
    t.start()
    yield {"url": f"http://127.0.0.1:{httpd.server_address[1]}", "h": h, "pts": pts, "ids": ids,
           "manager": manager}
    httpd.shutdown()
    httpd.server_close()
    manager.close()


def test_concurrent_queries_equal_alone(tb, site, oracle_mod):
    h, pts, ids, url = site["h"], site["pts"], site["ids"], site["url"]
    D = pts.shape[1]
    rng = np.random.default_rng(8)
    ext = pts.max(0) - pts.min(0)
    reqs = []
    for i in range(64):
        c = pts[rng.integers(0, len(pts))]
        if i % 2:
            hw = np.exp(rng.uniform(np.log(0.005), np.log(0.05), D)) * ext
            reqs.append({"dataset_name": "synth", "query_type": "RANGE", "lower_bound": list(c - hw),
                         "upper_bound": list(c + hw)})
        else:
            reqs.append({"dataset_name": "synth", "query_type": "knn",
                         "query_point": list(c + rng.normal(0, 0.01, D) * ext), "k": int(rng.integers(1, 40))})
    with ThreadPoolExecutor(16) as ex:
        out = list(ex.map(lambda r: _post(url, "/query", r), reqs))
    for i, (r, (status, body)) in enumerate(zip(reqs, out)):
        assert status == 200 and body["success"] is True, (i, body)
        assert body["result_count"] == len(body["result"])
        got = np.array(body["result"], dtype=np.uint64)
        if r["query_type"] == "RANGE":
            box = np.concatenate([r["lower_bound"], r["upper_bound"]])[None, :]
            alone = h.query_batch(tb.QueryType.RANGE, box, tb.Mode.EXACT, flags=tb.WANT_LEVELS)
            assert np.array_equal(np.sort(got), np.sort(alone.ids.numpy())), i
            assert body["level_pruned_sizes"] == [int(x) for x in alone.level_items.numpy()[:, 0]], i
            if i % 7 == 1:
                b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, box)
                assert np.array_equal(np.sort(got), b.query(0)), i
        else:
            p = np.array(r["query_point"])[None, :]
            alone = h.query_batch(tb.QueryType.POINT, p, tb.Mode.EXACT, K=r["k"])
            assert np.array_equal(got, alone.ids.numpy()), i
            if i % 8 == 0:
                b = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, p, K=r["k"])
                assert np.array_equal(got, b.ids), i
        assert len(body["level_original_sizes"]) == 3 and body["query_runtime"]["query_count"] == 1
    status, body = _post(url, "/query", {"dataset_name": "synth", "query_type": "KNN", "query_point": [0, 0]})
    assert status == 400 and body["message"] == "query_point dimension mismatch: expected 5"


def test_build_index_from_text_file(tb, site, oracle_mod, tmp_path):
    url = site["url"]
    rng = np.random.default_rng(12)
    centres = rng.uniform(0, 1, (60, 4))
    X = np.concatenate([centres[rng.integers(0, 60, 24000)] + rng.normal(0, 0.01, (24000, 4)),
                        rng.uniform(0, 1, (6000, 4))])
    path = tmp_path / "clusters_4d.txt"
    with open(path, "w") as f:
        f.write(f"{len(X)} 4\n")
        for r in X:
            f.write(" ".join("%.9g" % v for v in r) + "\n")
    status, body = _post(url, "/build-index", {"dataset_name": "built", "dataset_path": str(path)})
    assert status == 200 and body["already_exists"] is False, body
    status, body = _post(url, "/build-index", {"dataset_name": "built"})
    assert status == 200 and body["already_exists"] is True
    with urllib.request.urlopen(url + "/datasets", timeout=60) as r:
        assert json.loads(r.read())["datasets"] == ["built", "synth"]
    hb = site["manager"].get_or_load("built")["handler"]
    info = hb.info()
    assert info["N"] == 30000 and info["meshSizes"][:4] == [30000, 300, 6, 1]
    o = oracle_from_handler(oracle_mod, hb, tmp_path / "o")
    pts, ids = oracle_mod.decoded_points(o)
    assert np.allclose(pts[np.argsort(ids)], X, atol=1e-5)
    lo, hi = np.full(4, 0.2), np.full(4, 0.6)
    status, body = _post(url, "/query", {"dataset_name": "built", "query_type": "RANGE", "lower_bound": list(lo),
                                         "upper_bound": list(hi)})
    b = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE, np.concatenate([lo, hi])[None, :])
    assert status == 200 and np.array_equal(np.sort(np.array(body["result"], np.uint64)), b.query(0))
    q = X[17] + 0.001
    status, body = _post(url, "/query", {"dataset_name": "built", "query_type": "KNN", "query_point": list(q), "k": 25})
    b = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, q[None, :], K=25)
    assert status == 200 and np.array_equal(np.array(body["result"], np.uint64), b.ids)
