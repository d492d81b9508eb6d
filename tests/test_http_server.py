"""HTTP front end (the reference's src/HTTPServer.cu routes) on the CPU, over a fake serving loop:
request validation and error messages, the response shape, and a real HTTP round trip on
127.0.0.1. The GPU test (test_gpu_http.py) runs the same routes over the real serving loop."""
import json
import os
import threading
import urllib.error
import urllib.request

import numpy as np
import pytest


@pytest.fixture(scope="module")
def http(tb):
    import importlib
    return importlib.import_module("tblaeq_b200.http_server")


class FakeServer:
    """Answers every request with ids 0..n-1 (n = K for KNN, 3 for range) and fixed level counts."""

    def __init__(self, tb):
        self.tb = tb
        self.requests = []
        self.results = {}
        self.lock = threading.Lock()  # HTTP handler threads submit concurrently

    def submit(self, qtype, query, K=0):
        n = K if qtype == self.tb.QueryType.POINT else 3
        with self.lock:
            t = len(self.requests)
            self.requests.append((qtype, list(query), K))
            self.results[t] = (np.arange(n, dtype=np.uint64), np.zeros(n), 1234.4, np.array([5, 7, 2]))
        return t

    def poll_levels(self, ticket, wait_ms):
        with self.lock:
            return self.results.pop(ticket)


class FakeManager:
    def __init__(self, tb, root):
        self.tb = tb
        self.root = root
        self.server = FakeServer(tb)
        self.built = []

    def exists_on_disk(self, name):
        return os.path.exists(os.path.join(self.root, name, "metadata.bin"))

    def list_datasets(self):
        return sorted(e for e in os.listdir(self.root) if self.exists_on_disk(e))

    def get_or_load(self, name):
        if name != "ds":
            raise RuntimeError("Dataset index does not exist: " + name)
        return {"server": self.server,
                "info": {"D": 3, "intervals": 3, "meshSizes": [100000, 2000, 40, 2], "policy": []}}

    def build_and_save(self, name, path, force_cpu):
        self.built.append((name, path, force_cpu))


@pytest.fixture
def svc(tb, http, tmp_path):
    return http.QueryService(FakeManager(tb, str(tmp_path)))


def call(svc, route, obj):
    body = obj if isinstance(obj, bytes) else json.dumps(obj).encode()
    return getattr(svc, route)(body)


@pytest.mark.parametrize("obj,msg", [
    (b"{bad", "Invalid JSON: "),
    (b"[1, 2]", "Request body must be a JSON object"),
    ({"query_type": "KNN"}, "Field 'dataset_name' is required and must be a string"),
    ({"dataset_name": "a/b", "query_type": "KNN"}, "Invalid dataset_name. Allowed: [A-Za-z0-9._-], non-empty"),
    ({"dataset_name": "", "query_type": "KNN"}, "Invalid dataset_name. Allowed: [A-Za-z0-9._-], non-empty"),
    ({"dataset_name": "ds"}, "Field 'query_type' is required and must be 'KNN' or 'RANGE'"),
    ({"dataset_name": "ds", "query_type": "BOX"}, "query_type must be 'KNN' or 'RANGE'"),
    ({"dataset_name": "nope", "query_type": "knn"}, "Dataset index does not exist: nope"),
    ({"dataset_name": "ds", "query_type": "KNN"}, "Field 'query_point' is required for KNN query"),
    ({"dataset_name": "ds", "query_type": "KNN", "query_point": [1, "x", 3]}, "Field 'query_point' must be a numeric array"),
    ({"dataset_name": "ds", "query_type": "KNN", "query_point": [1, 2]}, "query_point dimension mismatch: expected 3"),
    ({"dataset_name": "ds", "query_type": "KNN", "query_point": [1, 2, 3], "k": 0}, "Field 'k' must be a positive integer"),
    ({"dataset_name": "ds", "query_type": "KNN", "query_point": [1, 2, 3], "k": 2.5}, "Field 'k' must be a positive integer"),
    ({"dataset_name": "ds", "query_type": "KNN", "query_point": [1, 2, 3], "k": True}, "Field 'k' must be a positive integer"),
    ({"dataset_name": "ds", "query_type": "RANGE", "lower_bound": [0, 0, 0]},
     "Fields 'upper_bound' and 'lower_bound' are required for RANGE query"),
    ({"dataset_name": "ds", "query_type": "RANGE", "lower_bound": [0, 0, 0], "upper_bound": 5},
     "upper_bound and lower_bound must be numeric arrays"),
    ({"dataset_name": "ds", "query_type": "RANGE", "lower_bound": [0, 0], "upper_bound": [1, 1, 1]},
     "Range bound dimension mismatch: expected 3"),
    ({"dataset_name": "ds", "query_type": "RANGE", "lower_bound": [0, 2, 0], "upper_bound": [1, 1, 1]},
     "Invalid range: lower_bound[1] > upper_bound[1]"),
])
def test_query_validation(svc, obj, msg):
    status, body = call(svc, "query", obj)
    assert status == 400 and body["success"] is False
    assert body["message"].startswith(msg), body["message"]
    assert not svc.manager.server.requests  # nothing reached the serving loop


def test_query_response_shape(svc, tb):
    status, body = call(svc, "query", {"dataset_name": "ds", "query_type": "knn", "query_point": [1, 2, 3.5],
                                       "k": 4.0})
    assert status == 200
    assert body["success"] is True and body["query_type"] == "KNN" and body["dataset_name"] == "ds"
    assert body["result"] == [0, 1, 2, 3] and body["result_count"] == 4
    # Per level, coarsest first: the size of the mesh the level expands into (meshSizes is finest first).
    assert body["level_original_sizes"] == [40, 2000, 100000] and body["level_pruned_sizes"] == [5, 7, 2]
    rt = body["query_runtime"]
    assert rt == {"query_time_us": 1234, "query_time_ms": 1.234, "total_time_us": 1234, "avg_time_us": 1234.0,
                  "query_count": 1}
    assert svc.manager.server.requests[-1] == (tb.QueryType.POINT, [1.0, 2.0, 3.5], 4)
    status, body = call(svc, "query", {"dataset_name": "ds", "query_type": "RANGE", "lower_bound": [0, 1, 2],
                                       "upper_bound": [3, 4, 5]})
    assert status == 200 and body["result_count"] == 3
    # The library takes a range request as lo[D] then hi[D].
    assert svc.manager.server.requests[-1] == (tb.QueryType.RANGE, [0.0, 1.0, 2.0, 3.0, 4.0, 5.0], 0)
    status, body = call(svc, "query", {"dataset_name": "ds", "query_type": "KNN", "query_point": [1, 2, 3]})
    assert status == 200 and body["result_count"] == 10  # k defaults to 10


def test_build_index_and_datasets(svc, tmp_path):
    assert svc.datasets() == (200, {"success": True, "datasets_count": 0, "datasets": []})
    status, body = call(svc, "build_index", {"dataset_name": "new"})
    assert status == 400 and body["message"] == \
        "Field 'dataset_path' is required and cannot be empty when index does not exist"
    status, body = call(svc, "build_index", {"dataset_name": "new", "dataset_path": str(tmp_path / "missing.txt")})
    assert status == 400 and body["message"] == "dataset_path does not exist or is not a file"
    data = tmp_path / "points.txt"
    data.write_text("2 2\n1 2\n3 4\n")
    status, body = call(svc, "build_index", {"dataset_name": "new", "dataset_path": str(data), "force_cpu": 1})
    assert status == 400 and body["message"] == "Field 'force_cpu' must be a boolean"
    status, body = call(svc, "build_index", {"dataset_name": "new", "dataset_path": str(data), "force_cpu": True})
    assert status == 200 and body["already_exists"] is False
    assert svc.manager.built == [("new", str(data), True)]
    os.makedirs(tmp_path / "old")
    (tmp_path / "old" / "metadata.bin").write_bytes(b"")
    status, body = call(svc, "build_index", {"dataset_name": "old"})
    assert status == 200 and body == {"success": True, "dataset_name": "old", "already_exists": True,
                                      "message": "Index already exists"}
    assert svc.datasets()[1]["datasets"] == ["old"]


def test_http_round_trip(svc, http):
    httpd = http.make_server(svc, "127.0.0.1", 0)
    t = threading.Thread(target=httpd.serve_forever, daemon=True)
    t.start()
    try:
        url = f"http://127.0.0.1:{httpd.server_address[1]}"

        def post(path, obj):
            req = urllib.request.Request(url + path, data=json.dumps(obj).encode(),
                                         headers={"Content-Type": "application/json"}, method="POST")
            try:
                with urllib.request.urlopen(req, timeout=10) as r:
                    return r.status, json.loads(r.read())
            except urllib.error.HTTPError as e:
                return e.code, json.loads(e.read())

        status, body = post("/query", {"dataset_name": "ds", "query_type": "KNN", "query_point": [0, 0, 0], "k": 2})
        assert status == 200 and body["result"] == [0, 1]
        status, body = post("/query", {"dataset_name": "ds", "query_type": "KNN"})
        assert status == 400 and body == {"success": False, "message": "Field 'query_point' is required for KNN query"}
        with urllib.request.urlopen(url + "/datasets", timeout=10) as r:
            assert json.loads(r.read()) == {"success": True, "datasets_count": 0, "datasets": []}
        status, body = post("/nowhere", {})
        assert status == 404
    finally:
        httpd.shutdown()
        httpd.server_close()


def test_index_manager_lists_cached_indexes(http, tmp_path):
    m = http.IndexManager(str(tmp_path / "cache"))
    os.makedirs(tmp_path / "cache" / "b")
    os.makedirs(tmp_path / "cache" / "a")
    os.makedirs(tmp_path / "cache" / "c")
    for n in ("a", "b"):
        (tmp_path / "cache" / n / "metadata.bin").write_bytes(b"")
    assert m.list_datasets() == ["a", "b"] and m.exists_on_disk("a") and not m.exists_on_disk("c")
    with pytest.raises(http.ApiError) as e:
        m.get_or_load("zzz")
    assert e.value.status == 400 and e.value.message == "Dataset index does not exist: zzz"


def test_burst_of_concurrent_clients(svc, http):
    """More simultaneous connections than the socket module's default listen backlog (5): every
    client is answered (the server's backlog is raised, so bursts queue instead of being reset)."""
    from concurrent.futures import ThreadPoolExecutor
    httpd = http.make_server(svc, "127.0.0.1", 0)
    t = threading.Thread(target=httpd.serve_forever, daemon=True)
    t.start()
    url = f"http://127.0.0.1:{httpd.server_address[1]}/query"
    body = json.dumps({"dataset_name": "ds", "query_type": "KNN", "query_point": [0, 0, 0], "k": 3}).encode()

    def one(_):
        req = urllib.request.Request(url, data=body, headers={"Content-Type": "application/json"}, method="POST")
        with urllib.request.urlopen(req, timeout=30) as r:
            return r.status, json.loads(r.read())["result"]

    try:
        with ThreadPoolExecutor(64) as ex:
            out = list(ex.map(one, range(256)))
        assert all(s == 200 and res == [0, 1, 2] for s, res in out)
    finally:
        httpd.shutdown()
        httpd.server_close()
