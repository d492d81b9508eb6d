"""HTTP front end over the serving loop (the reference's src/HTTPServer.cu:343-550).

Same routes, request fields, response fields and error messages as the reference:

  POST /build-index  {"dataset_name", "dataset_path", "force_cpu"} -> builds the index from a dataset
                     text file on the GPU and saves it under <index-cache>/<dataset_name>
  GET|POST /datasets -> {"success", "datasets_count", "datasets"}
  POST /query        {"dataset_name", "query_type": "KNN"|"RANGE", "query_point", "k"} or
                     {..., "lower_bound", "upper_bound"} -> {"success", "dataset_name", "query_type",
                     "result_count", "result", "memory_policy", "level_original_sizes",
                     "level_pruned_sizes", "query_runtime": {...}}
  failures           {"success": false, "message": "..."} with status 400 or 500

The difference is underneath: the reference answers one request at a time (its handlers race on a
shared QueryHandler), while every /query here is submitted to the dataset's serving loop, which
batches concurrent requests continuously on the GPU (range and KNN lanes). HTTP threads only parse,
submit, wait for their ticket and format. `query_time_us` is the request's latency inside the
serving loop (arrival to result).

Run: python http_server.py [-p 8080] [-i ./tempIndexCache] [-H 0.0.0.0] [--mode exact|ref-parity]
"""
import argparse
import importlib.util
import json
import math
import os
import re
import sys
import threading
from http.server import BaseHTTPRequestHandler, ThreadingHTTPServer

_DATASET_NAME = re.compile(r"^[A-Za-z0-9._-]+$")


def _package():
    """The library package this file belongs to (importable whether or not it is on sys.path)."""
    mod = sys.modules.get("tblaeq_b200")
    if mod is not None:
        return mod
    pkg_dir = os.path.dirname(os.path.abspath(__file__))
    spec = importlib.util.spec_from_file_location("tblaeq_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["tblaeq_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


class ApiError(Exception):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status
        self.message = message


def _is_number(v) -> bool:
    return isinstance(v, (int, float)) and not isinstance(v, bool)


def _numeric_vector(v):
    if not isinstance(v, list) or not all(_is_number(x) for x in v):
        return None
    return [float(x) for x in v]


class IndexManager:
    """Index cache directory of one index per dataset (<root>/<name>/metadata.bin), each loaded once
    and served by its own serving loop (IndexManager, src/HTTPServer.cu:236-302)."""

    def __init__(self, root: str, mode=None, max_batch: int = 4096):
        self.tb = _package()
        self.root = root
        self.mode = self.tb.Mode.EXACT if mode is None else mode
        self.max_batch = max_batch
        self._entries = {}
        self._lock = threading.Lock()
        os.makedirs(root, exist_ok=True)

    def exists_on_disk(self, name: str) -> bool:
        return os.path.exists(os.path.join(self.root, name, "metadata.bin"))

    def list_datasets(self):
        if not os.path.isdir(self.root):
            return []
        return sorted(e for e in os.listdir(self.root)
                      if os.path.isdir(os.path.join(self.root, e)) and self.exists_on_disk(e))

    def _serve(self, name, handler):
        handler.prepare_for_query()
        server = self.tb.Server(handler, max_batch=self.max_batch, mode=self.mode, levels=True)
        return {"handler": handler, "server": server, "info": handler.info()}

    def build_and_save(self, name: str, dataset_path: str, force_cpu: bool):
        handler, _ = self.tb.QueryHandler.build_from_file(dataset_path, force_cpu=force_cpu)
        handler.save_index(os.path.join(self.root, name))
        entry = self._serve(name, handler)
        with self._lock:
            old = self._entries.pop(name, None)
            self._entries[name] = entry
        if old:
            old["server"].stop()

    def get_or_load(self, name: str) -> dict:
        with self._lock:
            if name in self._entries:
                return self._entries[name]
            if not self.exists_on_disk(name):
                raise ApiError(400, "Dataset index does not exist: " + name)
            entry = self._serve(name, self.tb.QueryHandler(os.path.join(self.root, name)))
            self._entries[name] = entry
            return entry

    def close(self):
        with self._lock:
            entries, self._entries = list(self._entries.values()), {}
        for e in entries:
            e["server"].stop()
            e["handler"].close()


class QueryService:
    """The routes' request logic, independent of the HTTP transport. Each method returns
    (status, response object)."""

    def __init__(self, manager):
        self.manager = manager

    @staticmethod
    def error(status: int, message: str):
        return status, {"success": False, "message": message}

    @staticmethod
    def parse(body: bytes):
        try:
            obj = json.loads(body.decode("utf-8") if body else "")
        except (ValueError, UnicodeDecodeError) as e:
            raise ApiError(400, "Invalid JSON: " + str(e))
        if not isinstance(obj, dict):
            raise ApiError(400, "Request body must be a JSON object")
        return obj

    @staticmethod
    def dataset_name(obj) -> str:
        name = obj.get("dataset_name")
        if not isinstance(name, str):
            raise ApiError(400, "Field 'dataset_name' is required and must be a string")
        if not _DATASET_NAME.match(name):
            raise ApiError(400, "Invalid dataset_name. Allowed: [A-Za-z0-9._-], non-empty")
        return name

    def datasets(self):
        names = self.manager.list_datasets()
        return 200, {"success": True, "datasets_count": len(names), "datasets": names}

    def build_index(self, body: bytes):
        try:
            obj = self.parse(body)
            name = self.dataset_name(obj)
            if self.manager.exists_on_disk(name):
                return 200, {"success": True, "dataset_name": name, "already_exists": True,
                             "message": "Index already exists"}
            path = obj.get("dataset_path")
            if not isinstance(path, str) or not path:
                raise ApiError(400, "Field 'dataset_path' is required and cannot be empty when index does not exist")
            if not os.path.isfile(path):
                raise ApiError(400, "dataset_path does not exist or is not a file")
            force_cpu = obj.get("force_cpu", False)
            if not isinstance(force_cpu, bool):
                raise ApiError(400, "Field 'force_cpu' must be a boolean")
        except ApiError as e:
            return self.error(e.status, e.message)
        try:
            self.manager.build_and_save(name, path, force_cpu)
        except Exception as e:  # noqa: BLE001 - reported to the client like the reference
            return self.error(500, "Failed to build index: " + str(e))
        return 200, {"success": True, "dataset_name": name, "already_exists": False,
                     "message": "Index build and save succeeded"}

    def query(self, body: bytes):
        tb = _package()
        try:
            obj = self.parse(body)
            name = self.dataset_name(obj)
            qtype = obj.get("query_type")
            if not isinstance(qtype, str):
                raise ApiError(400, "Field 'query_type' is required and must be 'KNN' or 'RANGE'")
            qtype = qtype.upper()
            if qtype not in ("KNN", "RANGE"):
                raise ApiError(400, "query_type must be 'KNN' or 'RANGE'")
            try:
                entry = self.manager.get_or_load(name)
            except ApiError:
                raise
            except Exception as e:  # noqa: BLE001
                raise ApiError(400, str(e))
            info = entry["info"]
            dim = int(info["D"])
            if qtype == "KNN":
                if "query_point" not in obj:
                    raise ApiError(400, "Field 'query_point' is required for KNN query")
                point = _numeric_vector(obj["query_point"])
                if point is None:
                    raise ApiError(400, "Field 'query_point' must be a numeric array")
                if len(point) != dim:
                    raise ApiError(400, "query_point dimension mismatch: expected " + str(dim))
                k = obj.get("k", 10)
                if not _is_number(k) or k <= 0 or math.floor(k) != k:
                    raise ApiError(400, "Field 'k' must be a positive integer")
                request = (tb.QueryType.POINT, point, int(k))
            else:
                if "upper_bound" not in obj or "lower_bound" not in obj:
                    raise ApiError(400, "Fields 'upper_bound' and 'lower_bound' are required for RANGE query")
                hi = _numeric_vector(obj["upper_bound"])
                lo = _numeric_vector(obj["lower_bound"])
                if hi is None or lo is None:
                    raise ApiError(400, "upper_bound and lower_bound must be numeric arrays")
                if len(hi) != dim or len(lo) != dim:
                    raise ApiError(400, "Range bound dimension mismatch: expected " + str(dim))
                for i in range(dim):
                    if lo[i] > hi[i]:
                        raise ApiError(400, f"Invalid range: lower_bound[{i}] > upper_bound[{i}]")
                request = (tb.QueryType.RANGE, lo + hi, 0)
        except ApiError as e:
            return self.error(e.status, e.message)
        try:
            server = entry["server"]
            ticket = server.submit(*request)
            got = None
            while got is None:
                got = server.poll_levels(ticket, 1000)
            ids, _, latency_us, levels = got
        except Exception as e:  # noqa: BLE001
            return self.error(500, "Query execution failed: " + str(e))
        intervals = int(info["intervals"])
        original = [int(info["meshSizes"][intervals - (l + 1)]) for l in range(intervals)]
        policy = "-".join(p.name for p in (info.get("policy") or []))
        us = int(round(latency_us))
        return 200, {
            "success": True, "dataset_name": name, "query_type": qtype,
            "result_count": int(len(ids)), "result": [int(x) for x in ids],
            "memory_policy": policy,
            "level_original_sizes": original,
            "level_pruned_sizes": [int(x) for x in levels],
            "query_runtime": {"query_time_us": us, "query_time_ms": us / 1000.0, "total_time_us": us,
                              "avg_time_us": float(us), "query_count": 1},
        }


def make_server(service: QueryService, host: str = "0.0.0.0", port: int = 8080) -> ThreadingHTTPServer:
    """A threading HTTP server whose handlers call `service` (port 0: any free port)."""

    class Handler(BaseHTTPRequestHandler):
        protocol_version = "HTTP/1.1"

        def _send(self, status: int, obj):
            data = json.dumps(obj).encode("utf-8")
            self.send_response(status)
            self.send_header("Content-Type", "application/json")
            self.send_header("Content-Length", str(len(data)))
            self.end_headers()
            self.wfile.write(data)

        def _body(self) -> bytes:
            n = int(self.headers.get("Content-Length") or 0)
            return self.rfile.read(n) if n > 0 else b""

        def do_GET(self):  # noqa: N802
            if self.path == "/datasets":
                self._send(*service.datasets())
            else:
                self._send(*QueryService.error(404, "Not found"))

        def do_POST(self):  # noqa: N802
            body = self._body()
            if self.path == "/query":
                self._send(*service.query(body))
            elif self.path == "/datasets":
                self._send(*service.datasets())
            elif self.path == "/build-index":
                self._send(*service.build_index(body))
            else:
                self._send(*QueryService.error(404, "Not found"))

        def log_message(self, fmt, *args):  # keep request logging off the hot path
            pass

    class Server(ThreadingHTTPServer):
        daemon_threads = True
        request_queue_size = 1024  # listen backlog: bursts of clients queue instead of being reset

    return Server((host, port), Handler)


def main(argv=None):
    ap = argparse.ArgumentParser(description="T-BLAEQ B200 HTTP server")
    ap.add_argument("-p", "--port", type=int, default=8080, help="HTTP listen port (default: 8080)")
    ap.add_argument("-i", "--index-cache", default="./tempIndexCache", help="index cache directory")
    ap.add_argument("-H", "--host", default="0.0.0.0", help="HTTP listen host (default: 0.0.0.0)")
    ap.add_argument("--mode", choices=["exact", "ref-parity"], default="exact",
                    help="range results: exact (default) or the reference's candidate sets")
    ap.add_argument("--max-batch", type=int, default=4096, help="requests per GPU batch and lane")
    args = ap.parse_args(argv)
    if args.port <= 0 or args.port > 65535:
        raise SystemExit("Invalid port. Must be in range (0, 65535].")
    tb = _package()
    mode = tb.Mode.EXACT if args.mode == "exact" else tb.Mode.REF_PARITY
    manager = IndexManager(args.index_cache, mode=mode, max_batch=args.max_batch)
    httpd = make_server(QueryService(manager), args.host, args.port)
    print(f"T-BLAEQ HTTP server listening on {args.host}:{args.port}, index cache path: {args.index_cache}",
          flush=True)
    try:
        httpd.serve_forever()
    finally:
        httpd.server_close()
        manager.close()


if __name__ == "__main__":
    main()
