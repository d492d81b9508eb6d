"""T-BLAEQ on B200: Python facade over the C ABI (include/tblaeq.h, libtblaeq_b200.so).

The names and argument meanings follow the reference's C++ facade
(src/core/QueryHandler.cuh:50-247): ``QueryHandler`` builds or loads an index,
``prepare_for_query`` uploads it under a per-level memory policy, and queries run
through ``perform_single_range_query(upper, lower)`` (upper bound first, as in the
reference), ``perform_single_knn_query``, ``perform_query`` (reference query-file
format) or the batched ``query_batch`` of the B200 engine.

Every query runs in the CUDA library; there is no CPU path. Importing this module
on a machine without the built library raises ImportError, and calls that need a
GPU fail loudly with ``TblaeqError`` when no device is present.
"""
from __future__ import annotations

import ctypes
import enum
import os
import time
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# TBLAEQ_LIBRARY selects another build of the same library (e.g. a differently tuned one).
LIB_PATH = os.environ.get("TBLAEQ_LIBRARY") or os.path.join(_HERE, "libtblaeq_b200.so")
ABI_VERSION = 3  # TBLAEQ_ABI_VERSION of include/tblaeq.h this binding is written against
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "tblaeq.h")


class QueryType(enum.IntEnum):
    POINT = 0  # KNN
    RANGE = 1


class LevelPolicy(enum.IntEnum):
    L0 = 0
    L1 = 1
    L2 = 2
    L3 = 3


class Mode(enum.IntEnum):
    REF_PARITY = 0  # the reference's candidate sets
    EXACT = 1       # exact answers (subtree radii + exact final filter / top-K)


WANT_VALS = 1
WANT_LEVELS = 2
USE_GRAPH = 4

ERR_NAMES = {0: "OK", 1: "INVALID", 2: "IO", 3: "CUDA", 4: "OOM", 5: "OVERFLOW", 6: "TIMEOUT", 7: "STATE",
             8: "TYPE"}


class TblaeqError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{ERR_NAMES.get(code, code)}] {msg}")
        self.code = code


class _GenParams(ctypes.Structure):
    _fields_ = [("N", ctypes.c_uint64), ("D", ctypes.c_uint64), ("valMin", ctypes.c_double),
                ("valMax", ctypes.c_double), ("isInt", ctypes.c_int), ("height", ctypes.c_uint64),
                ("ratios", ctypes.POINTER(ctypes.c_uint64)), ("nRatios", ctypes.c_uint64), ("seed", ctypes.c_uint64),
                ("sigmaDivisor", ctypes.c_double)]


class _BuildConfig(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int), ("seed", ctypes.c_uint64), ("precision", ctypes.c_int),
                ("host_assembly", ctypes.c_int)]


class _BuildReport(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("k", ctypes.c_uint64), ("iters", ctypes.c_int),
                ("objective", ctypes.c_double), ("assign_seconds", ctypes.c_double),
                ("assemble_seconds", ctypes.c_double), ("seconds", ctypes.c_double)]


class KmeansPrecision(enum.IntEnum):
    TENSOR = 0   # tcgen05 tensor cores, TF32 hi/lo split operands, FP32 accumulation
    FP32 = 1     # CUDA cores, FP32
    FP64 = 2     # CUDA cores, FP64 (the precision reference)


class _Info(ctypes.Structure):
    _fields_ = [("D", ctypes.c_uint64), ("N", ctypes.c_uint64), ("height", ctypes.c_uint64),
                ("intervals", ctypes.c_uint64), ("meshSizes", ctypes.c_uint64 * 16),
                ("ratios", ctypes.c_uint64 * 16), ("hostBytes", ctypes.c_uint64),
                ("deviceBytes", ctypes.c_uint64), ("prepared", ctypes.c_int), ("policy", ctypes.c_int * 16)]


class Grid(ctypes.Structure):
    """tblaeq_grid: one query's grid at one level (device pointers)."""
    _fields_ = [("numRows", ctypes.c_uint64), ("dim", ctypes.c_uint64), ("nnz", ctypes.c_uint64),
                ("ids", ctypes.c_void_p), ("vals", ctypes.c_void_p)]


class _Batch(ctypes.Structure):
    _fields_ = [("qtype", ctypes.c_int), ("mode", ctypes.c_int), ("nq", ctypes.c_uint64),
                ("queries", ctypes.c_void_p), ("queriesOnDevice", ctypes.c_int), ("K", ctypes.c_uint64),
                ("flags", ctypes.c_uint), ("kPerQuery", ctypes.c_void_p)]


class _BatchResult(ctypes.Structure):
    _fields_ = [("nq", ctypes.c_uint64), ("total", ctypes.c_uint64), ("offsets", ctypes.c_void_p),
                ("ids", ctypes.c_void_p), ("vals", ctypes.c_void_p), ("dist2", ctypes.c_void_p),
                ("levelItems", ctypes.c_void_p)]


_lib = None


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `make -C t-blaeq_b200` (or __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    sig = {
        "tblaeq_last_error": ([], ctypes.c_char_p),
        "tblaeq_abi_version": ([], ctypes.c_int),
        "tblaeq_open": ([ctypes.c_char_p, P(vp)], ctypes.c_int),
        "tblaeq_generate": ([P(_GenParams), P(vp)], ctypes.c_int),
        "tblaeq_save": ([vp, ctypes.c_char_p], ctypes.c_int),
        "tblaeq_close": ([vp], None),
        "tblaeq_info": ([vp, P(_Info)], ctypes.c_int),
        "tblaeq_recommend": ([vp, ctypes.c_uint64, P(ctypes.c_int)], ctypes.c_int),
        "tblaeq_prepare": ([vp, P(ctypes.c_int), ctypes.c_uint64], ctypes.c_int),
        "tblaeq_level": ([vp, ctypes.c_uint64, P(Grid), ctypes.c_int, P(ctypes.c_double), P(ctypes.c_double),
                          P(ctypes.c_double), ctypes.c_uint64, P(Grid)], ctypes.c_int),
        "tblaeq_coarsest_grid": ([vp, P(Grid)], ctypes.c_int),
        "tblaeq_query_batch": ([vp, P(_Batch), P(_BatchResult)], ctypes.c_int),
        "tblaeq_query_batch_host": ([vp, P(_Batch), P(ctypes.c_uint64), P(ctypes.c_uint64), ctypes.c_uint64,
                                     P(ctypes.c_double), P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_host_array": ([vp, ctypes.c_int, ctypes.c_uint64, P(vp), P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_decode_points": ([vp, P(ctypes.c_uint64), ctypes.c_uint64, P(ctypes.c_double),
                                  P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_query_batch_async": ([vp, P(_Batch)], ctypes.c_int),
        "tblaeq_batch_wait": ([vp, P(_BatchResult)], ctypes.c_int),
        "tblaeq_graph_launches": ([vp, P(ctypes.c_uint64), P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_kernel_launches": ([], ctypes.c_uint64),
        "tblaeq_stream": ([vp], vp),
        "tblaeq_level_counts": ([vp, P(ctypes.c_uint64), P(ctypes.c_uint64), ctypes.c_int, P(ctypes.c_uint64)],
                                ctypes.c_int),
        "tblaeq_set_device": ([ctypes.c_int], ctypes.c_int),
        "tblaeq_set_timing": ([vp, ctypes.c_int], ctypes.c_int),
        "tblaeq_stage_times": ([vp, P(ctypes.c_float), ctypes.c_int], ctypes.c_int),
        "tblaeq_autotune": ([vp, P(_Batch), ctypes.c_int, P(ctypes.c_int), P(ctypes.c_float)], ctypes.c_int),
        "tblaeq_set_variants": ([vp, P(ctypes.c_int), ctypes.c_uint64], ctypes.c_int),
        "tblaeq_set_node_major": ([vp, ctypes.c_int], ctypes.c_int),
        "tblaeq_set_float_points": ([vp, ctypes.c_int], ctypes.c_int),
        "tblaeq_set_point_groups": ([vp, ctypes.c_int], ctypes.c_int),
        "tblaeq_group_counts": ([vp, P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_set_knn_chunk": ([vp, ctypes.c_uint64], ctypes.c_int),
        "tblaeq_set_knn_wave1": ([vp, ctypes.c_double], ctypes.c_int),
        "tblaeq_set_knn_refine": ([vp, ctypes.c_uint32], ctypes.c_int),
        "tblaeq_set_knn_refine_stages": ([vp, ctypes.c_uint32], ctypes.c_int),
        "tblaeq_knn_split_reason": ([vp, ctypes.c_char_p, ctypes.c_uint64], ctypes.c_int),
        "tblaeq_last_batch_runs": ([vp, P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_knn_batch_info": ([vp, P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_set_knn_probe": ([vp, ctypes.c_uint32, ctypes.c_int], ctypes.c_int),
        "tblaeq_set_launch_shapes": ([vp, P(ctypes.c_int), P(ctypes.c_int), ctypes.c_uint64], ctypes.c_int),
        "tblaeq_get_launch_shapes": ([vp, P(ctypes.c_int), P(ctypes.c_int), ctypes.c_uint64], ctypes.c_int),
        "tblaeq_tuning_key": ([vp, ctypes.c_int, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint64], ctypes.c_int),
        "tblaeq_tuning_store": ([ctypes.c_char_p, ctypes.c_char_p, P(ctypes.c_int), P(ctypes.c_int), ctypes.c_uint64],
                                ctypes.c_int),
        "tblaeq_tuning_lookup": ([ctypes.c_char_p, ctypes.c_char_p, P(ctypes.c_int), P(ctypes.c_int), ctypes.c_uint64,
                                  P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_set_two_wave": ([vp, ctypes.c_int], ctypes.c_int),
        "tblaeq_knn_counters": ([vp, P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_scorer_train": ([vp, P(ctypes.c_double), ctypes.c_uint64, vp, ctypes.c_uint64, ctypes.c_uint64,
                                 ctypes.c_int, ctypes.c_float, ctypes.c_uint64, P(ctypes.c_float)], ctypes.c_int),
        "tblaeq_scorer_enable": ([vp, ctypes.c_int], ctypes.c_int),
        "tblaeq_scorer_get_params": ([vp, P(ctypes.c_float), ctypes.c_uint64, P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_scorer_set_params": ([vp, P(ctypes.c_float), ctypes.c_uint64], ctypes.c_int),
        "tblaeq_scorer_loss_grad": ([vp, P(ctypes.c_float), P(ctypes.c_float), ctypes.c_uint64, P(ctypes.c_float),
                                     P(ctypes.c_float)], ctypes.c_int),
        "tblaeq_scorer_logits": ([vp, P(ctypes.c_float), ctypes.c_uint64, P(ctypes.c_float)], ctypes.c_int),
        "tblaeq_scorer_logits_tensor": ([vp, P(ctypes.c_float), ctypes.c_uint64, P(ctypes.c_float)], ctypes.c_int),
        "tblaeq_scorer_stats": ([vp, P(ctypes.c_uint64), P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_scorer_save": ([vp, ctypes.c_char_p], ctypes.c_int),
        "tblaeq_scorer_load": ([vp, ctypes.c_char_p], ctypes.c_int),
        "tblaeq_live_device_bytes": ([], ctypes.c_uint64),
        "tblaeq_debug_fail_alloc_after": ([ctypes.c_uint64], None),
        "tblaeq_debug_lookback_timeout": ([ctypes.c_uint64, ctypes.c_uint64], None),
        "tblaeq_debug_split_above": ([vp, ctypes.c_uint64], ctypes.c_int),
        "tblaeq_kmeans_build": ([P(ctypes.c_float), ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                 P(ctypes.c_uint64), P(_BuildConfig), P(vp), P(_BuildReport)], ctypes.c_int),
        "tblaeq_kmeans": ([P(ctypes.c_float), ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, P(_BuildConfig),
                           P(ctypes.c_float), P(ctypes.c_uint32), P(ctypes.c_double)], ctypes.c_int),
        "tblaeq_serve_start": ([vp, P(_ServeConfig), P(vp)], ctypes.c_int),
        "tblaeq_serve_submit": ([vp, ctypes.c_int, P(ctypes.c_double), ctypes.c_uint64, P(ctypes.c_uint64)],
                                ctypes.c_int),
        "tblaeq_serve_replay": ([vp, ctypes.c_uint64, P(ctypes.c_int), P(ctypes.c_double), P(ctypes.c_uint64),
                                 P(ctypes.c_uint32), P(ctypes.c_double), P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_serve_poll": ([vp, ctypes.c_uint64, ctypes.c_int, P(ctypes.c_uint64), P(ctypes.c_double),
                               ctypes.c_uint64, P(ctypes.c_uint64), P(ctypes.c_double)], ctypes.c_int),
        "tblaeq_serve_poll_levels": ([vp, ctypes.c_uint64, ctypes.c_int, P(ctypes.c_uint64), P(ctypes.c_double),
                                      ctypes.c_uint64, P(ctypes.c_uint64), P(ctypes.c_double), P(ctypes.c_uint32),
                                      ctypes.c_uint64, P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_serve_wait_idle": ([vp, ctypes.c_int], ctypes.c_int),
        "tblaeq_load_points_text": ([ctypes.c_char_p, P(ctypes.c_double), ctypes.c_uint64, P(ctypes.c_uint64),
                                     P(ctypes.c_uint64)], ctypes.c_int),
        "tblaeq_serve_stats": ([vp, ctypes.c_int, P(_ServeMetrics)], ctypes.c_int),
        "tblaeq_serve_stop": ([vp], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    if lib.tblaeq_abi_version() != ABI_VERSION:
        raise ImportError(f"{LIB_PATH} has C ABI version {lib.tblaeq_abi_version()}, this binding expects "
                          f"{ABI_VERSION}; rebuild it (make -C t-blaeq_b200)")
    _lib = lib
    return lib


class _ServeConfig(ctypes.Structure):
    _fields_ = [("max_batch", ctypes.c_uint32), ("memory_budget", ctypes.c_uint64), ("mode", ctypes.c_int),
                ("learned", ctypes.c_int), ("lanes", ctypes.c_int), ("levels", ctypes.c_int)]


class _ServeMetrics(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("batches", ctypes.c_uint64), ("max_batch", ctypes.c_uint64), ("mean_batch", ctypes.c_double),
                ("p50_us", ctypes.c_double), ("p99_us", ctypes.c_double), ("mean_us", ctypes.c_double),
                ("max_us", ctypes.c_double), ("span_s", ctypes.c_double)]


def lib():
    """The loaded C library (ctypes.CDLL)."""
    return _load()


def _check(code: int):
    if code != 0:
        raise TblaeqError(code, _load().tblaeq_last_error().decode())


def _k_args(K, nq):
    """(per-query uint32 array or None, uniform K) for a batch."""
    if np.isscalar(K):
        return None, int(K)
    kq = np.ascontiguousarray(np.asarray(K, dtype=np.uint32))
    if kq.shape != (nq,):
        raise ValueError("K must be an int or one value per query")
    return kq, 0


def _dptr(a: np.ndarray, ctype=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class DeviceArray:
    """A borrowed device buffer, exposed through __cuda_array_interface__ (torch.as_tensor works)."""

    def __init__(self, ptr: int, shape, typestr: str, owner=None):
        self.ptr = int(ptr or 0)
        self.shape = tuple(int(s) for s in shape)
        self.typestr = typestr
        self._owner = owner

    @property
    def __cuda_array_interface__(self):
        return {"shape": self.shape, "typestr": self.typestr, "data": (self.ptr, False), "version": 3}

    def torch(self):
        import torch
        if self.ptr == 0 or 0 in self.shape:
            dt = {"<u8": torch.uint64, "<f8": torch.float64, "<u4": torch.uint32}[self.typestr]
            return torch.empty(self.shape, dtype=dt, device="cuda")
        return torch.as_tensor(self, device="cuda")

    def numpy(self) -> np.ndarray:
        t = self.torch()
        return t.cpu().numpy()


@dataclass
class BatchResult:
    """Device-resident results of one batch (valid until the next batch call on the handle)."""
    nq: int
    total: int
    offsets: DeviceArray
    ids: DeviceArray
    vals: Optional[DeviceArray]
    dist2: Optional[DeviceArray]
    level_items: Optional[DeviceArray]


@dataclass
class QueryResult:
    """Mirror of the reference's QueryResult (src/core/QueryEngine.cuh:38-61)."""
    type: QueryType = QueryType.RANGE
    errorCode: int = 0
    totalTimeUs: float = 0.0
    queryCount: int = 0
    datasetName: str = ""
    queryParam: str = ""
    memoryPolicy: str = ""
    datasetSize: int = 0
    datasetDim: int = 0
    fineMeshSize: list = field(default_factory=list)
    levelOriginalSize: list = field(default_factory=list)
    levelFineMeshSize: list = field(default_factory=list)
    queryTimeUs: list = field(default_factory=list)
    fineMesh: list = field(default_factory=list)     # per query: np.ndarray of ids (saveFineMesh)
    fineMeshDist2: list = field(default_factory=list)  # per query, KNN exact mode


class QueryHandler:
    """B200 counterpart of the reference's QueryHandler (src/core/QueryHandler.cuh:50-247)."""

    def __init__(self, index_path: Optional[str] = None, load_from_index: bool = True, *, _handle=None):
        lib = _load()
        self._h = ctypes.c_void_p()
        if _handle is not None:
            self._h = _handle
        else:
            if index_path is None:
                raise ValueError("index_path is required (or use QueryHandler.generate)")
            if not load_from_index:
                raise ValueError("Use QueryHandler(datasetPath) to build a new index.")
            _check(lib.tblaeq_open(os.fsencode(index_path), ctypes.byref(self._h)))
        self.mode = Mode.REF_PARITY
        self.dataset_name = os.path.basename(os.path.normpath(index_path)) if index_path else "random"

    @classmethod
    def generate(cls, N: int, D: int, val_min: float = 1.0, val_max: float = 100.0, is_int: bool = False,
                 height: int = 4, ratios: Sequence[int] = (100, 50, 20), seed: int = 12345,
                 sigma_divisor: float = 3.0) -> "QueryHandler":
        """QueryHandler(N, D, valMin, valMax, isInt, height, ratios, seed, sigmaDivisor)."""
        lib = _load()
        r = np.ascontiguousarray(np.array(list(ratios), dtype=np.uint64))
        p = _GenParams(N, D, val_min, val_max, int(is_int), height, _dptr(r, ctypes.c_uint64), len(r), seed,
                       sigma_divisor)
        h = ctypes.c_void_p()
        _check(lib.tblaeq_generate(ctypes.byref(p), ctypes.byref(h)))
        obj = cls(_handle=h)
        obj.dataset_name = f"Gen{N}D{D}"
        return obj

    @classmethod
    def build_from_file(cls, dataset_path: str, force_cpu: bool = False, height: int = 4,
                        ratios: Sequence[int] = (100, 50, 20), iters: int = 20, seed: int = 1) -> tuple:
        """QueryHandler(forceUseCPU, datasetPath, height, ratios) (src/core/QueryHandler.cu:60-77):
        reads the dataset text file, truncates the plan like adjustBuildPlan and builds on the GPU.
        force_cpu (the reference's CPU k-means) selects the FP64 CUDA-core assignment here: the
        precision of a CPU build, still on the device. Returns (handler, per-level reports)."""
        X = load_dataset_file(dataset_path)
        height, ratios = adjust_build_plan(X.shape[0], height, ratios)
        prec = KmeansPrecision.FP64 if force_cpu else KmeansPrecision.TENSOR
        h, rep = cls.build(X, height=height, ratios=ratios, iters=iters, seed=seed, precision=prec)
        h.dataset_name = extract_dataset_name(dataset_path)
        return h, rep

    @classmethod
    def build(cls, points, height: int = 4, ratios: Sequence[int] = (100, 50, 20), iters: int = 20, seed: int = 1,
              precision: "KmeansPrecision" = None, host_assembly: int = 0) -> tuple:
        """IndexBuilder::build over FP32 points (N x D): GPU k-means per level, then the reference's
        P-tensor / map / radius assembly, on the device (host_assembly=1: on the host from
        downloaded labels and centroids, like the reference; 2: both, the device result checked
        byte for byte against the host's). Returns (handler, per-level reports, finest first)."""
        X = np.ascontiguousarray(np.asarray(points, dtype=np.float32))
        N, D = X.shape
        r = np.ascontiguousarray(np.array(list(ratios), dtype=np.uint64))
        prec = KmeansPrecision.TENSOR if precision is None else precision
        cfg = _BuildConfig(iters, seed, int(prec), int(host_assembly))
        reps = (_BuildReport * max(1, height - 1))()
        h = ctypes.c_void_p()
        _check(_load().tblaeq_kmeans_build(_dptr(X, ctypes.c_float), N, D, height, _dptr(r, ctypes.c_uint64),
                                           ctypes.byref(cfg), ctypes.byref(h), reps))
        obj = cls(_handle=h)
        obj.dataset_name = f"Kmeans{N}D{D}"
        return obj, [{f: getattr(x, f) for f, _ in _BuildReport._fields_} for x in reps[:height - 1]]

    # -- lifecycle -------------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _load().tblaeq_close(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def save_index(self, dir_path: str):
        _check(_load().tblaeq_save(self._h, os.fsencode(dir_path)))

    def info(self) -> dict:
        inf = _Info()
        _check(_load().tblaeq_info(self._h, ctypes.byref(inf)))
        h = inf.height
        return {"D": inf.D, "N": inf.N, "height": h, "intervals": inf.intervals,
                "meshSizes": list(inf.meshSizes[:h]), "ratios": list(inf.ratios[:inf.intervals]),
                "hostBytes": inf.hostBytes, "deviceBytes": inf.deviceBytes, "prepared": bool(inf.prepared),
                "policy": [LevelPolicy(p) for p in inf.policy[:inf.intervals]] if inf.prepared else None}

    def getSize(self) -> int:
        return self.info()["N"]

    def getDim(self) -> int:
        return self.info()["D"]

    def recommend(self, free_bytes: int = 0) -> list:
        n = self.info()["intervals"]
        out = (ctypes.c_int * n)()
        _check(_load().tblaeq_recommend(self._h, free_bytes, out))
        return [LevelPolicy(v) for v in out]

    def prepare_for_query(self, policy=None):
        """prepareForQuery(): None = recommendation, a LevelPolicy for every level, or a list."""
        lib = _load()
        if policy is None:
            _check(lib.tblaeq_prepare(self._h, None, 0))
            return
        n = self.info()["intervals"]
        levels = [policy] * n if isinstance(policy, (int, LevelPolicy)) else list(policy)
        arr = (ctypes.c_int * len(levels))(*[int(x) for x in levels])
        _check(lib.tblaeq_prepare(self._h, arr, len(levels)))

    prepareForQuery = prepare_for_query

    # -- host views ------------------------------------------------------------------------------
    def host_array(self, which: int, l: int = 0) -> np.ndarray:
        ptr = ctypes.c_void_p()
        cnt = ctypes.c_uint64()
        _check(_load().tblaeq_host_array(self._h, which, l, ctypes.byref(ptr), ctypes.byref(cnt)))
        ct = ctypes.c_double if which in (0, 2, 5) else ctypes.c_uint64
        if cnt.value == 0:
            return np.zeros(0, dtype=np.float64 if ct is ctypes.c_double else np.uint64)
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), (cnt.value,)).copy()

    def decode_points(self, positions) -> tuple:
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.uint64))
        D = self.info()["D"]
        out = np.empty((len(pos), D), np.float64)
        ids = np.empty(len(pos), np.uint64)
        _check(_load().tblaeq_decode_points(self._h, _dptr(pos, ctypes.c_uint64), len(pos), _dptr(out),
                                            _dptr(ids, ctypes.c_uint64)))
        return out, ids

    # -- per-level plugin (IQueryStrategy::runLevel) ----------------------------------------------
    def coarsest_grid(self) -> Grid:
        g = Grid()
        _check(_load().tblaeq_coarsest_grid(self._h, ctypes.byref(g)))
        return g

    def run_level(self, l: int, grid: Grid, qtype: QueryType, lo=None, hi=None, point=None, K: int = 0) -> Grid:
        out = Grid()
        D = int(grid.dim)
        def arr(v):
            if v is None:
                return None
            a = np.ascontiguousarray(np.asarray(v, dtype=np.float64))
            if a.shape != (D,):
                raise ValueError(f"expected {D} values")
            return a
        lo_a, hi_a, p_a = arr(lo), arr(hi), arr(point)
        _check(_load().tblaeq_level(self._h, l, ctypes.byref(grid), int(qtype),
                                    _dptr(lo_a) if lo_a is not None else None,
                                    _dptr(hi_a) if hi_a is not None else None,
                                    _dptr(p_a) if p_a is not None else None, K, ctypes.byref(out)))
        return out

    @staticmethod
    def grid_arrays(g: Grid):
        """(ids, vals) of a device grid as numpy copies."""
        ids = DeviceArray(g.ids, (g.nnz,), "<u8").numpy() if g.nnz else np.zeros(0, np.uint64)
        vals = DeviceArray(g.vals, (g.nnz, g.dim), "<f8").numpy() if g.nnz else np.zeros((0, g.dim))
        return ids, vals

    # -- batched engine --------------------------------------------------------------------------
    def query_batch(self, qtype: QueryType, queries, mode: Mode = Mode.EXACT, K=0,
                    flags: int = 0) -> BatchResult:
        """Batched traversal; `queries` is a numpy array (host) or a CUDA tensor (device).
        For KNN, K is an int or a per-query sequence."""
        on_dev = hasattr(queries, "__cuda_array_interface__")
        if on_dev:
            ptr = queries.__cuda_array_interface__["data"][0]
            nq = int(queries.shape[0])
            keep = queries
        else:
            keep = np.ascontiguousarray(np.asarray(queries, dtype=np.float64))
            ptr = keep.ctypes.data
            nq = keep.shape[0]
        kq, kval = _k_args(K, nq)
        b = _Batch(int(qtype), int(mode), nq, ptr, int(on_dev), kval, flags, kq.ctypes.data if kq is not None else None)
        r = _BatchResult()
        _check(_load().tblaeq_query_batch(self._h, ctypes.byref(b), ctypes.byref(r)))
        del keep, kq
        D = self.info()["D"]
        ivl = self.info()["intervals"]
        return BatchResult(
            nq=r.nq, total=r.total,
            offsets=DeviceArray(r.offsets, (r.nq + 1,), "<u8", self),
            ids=DeviceArray(r.ids, (r.total,), "<u8", self),
            vals=DeviceArray(r.vals, (r.total, D), "<f8", self) if r.vals else None,
            dist2=DeviceArray(r.dist2, (r.total,), "<f8", self) if r.dist2 else None,
            level_items=DeviceArray(r.levelItems, (ivl, r.nq), "<u4", self) if r.levelItems else None)

    def query_batch_async(self, qtype: QueryType, dqueries, mode: Mode = Mode.EXACT, K: int = 0, flags: int = 0):
        """Enqueue on the handle's stream without waiting (device queries; see tblaeq_query_batch_async)."""
        ptr = dqueries.__cuda_array_interface__["data"][0]
        b = _Batch(int(qtype), int(mode), int(dqueries.shape[0]), ptr, 1, K, flags, None)
        _check(_load().tblaeq_query_batch_async(self._h, ctypes.byref(b)))

    def batch_wait(self) -> int:
        r = _BatchResult()
        _check(_load().tblaeq_batch_wait(self._h, ctypes.byref(r)))
        return int(r.total)

    def level_counts(self):
        """(entries per frontier, children per frontier, results) of the last batch."""
        e = (ctypes.c_uint64 * 32)()
        it = (ctypes.c_uint64 * 32)()
        r = ctypes.c_uint64()
        n = _load().tblaeq_level_counts(self._h, e, it, 32, ctypes.byref(r))
        if n < 0:
            _check(-n)
        return list(e[:n]), list(it[:n]), int(r.value)

    def autotune(self, dqueries, mode: Mode = Mode.EXACT, reps: int = 5, flags: int = 0):
        """Search the launch shapes (variant x persistent-grid size) per level on this batch and keep
        the fastest; returns (variants, ms)."""
        H = self.info()["height"]
        ptr = dqueries.__cuda_array_interface__["data"][0]
        b = _Batch(int(QueryType.RANGE), int(mode), int(dqueries.shape[0]), ptr, 1, 0, flags, None)
        v = (ctypes.c_int * H)()
        ms = (ctypes.c_float * H)()
        _check(_load().tblaeq_autotune(self._h, ctypes.byref(b), reps, v, ms))
        return list(v), list(ms)

    def set_knn_probe(self, beam: int = 32, node_major_completion: bool = True):
        """Exact KNN: the probe's beam (0 = rank every surviving cluster) and the node-major
        completion after wave 1 (False: the query-major wave 2)."""
        _check(_load().tblaeq_set_knn_probe(self._h, beam, int(node_major_completion)))

    def set_node_major(self, on: bool = True):
        """Exact range batches: node-major inner levels (default) or entry-major."""
        _check(_load().tblaeq_set_node_major(self._h, int(on)))

    def set_float_points(self, on: bool = True):
        """Exact range batches: finest points decided from their float copies first (default;
        same results), or every point's FP64 test."""
        _check(_load().tblaeq_set_float_points(self._h, int(on)))

    def set_point_groups(self, on: bool = True):
        """Exact range batches with float points: test the finest clusters' point groups (at most
        32 points each, with their boxes) before their points (default; same results)."""
        _check(_load().tblaeq_set_point_groups(self._h, int(on)))

    def group_counts(self) -> dict:
        """The last range batch's point groups: tested, (query, group) pairs kept, points tested."""
        out = (ctypes.c_uint64 * 3)()
        _check(_load().tblaeq_group_counts(self._h, out))
        return {"groups": out[0], "kept": out[1], "points": out[2]}

    def launch_shapes(self):
        """(variants, grid percentages) per expand launch."""
        H = self.info()["height"]
        v, g = (ctypes.c_int * H)(), (ctypes.c_int * H)()
        _check(_load().tblaeq_get_launch_shapes(self._h, v, g, H))
        return list(v), list(g)

    def set_launch_shapes(self, variants, grid_percent):
        n = len(variants)
        _check(_load().tblaeq_set_launch_shapes(self._h, (ctypes.c_int * n)(*variants),
                                                (ctypes.c_int * n)(*grid_percent), n))

    def tuning_key(self, mode: Mode, nq: int) -> str:
        buf = ctypes.create_string_buffer(512)
        _check(_load().tblaeq_tuning_key(self._h, int(mode), nq, buf, 512))
        return buf.value.decode()

    def autotune_cached(self, dqueries, cache_path: str, mode: Mode = Mode.EXACT, reps: int = 5, flags: int = 0):
        """Launch shapes from the tuning cache when it holds this GPU, index shape, mode and batch
        size; otherwise autotune on this batch and store the result. Returns (variants, grid
        percentages, per-level ms or None when cached, "cache" | "tuned")."""
        key = self.tuning_key(mode, int(dqueries.shape[0]))
        hit = tuning_lookup(cache_path, key)
        if hit is not None:
            self.set_launch_shapes(*hit)
            return hit[0], hit[1], None, "cache"
        _, ms = self.autotune(dqueries, mode, reps, flags)
        v, g = self.launch_shapes()
        tuning_store(cache_path, key, v, g)
        return v, g, ms, "tuned"

    def set_variants(self, variants):
        arr = (ctypes.c_int * len(variants))(*[int(x) for x in variants])
        _check(_load().tblaeq_set_variants(self._h, arr, len(variants)))

    # -- exact KNN tuning and the learned scorer ----------------------------------------------------
    def set_two_wave(self, on: bool):
        _check(_load().tblaeq_set_two_wave(self._h, int(on)))

    def set_knn_chunk(self, max_queries: int = 0):
        """KNN batches: at most this many queries per traversal (0: automatic, halving on overflow
        or out-of-memory and starting later batches at the size that fitted)."""
        _check(_load().tblaeq_set_knn_chunk(self._h, int(max_queries)))

    def set_knn_wave1(self, scale: float = 16.0):
        """Two-wave KNN: wave 1 reads each query's ceil(scale * K / leaf) + 1 best-ranked clusters
        (2..32); larger tightens the bound the rest of the batch prunes with. Same results."""
        _check(_load().tblaeq_set_knn_wave1(self._h, float(scale)))

    def set_knn_refine(self, stride: int = 16):
        """Node-major KNN completion: a pass over every stride-th point of the listed clusters first
        tightens each query's bound (0 or 1: off). Same results."""
        _check(_load().tblaeq_set_knn_refine(self._h, int(stride)))

    def set_knn_refine_stages(self, stages: int = 2):
        """How many refinement stages run (1..4): strides stride^stages, ..., stride."""
        _check(_load().tblaeq_set_knn_refine_stages(self._h, int(stages)))

    def knn_batch_info(self) -> dict:
        """The last KNN batch: queries per traversal and traversals."""
        out = (ctypes.c_uint64 * 2)()
        _check(_load().tblaeq_knn_batch_info(self._h, out))
        buf = ctypes.create_string_buffer(512)
        _check(_load().tblaeq_knn_split_reason(self._h, buf, 512))
        runs = ctypes.c_uint64()
        _check(_load().tblaeq_last_batch_runs(self._h, ctypes.byref(runs)))
        return {"chunk": out[0], "traversals": out[1], "split_reason": buf.value.decode(), "runs": runs.value}

    def knn_counters(self) -> dict:
        out = (ctypes.c_uint64 * 5)()
        _check(_load().tblaeq_knn_counters(self._h, out))
        return {"frontier": out[0], "wave1": out[1], "wave2": out[2], "rows1": out[3], "rows2": out[4],
                "rows": out[3] + out[4]}

    def scorer_train(self, points, K=10, max_samples: int = 200000, epochs: int = 8, lr: float = 3e-3,
                     seed: int = 1) -> list:
        p = np.ascontiguousarray(np.asarray(points, dtype=np.float64))
        nq = p.shape[0]
        kq, kval = _k_args(K, nq)
        losses = (ctypes.c_float * epochs)()
        _check(_load().tblaeq_scorer_train(self._h, _dptr(p), nq, kq.ctypes.data if kq is not None else None, kval,
                                           max_samples, epochs, lr, seed, losses))
        return list(losses)

    def scorer_enable(self, on: bool = True):
        _check(_load().tblaeq_scorer_enable(self._h, int(on)))

    def scorer_params(self) -> np.ndarray:
        n = ctypes.c_uint64()
        _check(_load().tblaeq_scorer_get_params(self._h, None, 0, ctypes.byref(n)))
        out = np.empty(n.value, np.float32)
        _check(_load().tblaeq_scorer_get_params(self._h, _dptr(out, ctypes.c_float), n.value, ctypes.byref(n)))
        return out

    def scorer_set_params(self, params):
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float32))
        _check(_load().tblaeq_scorer_set_params(self._h, _dptr(p, ctypes.c_float), p.size))

    def scorer_loss_grad(self, X, y):
        X = np.ascontiguousarray(np.asarray(X, dtype=np.float32))
        y = np.ascontiguousarray(np.asarray(y, dtype=np.float32))
        grad = np.empty(self.scorer_params().size, np.float32)
        loss = ctypes.c_float()
        _check(_load().tblaeq_scorer_loss_grad(self._h, _dptr(X, ctypes.c_float), _dptr(y, ctypes.c_float), X.shape[0],
                                               _dptr(grad, ctypes.c_float), ctypes.byref(loss)))
        return float(loss.value), grad

    def scorer_logits(self, X, tensor: bool = False) -> np.ndarray:
        """Logits of feature rows X (n x in). tensor=True runs the tensor-core kernel that scores KNN
        frontiers (BF16 inputs and hidden layer, FP32 accumulation)."""
        X = np.ascontiguousarray(np.asarray(X, dtype=np.float32))
        z = np.empty(X.shape[0], np.float32)
        fn = _load().tblaeq_scorer_logits_tensor if tensor else _load().tblaeq_scorer_logits
        _check(fn(self._h, _dptr(X, ctypes.c_float), X.shape[0], _dptr(z, ctypes.c_float)))
        return z

    def scorer_save(self, path: str):
        _check(_load().tblaeq_scorer_save(self._h, os.fsencode(path)))

    def scorer_load(self, path: str):
        """Loads a saved scorer (same index shape) and enables it."""
        _check(_load().tblaeq_scorer_load(self._h, os.fsencode(path)))

    def scorer_stats(self) -> dict:
        s, p = ctypes.c_uint64(), ctypes.c_uint64()
        _check(_load().tblaeq_scorer_stats(self._h, ctypes.byref(s), ctypes.byref(p)))
        return {"samples": s.value, "positives": p.value}

    def stream_handle(self) -> int:
        return _load().tblaeq_stream(self._h) or 0

    def set_timing(self, on: bool = True):
        _check(_load().tblaeq_set_timing(self._h, int(on)))

    def graph_launches(self) -> dict:
        """Kernel nodes and all nodes of the CUDA graph that USE_GRAPH batches replay (zeros when none
        is held)."""
        k, n = ctypes.c_uint64(), ctypes.c_uint64()
        _check(_load().tblaeq_graph_launches(self._h, ctypes.byref(k), ctypes.byref(n)))
        return {"kernels": k.value, "nodes": n.value}

    def stage_times(self) -> list:
        buf = (ctypes.c_float * 64)()
        n = _load().tblaeq_stage_times(self._h, buf, 64)
        if n < 0:
            raise TblaeqError(7, "stage times unavailable: " + _load().tblaeq_last_error().decode())
        return list(buf[:n])

    def query_batch_host(self, qtype: QueryType, queries: np.ndarray, mode: Mode = Mode.EXACT, K: int = 0,
                         ids_cap: Optional[int] = None):
        """Host-buffer batch: returns (offsets, ids, dist2 or None)."""
        q = np.ascontiguousarray(np.asarray(queries, dtype=np.float64))
        nq = q.shape[0]
        cap = ids_cap if ids_cap is not None else max(1024, nq * 64)
        while True:
            offs = np.empty(nq + 1, np.uint64)
            ids = np.empty(cap, np.uint64)
            d2 = np.empty(cap, np.float64) if qtype == QueryType.POINT else None
            total = ctypes.c_uint64()
            kq, kval = _k_args(K, nq)
            b = _Batch(int(qtype), int(mode), nq, q.ctypes.data, 0, kval, 0,
                       kq.ctypes.data if kq is not None else None)
            code = _load().tblaeq_query_batch_host(self._h, ctypes.byref(b), _dptr(offs, ctypes.c_uint64),
                                                   _dptr(ids, ctypes.c_uint64), cap,
                                                   _dptr(d2) if d2 is not None else None, ctypes.byref(total))
            if code == 5 and ids_cap is None and total.value > cap:
                cap = int(total.value)
                continue
            _check(code)
            n = int(total.value)
            return offs, ids[:n], (d2[:n] if d2 is not None else None)

    # -- reference-style query APIs ----------------------------------------------------------------
    def _run_plain(self, qtype: QueryType, rows: np.ndarray, K: int, save: bool) -> QueryResult:
        info = self.info()
        res = QueryResult(type=qtype, datasetName=self.dataset_name, datasetSize=info["N"], datasetDim=info["D"])
        res.queryParam = f"K={K}" if qtype == QueryType.POINT else res.queryParam
        res.levelOriginalSize = [info["meshSizes"][info["intervals"] - (l + 1)] for l in range(info["intervals"])]
        pol = info["policy"] or []
        res.memoryPolicy = "-".join(p.name for p in pol)
        for i in range(rows.shape[0]):
            t0 = time.perf_counter()
            offs, ids, d2 = self.query_batch_host(qtype, rows[i:i + 1], self.mode, K)
            us = (time.perf_counter() - t0) * 1e6
            res.queryTimeUs.append(us)
            res.fineMeshSize.append(int(offs[1] - offs[0]))
            if save:
                res.fineMesh.append(ids)
                if d2 is not None:
                    res.fineMeshDist2.append(d2)
        times = sorted(res.queryTimeUs)
        cnt = len(times)
        total = sum(times)
        if cnt > 2:  # the reference drops the fastest and slowest query (QueryEngine.cu:216-220)
            total -= times[0] + times[-1]
            cnt -= 2
        res.totalTimeUs = total
        res.queryCount = cnt
        return res

    def perform_single_range_query(self, query_upper_bound, query_lower_bound,
                                   save_fine_mesh: bool = False) -> QueryResult:
        """performSingleRangeQuery(upper, lower, saveFineMesh): note the upper-bound-first order."""
        lo = np.asarray(query_lower_bound, dtype=np.float64)
        hi = np.asarray(query_upper_bound, dtype=np.float64)
        r = self._run_plain(QueryType.RANGE, np.concatenate([lo, hi])[None, :], 0, save_fine_mesh)
        r.queryParam = "single-range-query"
        return r

    performSingleRangeQuery = perform_single_range_query

    def perform_single_knn_query(self, query_point, k: int, save_fine_mesh: bool = False) -> QueryResult:
        p = np.asarray(query_point, dtype=np.float64)[None, :]
        return self._run_plain(QueryType.POINT, p, k, save_fine_mesh)

    performSingleKNNQuery = perform_single_knn_query

    def perform_query(self, query_path: str, q_type: QueryType, save_fine_mesh: bool = False,
                      max_query_count: int = 2 ** 31 - 1, K: int = 0) -> QueryResult:
        rows, ftype = load_query_file(query_path, q_type)
        if ftype != q_type:
            return QueryResult(errorCode=1)
        rows = rows[:max_query_count]
        return self._run_plain(q_type, rows, K, save_fine_mesh)

    performQuery = perform_query


# ---- reference query-file format (src/Data_Structures/File.cu:139-216) ---------------------------
class Server:
    """Serving loop over a prepared handle: continuous batching of range and KNN requests
    (the batched replacement for the reference's one-query-at-a-time request loop,
    src/HTTPServer.cu:414-550). Results are exact; KNN results carry squared distances."""

    def __init__(self, handler: "QueryHandler", max_batch: int = 4096, memory_budget: int = 0,
                 mode: Mode = Mode.EXACT, learned: bool = True, lanes: int = 2, levels: bool = False):
        """levels=True records every request's generated-children count per level (returned by
        poll_levels), at the cost of per-query counters in every expand launch."""
        self._owner = handler
        self._D = handler.info()["D"]
        self._intervals = handler.info()["intervals"]
        cfg = _ServeConfig(max_batch, memory_budget, int(mode), int(learned), lanes, int(levels))
        s = ctypes.c_void_p()
        _check(_load().tblaeq_serve_start(handler._h, ctypes.byref(cfg), ctypes.byref(s)))
        self._s = s

    def submit(self, qtype: QueryType, query, K: int = 0) -> int:
        q = np.ascontiguousarray(np.asarray(query, dtype=np.float64).ravel())
        t = ctypes.c_uint64()
        _check(_load().tblaeq_serve_submit(self._s, int(qtype), _dptr(q), int(K), ctypes.byref(t)))
        return t.value

    def replay(self, qtypes, queries, K, arrival_us) -> np.ndarray:
        """Submit request i at arrival_us[i] µs from now; queries[i] is a row (2D values for range, D
        for KNN, any padding after them ignored). Returns the tickets."""
        qt = np.ascontiguousarray(np.asarray(qtypes, dtype=np.int32))
        Q = np.ascontiguousarray(np.asarray(queries, dtype=np.float64))
        n = len(qt)
        offs = (np.arange(n, dtype=np.uint64) * np.uint64(Q.shape[1])).astype(np.uint64)
        k = np.ascontiguousarray(np.asarray(K, dtype=np.uint32))
        at = np.ascontiguousarray(np.asarray(arrival_us, dtype=np.float64))
        tickets = np.empty(n, np.uint64)
        _check(_load().tblaeq_serve_replay(self._s, n, qt.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dptr(Q),
                                           _dptr(offs, ctypes.c_uint64), k.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                           _dptr(at), _dptr(tickets, ctypes.c_uint64)))
        return tickets

    def poll(self, ticket: int, wait_ms: int = 10000):
        """(ids, dist2 or None, latency_us) once done; None if not done within wait_ms."""
        r = self.poll_levels(ticket, wait_ms)
        return None if r is None else r[:3]

    def poll_levels(self, ticket: int, wait_ms: int = 10000):
        """(ids, dist2, latency_us, per-level child counts) once done (the counts are empty unless
        the server was started with levels=True); None if not done within wait_ms."""
        lib = _load()
        cap = 1024
        while True:
            ids = np.empty(cap, np.uint64)
            d2 = np.empty(cap, np.float64)
            lv = np.zeros(max(1, self._intervals), np.uint32)
            n, lat, nl = ctypes.c_uint64(), ctypes.c_double(), ctypes.c_uint64()
            code = lib.tblaeq_serve_poll_levels(self._s, int(ticket), wait_ms, _dptr(ids, ctypes.c_uint64), _dptr(d2),
                                                cap, ctypes.byref(n), ctypes.byref(lat),
                                                lv.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), len(lv),
                                                ctypes.byref(nl))
            if code == 6:
                return None
            if code == 5:
                cap = int(n.value)
                continue
            _check(code)
            k = int(n.value)
            return ids[:k], d2[:k], lat.value, lv[:min(int(nl.value), len(lv))].astype(np.int64)

    def wait_idle(self, wait_ms: int = 60000) -> bool:
        code = _load().tblaeq_serve_wait_idle(self._s, wait_ms)
        if code == 6:
            return False
        _check(code)
        return True

    def stats(self, reset: bool = False) -> dict:
        m = _ServeMetrics()
        _check(_load().tblaeq_serve_stats(self._s, int(reset), ctypes.byref(m)))
        return {f: getattr(m, f) for f, _ in _ServeMetrics._fields_}

    def stop(self):
        if self._s:
            _check(_load().tblaeq_serve_stop(self._s))
            self._s = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


def kmeans(points, k: int, iters: int = 20, seed: int = 1, precision: KmeansPrecision = KmeansPrecision.TENSOR):
    """One level of GPU k-means: (centroids k x D FP32, labels, FP64 objective per iteration)."""
    X = np.ascontiguousarray(np.asarray(points, dtype=np.float32))
    n, D = X.shape
    C = np.empty((k, D), np.float32)
    L = np.empty(n, np.uint32)
    obj = np.empty(iters, np.float64)
    cfg = _BuildConfig(iters, seed, int(precision), 0)
    _check(_load().tblaeq_kmeans(_dptr(X, ctypes.c_float), n, D, k, ctypes.byref(cfg), _dptr(C, ctypes.c_float),
                                 L.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), _dptr(obj)))
    return C, L, obj


def save_query_file(path: str, q_type: QueryType, rows: np.ndarray, D: int):
    """Header 'n D', then one row per query: 2D values (lo then hi) for RANGE, D values for POINT."""
    rows = np.asarray(rows, dtype=np.float64)
    with open(path, "w") as f:
        f.write(f"{rows.shape[0]} {D}\n")
        for r in rows:
            f.write(" ".join("%.17g" % v for v in r) + "\n")


def load_dataset_file(path: str) -> np.ndarray:
    """Dataset text file (loadFromFile, src/Data_Structures/File.cu:8-50): header "N D", then N rows
    of D values; returns an (N, D) float64 array. Raises TblaeqError (TBLAEQ_ERR_IO) with the
    reference's message on a malformed file."""
    lib = _load()
    n, d = ctypes.c_uint64(), ctypes.c_uint64()
    _check(lib.tblaeq_load_points_text(os.fsencode(path), None, 0, ctypes.byref(n), ctypes.byref(d)))
    X = np.empty((n.value, d.value), np.float64)
    _check(lib.tblaeq_load_points_text(os.fsencode(path), _dptr(X), X.size, ctypes.byref(n), ctypes.byref(d)))
    return X


def adjust_build_plan(N: int, height: int, ratios: Sequence[int]):
    """adjustBuildPlan (src/core/QueryHandler.cu:23-45): drops the levels above the first one that
    would hold a single centroid. Returns (height, ratios)."""
    if height < 2:
        raise ValueError("QueryHandler: height must be >= 2")
    ratios = [int(r) for r in ratios]
    if len(ratios) != height - 1:
        raise ValueError("QueryHandler: ratios size must equal height - 1")
    n, keep = int(N), len(ratios)
    for i, r in enumerate(ratios):
        c = 1 if r == 0 or n // r == 0 else n // r
        if c == 1:
            keep = i + 1
            break
        n = c
    return keep + 1, ratios[:keep]


def extract_dataset_name(path: str) -> str:
    """extractDatasetName (src/utils/Utils.cu:6-10): the file name up to its first '_'."""
    base = path[path.rfind("/") + 1:]
    cut = base.find("_")
    return base if cut < 0 else base[:cut]


def load_query_file(path: str, q_type: QueryType):
    with open(path) as f:
        header = f.readline().split()
        if len(header) < 2:
            raise ValueError("loadQueryFromFile: invalid header")
        n, D = int(header[0]), int(header[1])
        if n <= 0 or D <= 0:
            raise ValueError("loadQueryFromFile: invalid header")
        cols = 2 * D if q_type == QueryType.RANGE else D
        rows = np.empty((n, cols), np.float64)
        for i in range(n):
            line = f.readline()
            vals = line.split()
            if len(vals) < cols:
                raise ValueError(f"loadQueryFromFile: expected {cols} values at row {i + 1}")
            rows[i] = [float(v) for v in vals[:cols]]
    return rows, q_type


def tuning_store(path: str, key: str, variants, grid_percent):
    """Adds or replaces `key`'s launch shapes in the tuning-cache file at `path`."""
    n = len(variants)
    _check(_load().tblaeq_tuning_store(path.encode(), key.encode(), (ctypes.c_int * n)(*variants),
                                       (ctypes.c_int * n)(*grid_percent), n))


def tuning_lookup(path: str, key: str):
    """(variants, grid percentages) stored for `key`, or None."""
    cap = 64
    v, g, n = (ctypes.c_int * cap)(), (ctypes.c_int * cap)(), ctypes.c_uint64()
    _check(_load().tblaeq_tuning_lookup(path.encode(), key.encode(), v, g, cap, ctypes.byref(n)))
    return None if n.value == 0 else (list(v[:n.value]), list(g[:n.value]))


def set_device(device: int):
    """cudaSetDevice for this library's CUDA runtime on the calling thread (before prepare)."""
    _check(_load().tblaeq_set_device(int(device)))


def kernel_launches() -> int:
    """Kernel launches this library has issued in the process so far (captures count once, graph
    replays not at all)."""
    return int(_load().tblaeq_kernel_launches())
