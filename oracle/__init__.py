"""Test infrastructure: Python access to the CPU oracle (oracle/liboracle.so).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this package,
and only as the checker or the timed CPU baseline; the product path never does.

``load_index`` is an independent numpy restatement of the reference's index reader
(src/core/IndexSerializer.cu:34-235), so the oracle never shares a loader with the product.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

RANGE = 0
KNN = 1


def build() -> str:
    """Compile liboracle.so (g++ only) if missing or stale."""
    src = [os.path.join(_HERE, f) for f in ("oracle.cpp", "oracle.h")]
    if not os.path.exists(_LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(_LIB_PATH) for s in src):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _LIB_PATH


class _OracleIndex(ctypes.Structure):
    _fields_ = [
        ("D", ctypes.c_uint64),
        ("height", ctypes.c_uint64),
        ("intervals", ctypes.c_uint64),
        ("meshCount", ctypes.POINTER(ctypes.c_uint64)),
        ("colRes", ctypes.POINTER(ctypes.POINTER(ctypes.c_uint64))),
        ("pvals", ctypes.POINTER(ctypes.POINTER(ctypes.c_double))),
        ("radius", ctypes.POINTER(ctypes.POINTER(ctypes.c_double))),
        ("maps", ctypes.POINTER(ctypes.POINTER(ctypes.c_uint64))),
        ("coarseIds", ctypes.POINTER(ctypes.c_uint64)),
        ("coarseVals", ctypes.POINTER(ctypes.c_double)),
    ]


class _OracleResults(ctypes.Structure):
    _fields_ = [
        ("nq", ctypes.c_uint64),
        ("intervals", ctypes.c_uint64),
        ("offsets", ctypes.POINTER(ctypes.c_uint64)),
        ("ids", ctypes.POINTER(ctypes.c_uint64)),
        ("dist2", ctypes.POINTER(ctypes.c_double)),
        ("levelSizes", ctypes.POINTER(ctypes.c_uint64)),
    ]


def _load():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        P = ctypes.POINTER
        _lib.oracle_ref_query.argtypes = [P(_OracleIndex), ctypes.c_int, ctypes.c_uint64, P(ctypes.c_double),
                                          ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int, P(_OracleResults)]
        _lib.oracle_exact_query.argtypes = [P(_OracleIndex), P(P(ctypes.c_double)), P(P(ctypes.c_uint64)),
                                            ctypes.c_int, ctypes.c_uint64, P(ctypes.c_double), ctypes.c_uint64,
                                            ctypes.c_int, P(_OracleResults)]
        _lib.oracle_decode_mesh.argtypes = [P(_OracleIndex), ctypes.c_uint64, P(ctypes.c_double)]
        _lib.oracle_subtree.argtypes = [P(_OracleIndex), P(P(ctypes.c_double)), P(P(ctypes.c_uint64))]
        _lib.oracle_brute_query.argtypes = [P(ctypes.c_double), P(ctypes.c_uint64), ctypes.c_uint64, ctypes.c_uint64,
                                            ctypes.c_int, ctypes.c_uint64, P(ctypes.c_double), ctypes.c_uint64,
                                            ctypes.c_int, P(_OracleResults)]
        _lib.oracle_free_results.argtypes = [P(_OracleResults)]
        _lib.oracle_sqrt_rd.argtypes = [ctypes.c_double]
        _lib.oracle_sqrt_rd.restype = ctypes.c_double
    return _lib


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


@dataclass
class OracleIndex:
    """An index in the reference's host layout, as numpy arrays (interval l = 0 is coarsest)."""

    D: int
    N: int
    height: int
    ratios: list
    mesh_sizes: list          # finest -> coarsest, like the reference metadata
    col_res: list             # [intervals] uint64
    nnz_per_col: list         # [intervals] uint64
    row_ids: list             # [intervals] uint64
    pvals: list               # [intervals] float64 (rows, D)
    radius: list              # [intervals] float64 by coarse original id
    maps: list                # [height] uint64, maps[0] is None
    coarse_ids: np.ndarray
    coarse_vals: np.ndarray
    _keep: list = field(default_factory=list, repr=False)

    @property
    def intervals(self) -> int:
        return self.height - 1

    def mesh_count(self, m: int) -> int:
        return int(self.mesh_sizes[self.intervals - m])

    def c_struct(self) -> _OracleIndex:
        L = self.intervals
        mc = np.array([self.mesh_count(m) for m in range(self.height)], dtype=np.uint64)
        colres = (ctypes.POINTER(ctypes.c_uint64) * L)(*[_ptr(a, ctypes.c_uint64) for a in self.col_res])
        pv = (ctypes.POINTER(ctypes.c_double) * L)(*[_ptr(a, ctypes.c_double) for a in self.pvals])
        rad = (ctypes.POINTER(ctypes.c_double) * L)(*[_ptr(a, ctypes.c_double) for a in self.radius])
        null_u64 = ctypes.POINTER(ctypes.c_uint64)()
        mp = (ctypes.POINTER(ctypes.c_uint64) * self.height)(
            *[null_u64 if a is None else _ptr(a, ctypes.c_uint64) for a in self.maps])
        s = _OracleIndex(self.D, self.height, L, _ptr(mc, ctypes.c_uint64), colres, pv, rad, mp,
                         _ptr(self.coarse_ids, ctypes.c_uint64), _ptr(self.coarse_vals, ctypes.c_double))
        self._keep = [mc, colres, pv, rad, mp]
        return s


def load_index(path: str) -> OracleIndex:
    """Read an index directory written by the reference (or by the B200 build) with numpy."""
    def rd(name):
        with open(os.path.join(path, name), "rb") as f:
            return f.read()

    meta = rd("metadata.bin")
    D, N, height, intervals = np.frombuffer(meta, np.uint64, 4, 0)
    off = 33
    ratios = np.frombuffer(meta, np.uint64, int(intervals), off).tolist()
    off += 8 * int(intervals)
    msz = int(np.frombuffer(meta, np.uint64, 1, off)[0])
    mesh_sizes = np.frombuffer(meta, np.uint64, msz, off + 8).tolist()
    col_res, nnz_per_col, row_ids, pvals, radius = [], [], [], [], []
    for l in range(int(intervals)):
        b = rd(f"P_Tensor_{l}.bin")
        d, rows, cols, nnz = (int(x) for x in np.frombuffer(b, np.uint64, 4, 0))
        o = 33
        row_ids.append(np.frombuffer(b, np.uint64, nnz, o).copy()); o += 8 * nnz
        nnz_per_col.append(np.frombuffer(b, np.uint64, cols, o).copy()); o += 8 * cols
        col_res.append(np.frombuffer(b, np.uint64, cols + 1, o).copy()); o += 8 * (cols + 1)
        pvals.append(np.frombuffer(b, np.float64, nnz * d, o).reshape(nnz, d).copy())
        rb = rd(f"MaxRadius_{l}.bin")
        cnt = int(np.frombuffer(rb, np.uint64, 1, 0)[0])
        radius.append(np.frombuffer(rb, np.float64, cnt, 8).copy())
    maps = [None]
    for m in range(1, int(height)):
        mb = rd(f"Map_{m}.bin")
        n = int(np.frombuffer(mb, np.uint64, 1, 0)[0])
        maps.append(np.frombuffer(mb, np.uint64, n, 8).copy())
    cb = rd("Coreast_Mesh.bin")
    rows, dim, nnz = (int(x) for x in np.frombuffer(cb, np.uint64, 3, 0))
    cids = np.frombuffer(cb, np.uint64, nnz, 25).copy()
    cvals = np.frombuffer(cb, np.float64, nnz * dim, 25 + 8 * nnz).reshape(nnz, dim).copy()
    return OracleIndex(int(D), int(N), int(height), ratios, mesh_sizes, col_res, nnz_per_col, row_ids, pvals,
                       radius, maps, cids, cvals)


@dataclass
class Results:
    offsets: np.ndarray
    ids: np.ndarray
    dist2: np.ndarray | None
    level_sizes: np.ndarray | None

    def query(self, q: int) -> np.ndarray:
        return self.ids[self.offsets[q]:self.offsets[q + 1]]


def _take(res: _OracleResults, lib) -> Results:
    nq = res.nq
    offs = np.ctypeslib.as_array(res.offsets, (nq + 1,)).copy()
    total = int(offs[-1])
    ids = np.ctypeslib.as_array(res.ids, (max(total, 1),))[:total].copy()
    d2 = None
    if res.dist2:
        d2 = np.ctypeslib.as_array(res.dist2, (max(total, 1),))[:total].copy()
    lv = None
    if res.intervals:
        lv = np.ctypeslib.as_array(res.levelSizes, (nq * res.intervals,)).reshape(nq, res.intervals).copy()
    lib.oracle_free_results(ctypes.byref(res))
    return Results(offs, ids, d2, lv)


def ref_query(idx: OracleIndex, qtype: int, queries: np.ndarray, K: int = 0, use_fma: bool = True,
              sorted_ids: bool = True, threads: int = 0) -> Results:
    """Reference traversal (ref-parity candidate sets)."""
    lib = _load()
    q = np.ascontiguousarray(queries, dtype=np.float64)
    nq = q.shape[0]
    res = _OracleResults()
    lib.oracle_ref_query(ctypes.byref(idx.c_struct()), qtype, nq, _ptr(q, ctypes.c_double), K, int(use_fma),
                         int(sorted_ids), threads, ctypes.byref(res))
    return _take(res, lib)


def subtree(idx: OracleIndex):
    """Subtree radii (with the conservative slack) and leaf counts per mesh, by original id."""
    lib = _load()
    L = idx.intervals
    R = [np.zeros(idx.mesh_count(m), np.float64) for m in range(L)]
    C = [np.zeros(idx.mesh_count(m), np.uint64) for m in range(L)]
    rp = (ctypes.POINTER(ctypes.c_double) * L)(*[_ptr(a, ctypes.c_double) for a in R])
    cp = (ctypes.POINTER(ctypes.c_uint64) * L)(*[_ptr(a, ctypes.c_uint64) for a in C])
    lib.oracle_subtree(ctypes.byref(idx.c_struct()), rp, cp)
    return R, C


def exact_query(idx: OracleIndex, qtype: int, queries: np.ndarray, K: int = 0, sub=None, threads: int = 0) -> Results:
    """Exact traversal: subtree radii + exact final filter (range) or top-K (KNN)."""
    lib = _load()
    R, C = sub if sub is not None else subtree(idx)
    L = idx.intervals
    rp = (ctypes.POINTER(ctypes.c_double) * L)(*[_ptr(a, ctypes.c_double) for a in R])
    cp = (ctypes.POINTER(ctypes.c_uint64) * L)(*[_ptr(a, ctypes.c_uint64) for a in C])
    q = np.ascontiguousarray(queries, dtype=np.float64)
    res = _OracleResults()
    lib.oracle_exact_query(ctypes.byref(idx.c_struct()), rp, cp, qtype, q.shape[0], _ptr(q, ctypes.c_double), K,
                           threads, ctypes.byref(res))
    return _take(res, lib)


def decode_mesh(idx: OracleIndex, m: int) -> np.ndarray:
    lib = _load()
    out = np.empty((idx.mesh_count(m), idx.D), np.float64)
    lib.oracle_decode_mesh(ctypes.byref(idx.c_struct()), m, _ptr(out, ctypes.c_double))
    return out


def decoded_points(idx: OracleIndex):
    """(points, ids): every finest point's decoded coordinates and its original dataset id."""
    pts = decode_mesh(idx, idx.height - 1)
    return pts, idx.maps[idx.height - 1]


def brute_query(points: np.ndarray, ids: np.ndarray, qtype: int, queries: np.ndarray, K: int = 0,
                threads: int = 0) -> Results:
    lib = _load()
    p = np.ascontiguousarray(points, dtype=np.float64)
    i = np.ascontiguousarray(ids, dtype=np.uint64)
    q = np.ascontiguousarray(queries, dtype=np.float64)
    res = _OracleResults()
    lib.oracle_brute_query(_ptr(p, ctypes.c_double), _ptr(i, ctypes.c_uint64), p.shape[0], p.shape[1], qtype,
                           q.shape[0], _ptr(q, ctypes.c_double), K, threads, ctypes.byref(res))
    return _take(res, lib)


def sqrt_rd(x: float) -> float:
    return _load().oracle_sqrt_rd(x)
