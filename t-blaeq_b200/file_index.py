"""JSONL + payload refine service over the batched traversal.

The reference's IndexJsonTblaeq tool keeps a dataset of timestamped payloads (images, point clouds,
coordinate records) in three parts: a JSONL main index (one fixed-layout record per group of
payloads), binary data files holding a copy of each record followed by its payloads, and a
T-BLAEQ index over one 4-D vector per record: the three 21-bit limbs (+1) of the group's mean
timestamp in microseconds and the sequence number (src/file_index/IndexJsonTblaeqBuild.cu:265-297,
src/file_index/IndexJsonTblaeqUtils.cu:132-153). Its query service
(src/file_index/IndexJsonTblaeqQuery.cu:294-380) answers one request at a time: a T-BLAEQ range or
KNN query yields candidate records, which it re-reads from the JSONL file and refines on the host
by timestamp.

This service opens the same on-disk layout and keeps the whole main index in memory as arrays.
`query` takes many requests at once: every range request's coarse query runs in one batched
traversal, every KNN request's in another, and the candidates are refined per request with the
reference's selection and ordering rules. Two coarse modes:

* Mode.REF_PARITY: the reference's candidate sets (its non-conservative per-level pruning and
  STEP selection), so the matches equal the reference tool's, request for request;
* Mode.EXACT: range candidates are exactly the records holding a slot whose timestamp lies in
  [start, end] (and whose sequence lies between the smallest and largest requested). A record's
  index vector encodes its group's mean timestamp, so the slots of a record lie within a fixed
  spread of that key (the largest over the index, measured when the service opens it): the interval
  widened by that spread is queried as the few boxes whose union it is (`interval_boxes_us`), and
  the records without a slot in the interval are dropped. The reference queries one box of
  per-limb minima and maxima of the bare interval and prunes non-conservatively, so it can miss
  such records. KNN candidates are exactly the K nearest points of the index (its decoded
  coordinates, FP64 distances, smaller id first on ties).

Refinement (same rules as the reference):
* knn: slots of candidate records of the request's sequence, ordered by |timestamp_us - target|,
  then timestamp_us, record, slot; the first knn_k (IndexJsonTblaeqQuery.cu:256-290);
* range: slots of candidate records whose sequence is listed, with timestamp_us in [start, end],
  ordered by timestamp_us, record, slot; at most range_limit (0: all) (:216-254).
Zero-size padding slots are skipped unless include_padding is set.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

KNN_DIM = 4
MAX_N = 255
MAX_FILE_NAME_BYTES = 256
TYPE_IMAGE, TYPE_LIDAR_360, TYPE_LIVOX_AVIA, TYPE_RADAR_ENCHANCE_PCL, TYPE_COORD = 0, 1, 2, 3, 4
DEFAULT_INDEX_DIR = "file_index"
DEFAULT_TBLAEQ_DIR = "tblaeq_index"


# ---- timestamps (src/file_index/IndexJsonTblaeqUtils.cu:132-153) ---------------------------------
def timestamp_to_us(timestamp: float) -> int:
    """Microseconds as the reference computes them: the timestamp times 1e6 in x87 extended
    precision, rounded half away from zero."""
    scaled = np.longdouble(timestamp) * np.longdouble(1000000.0)
    if not np.isfinite(scaled) or abs(scaled) > np.longdouble(2.0 ** 63 - 1):
        raise RuntimeError("timestamp microseconds overflow int64")
    r = np.floor(abs(scaled) + np.longdouble(0.5))
    return int(r) if scaled >= 0 else -int(r)


def split_timestamp_3d(timestamp: float):
    """The three 21-bit limbs (bits 42..62, 21..41, 0..20) of the microsecond timestamp, each + 1."""
    us = timestamp_to_us(timestamp)
    if us < 0:
        raise RuntimeError("negative timestamp is not supported")
    mask = (1 << 21) - 1
    return (float(((us >> 42) & mask) + 1), float(((us >> 21) & mask) + 1), float((us & mask) + 1))


def interval_boxes(start: float, end: float, seq_lo: int, seq_hi: int):
    """Boxes in index-vector space (lo[4] | hi[4]) whose union holds exactly the vectors of the
    microsecond timestamps in [start, end] (sequences seq_lo..seq_hi). The vector splits a timestamp
    into three 21-bit limbs, so the interval is a run in lexicographic limb order: at most five boxes
    (a partial low limb, partial middle limbs, whole top limbs, and the mirror images at the end).
    The reference's single box of per-limb minima and maxima is not this set: it misses timestamps
    whose low limbs fall outside the end points' (and can hold ones outside the interval)."""
    return interval_boxes_us(timestamp_to_us(start), timestamp_to_us(end), seq_lo, seq_hi)


def interval_boxes_us(s_us: int, e_us: int, seq_lo: int, seq_hi: int):
    """`interval_boxes` of the microsecond interval [s_us, e_us]."""
    if s_us < 0 or e_us < 0:
        raise RuntimeError("negative timestamp is not supported")
    m = (1 << 21) - 1
    a0, b0, c0 = s_us >> 42, (s_us >> 21) & m, s_us & m
    a1, b1, c1 = e_us >> 42, (e_us >> 21) & m, e_us & m
    runs = []  # (a range, b range, c range), limb values before the + 1
    if a0 == a1 and b0 == b1:
        runs.append(((a0, a0), (b0, b0), (c0, c1)))
    elif a0 == a1:
        runs.append(((a0, a0), (b0, b0), (c0, m)))
        if b0 + 1 <= b1 - 1:
            runs.append(((a0, a0), (b0 + 1, b1 - 1), (0, m)))
        runs.append(((a0, a0), (b1, b1), (0, c1)))
    else:
        runs.append(((a0, a0), (b0, b0), (c0, m)))
        if b0 < m:
            runs.append(((a0, a0), (b0 + 1, m), (0, m)))
        if a0 + 1 <= a1 - 1:
            runs.append(((a0 + 1, a1 - 1), (0, m), (0, m)))
        if b1 > 0:
            runs.append(((a1, a1), (0, b1 - 1), (0, m)))
        runs.append(((a1, a1), (b1, b1), (0, c1)))
    return [np.array([ra[0] + 1, rb[0] + 1, rc[0] + 1, seq_lo, ra[1] + 1, rb[1] + 1, rc[1] + 1, seq_hi],
                     dtype=np.float64) for ra, rb, rc in runs]


def binary_index_record_size(n: int, file_name_bytes: int) -> int:
    """Bytes of a record's binary copy in its data file (<4dBB{n}dB{fnb}sQ{n+1}Q)."""
    return 4 * 8 + 1 + 1 + n * 8 + 1 + file_name_bytes + 8 + (n + 1) * 8


# ---- the main index --------------------------------------------------------------------------------
@dataclass
class Meta:
    index_file: str
    index_record_count: int
    group_size: int
    file_name_bytes: int
    binary_index_record_size: int


def _u64(obj, key):
    v = obj.get(key)
    if v is None:
        raise RuntimeError("missing JSON field: " + key)
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise RuntimeError("JSON field must be integer number: " + key)
    if isinstance(v, float) and v != round(v):
        raise RuntimeError("JSON field is not integral: " + key)
    if v < 0:
        raise RuntimeError("JSON field must be non-negative: " + key)
    return int(v)


def load_meta(index_dir: str) -> Meta:
    """meta.json of a main index (IndexJsonTblaeqJson.cu:84-109), checked for consistency."""
    path = os.path.join(index_dir, "meta.json")
    if not os.path.exists(path):
        raise RuntimeError("missing meta.json: " + path)
    try:
        obj = json.load(open(path))
    except ValueError as e:
        raise RuntimeError("failed to parse meta.json: " + str(e))
    if not isinstance(obj, dict):
        raise RuntimeError("JSON root must be object: meta.json")
    m = Meta(index_file=obj.get("index_file", "index.jsonl"),
             index_record_count=_u64(obj, "index_record_count") if "index_record_count" in obj else 0,
             group_size=_u64(obj, "group_size_N"), file_name_bytes=_u64(obj, "file_name_bytes"),
             binary_index_record_size=_u64(obj, "binary_index_record_size"))
    if not 1 <= m.group_size <= MAX_N:
        raise RuntimeError("meta group_size_N must be in [1, 255]")
    if not 1 <= m.file_name_bytes <= MAX_FILE_NAME_BYTES:
        raise RuntimeError("meta file_name_bytes must be in [1, 256]")
    expected = binary_index_record_size(m.group_size, m.file_name_bytes)
    if m.binary_index_record_size != expected:
        raise RuntimeError(f"binary_index_record_size={m.binary_index_record_size}, expected={expected}")
    return m


@dataclass
class Records:
    """The main index as arrays, row r = the record with item_no r."""
    item_no: np.ndarray          # (n,) uint64
    seq: np.ndarray              # (n,) uint8
    dtype: np.ndarray            # (n,) uint8
    index_vector: np.ndarray     # (n, 4) float64
    timestamps: np.ndarray       # (n, N) float64
    timestamp_us: np.ndarray     # (n, N) int64
    sizes: np.ndarray            # (n, N) uint64
    data_offsets: np.ndarray     # (n, N + 1) uint64
    index_copy_offset: np.ndarray  # (n,) uint64
    bin_size: int
    file_name: List[str]
    group_size: int


def record_keys_us(records: Records) -> np.ndarray:
    """Each record's key in microseconds: the timestamp its index vector's limbs encode."""
    lim = np.rint(records.index_vector[:, :3]).astype(np.int64) - 1
    return (lim[:, 0] << 42) | (lim[:, 1] << 21) | lim[:, 2]


def load_records(index_dir: str, meta: Meta) -> Records:
    """Every line of the JSONL main index, validated like the reference's parser
    (IndexJsonTblaeqJson.cu:111-168), in item_no order."""
    path = os.path.join(index_dir, meta.index_file)
    if not os.path.exists(path):
        raise RuntimeError("missing index file: " + path)
    n = meta.group_size
    rows = []
    with open(path) as f:
        for line_no, line in enumerate(f, 1):
            line = line.rstrip("\r\n")
            if not line.strip():
                continue
            try:
                o = json.loads(line)
            except ValueError as e:
                raise RuntimeError(f"failed to parse index JSONL line {line_no}: {e}")
            if not isinstance(o, dict):
                raise RuntimeError("JSON root must be object: index JSONL line")
            slot_count, valid_count = _u64(o, "slot_count"), _u64(o, "valid_count")
            if slot_count != n:
                raise RuntimeError(f"slot_count does not match meta at line {line_no}")
            if valid_count > slot_count:
                raise RuntimeError(f"valid_count > slot_count at line {line_no}")
            if _u64(o, "binary_index_record_size") != meta.binary_index_record_size:
                raise RuntimeError(f"binary_index_record_size mismatch at line {line_no}")
            name = o.get("file_name")
            if not isinstance(name, str):
                raise RuntimeError("JSON field must be string: file_name")
            if len(name.encode()) > meta.file_name_bytes:
                raise RuntimeError("file_name too long for fixed field: " + name)
            vec = o.get("index_vector")
            if not isinstance(vec, list) or len(vec) != 4:
                raise RuntimeError(f"index_vector length must be 4 at line {line_no}")
            ts, tus, offs, sizes = (o.get(k) for k in ("timestamps", "timestamp_us", "data_offsets", "sizes"))
            if not all(isinstance(a, list) for a in (ts, tus, offs, sizes)) or len(ts) != n or len(tus) != n \
                    or len(sizes) != n or len(offs) != n + 1:
                raise RuntimeError(f"fixed array length mismatch at line {line_no}")
            if any(s < 0 for s in sizes):
                raise RuntimeError(f"negative size at line {line_no}")
            if any(x < 0 for x in offs):
                raise RuntimeError(f"negative data offset at line {line_no}")
            if offs[0] != 0:
                raise RuntimeError(f"data_offsets[0] must be 0 at line {line_no}")
            for i in range(n):
                if offs[i + 1] < offs[i]:
                    raise RuntimeError(f"data_offsets not monotonic at line {line_no}")
                if offs[i + 1] - offs[i] != sizes[i]:
                    raise RuntimeError(f"sizes[i] != data_offsets[i+1]-data_offsets[i] at line {line_no}")
                if i >= valid_count and sizes[i] != 0:
                    raise RuntimeError(f"padding slot has non-zero size at line {line_no}")
            seq, dt = _u64(o, "seq"), _u64(o, "dtype_id")
            if seq > 255:
                raise RuntimeError("field does not fit uint8: seq")
            if dt > 255:
                raise RuntimeError("field does not fit uint8: dtype_id")
            rows.append((_u64(o, "item_no"), seq, dt, [float(v) for v in vec], [float(v) for v in ts],
                         [int(v) for v in tus], [int(v) for v in sizes], [int(v) for v in offs],
                         _u64(o, "index_copy_offset"), name))
    if meta.index_record_count and len(rows) != meta.index_record_count:
        raise RuntimeError("index_record_count does not match actual JSONL line count")
    rows.sort(key=lambda r: r[0])
    items = np.array([r[0] for r in rows], np.uint64)
    if len(rows) and not np.array_equal(items, np.arange(len(rows), dtype=np.uint64)):
        raise RuntimeError("item_no values must be 0..n-1 (the T-BLAEQ dataset rows)")
    return Records(item_no=items, seq=np.array([r[1] for r in rows], np.uint8),
                   dtype=np.array([r[2] for r in rows], np.uint8),
                   index_vector=np.array([r[3] for r in rows], np.float64).reshape(-1, 4),
                   timestamps=np.array([r[4] for r in rows], np.float64).reshape(-1, n),
                   timestamp_us=np.array([r[5] for r in rows], np.int64).reshape(-1, n),
                   sizes=np.array([r[6] for r in rows], np.uint64).reshape(-1, n),
                   data_offsets=np.array([r[7] for r in rows], np.uint64).reshape(-1, n + 1),
                   index_copy_offset=np.array([r[8] for r in rows], np.uint64),
                   bin_size=meta.binary_index_record_size, file_name=[r[9] for r in rows], group_size=n)


# ---- requests and results (QueryArgs / QueryServiceResult of IndexJsonTblaeqTypes.cuh) ------------
@dataclass
class Request:
    mode: str = "knn"                 # "knn" | "range"
    timestamp: Optional[float] = None  # knn
    start: Optional[float] = None      # range
    end: Optional[float] = None        # range
    seqs: Sequence[int] = ()
    knn_k: int = 10
    range_limit: int = 0               # 0: all
    include_padding: bool = False


@dataclass
class PayloadMatch:
    rank: int
    item_no: int
    seq: int
    dtype: int
    slot: int
    timestamp: float
    diff_us: int
    payload_offset: int
    payload_size: int
    data_file: str


@dataclass
class ServiceResult:
    candidate_count: int = 0
    record_count: int = 0
    slot_count: int = 0
    matches: List[PayloadMatch] = field(default_factory=list)
    error: Optional[str] = None


def _check_request(r: Request):
    """The reference's argument checks, with its messages (IndexJsonTblaeqQuery.cu:306-336)."""
    seqs = sorted(set(int(s) for s in r.seqs))
    if any(s < 0 or s > 255 for s in seqs):
        raise ValueError("seq does not fit uint8")
    if r.mode == "knn":
        if r.timestamp is None:
            raise ValueError("--timestamp is required for knn mode")
        if len(seqs) != 1:
            raise ValueError("--seq must specify exactly one value for knn mode")
        if r.knn_k <= 0:
            raise ValueError("--knn-k must be > 0 for knn mode")
        v = split_timestamp_3d(r.timestamp)
        return seqs, np.array([v[0], v[1], v[2], float(seqs[0])])
    if r.mode == "range":
        if r.start is None or r.end is None:
            raise ValueError("--start and --end are required for range mode")
        if not seqs:
            raise ValueError("--seq is required for range mode")
        if r.end < r.start:
            raise ValueError("--end must be >= --start")
        a, b = split_timestamp_3d(r.start), split_timestamp_3d(r.end)
        lo = [min(a[i], b[i]) for i in range(3)] + [float(seqs[0])]
        hi = [max(a[i], b[i]) for i in range(3)] + [float(seqs[-1])]
        return seqs, np.array(lo + hi)
    raise ValueError("unsupported mode: " + str(r.mode))


def refine(records: Records, r: Request, seqs, candidates: np.ndarray) -> ServiceResult:
    """Refines one request's candidate records (item numbers) by timestamp, with the reference's
    selection and ordering rules, into payload matches."""
    cand = np.unique(np.asarray(candidates, np.uint64))
    out = ServiceResult(candidate_count=int(len(cand)))
    if len(cand) == 0:
        return out
    if int(cand[-1]) >= len(records.item_no):
        raise RuntimeError(f"missing {int(np.sum(cand >= len(records.item_no)))} candidate index record(s)")
    rec = cand.astype(np.int64)  # rows of the candidate records, ascending item_no = record order
    out.record_count = int(len(rec))
    N = records.group_size
    ridx = np.repeat(np.arange(len(rec)), N)        # record index among the candidates
    slot = np.tile(np.arange(N), len(rec))
    rows = rec[ridx]
    ts_us = records.timestamp_us[rows, slot]
    if r.mode == "knn":
        keep = records.seq[rows] == seqs[0]
        if not r.include_padding:
            keep &= records.sizes[rows, slot] != 0
        target = timestamp_to_us(r.timestamp)
        diff = np.abs(ts_us - target)
        sel = np.nonzero(keep)[0]
        order = sel[np.lexsort((slot[sel], ridx[sel], ts_us[sel], diff[sel]))]
        order = order[:r.knn_k] if r.knn_k > 0 else order
    else:
        keep = np.isin(records.seq[rows], np.array(seqs, np.uint8))
        if not r.include_padding:
            keep &= (records.data_offsets[rows, slot + 1] - records.data_offsets[rows, slot]) != 0
        out.slot_count = int(np.count_nonzero(keep))
        lo, hi = timestamp_to_us(r.start), timestamp_to_us(r.end)
        keep &= (ts_us >= lo) & (ts_us <= hi)
        sel = np.nonzero(keep)[0]
        order = sel[np.lexsort((slot[sel], ridx[sel], ts_us[sel]))]
        diff = np.zeros(len(ts_us), np.int64)
        if r.range_limit > 0:
            order = order[:r.range_limit]
    for rank, i in enumerate(order):
        row, s = int(rows[i]), int(slot[i])
        start_rel = int(records.data_offsets[row, s])
        end_rel = int(records.data_offsets[row, s + 1])
        base = int(records.index_copy_offset[row]) + records.bin_size
        out.matches.append(PayloadMatch(rank=rank, item_no=int(records.item_no[row]), seq=int(records.seq[row]),
                                        dtype=int(records.dtype[row]), slot=s,
                                        timestamp=float(records.timestamps[row, s]), diff_us=int(diff[i]),
                                        payload_offset=base + start_rel, payload_size=end_rel - start_rel,
                                        data_file=records.file_name[row]))
    return out


class FileIndexService:
    """The refine service over one index root (<root>/file_index and <root>/tblaeq_index, as the
    reference's tool writes them). The T-BLAEQ index is opened and prepared once; the main index is
    loaded once into arrays."""

    def __init__(self, index_root: str, index_dir: str = DEFAULT_INDEX_DIR, tblaeq_dir: str = DEFAULT_TBLAEQ_DIR,
                 policy=None, handler=None):
        from . import QueryHandler, LevelPolicy
        self.index_dir = os.path.join(index_root, index_dir)
        tdir = os.path.join(index_root, tblaeq_dir)
        if not os.path.exists(self.index_dir):
            raise RuntimeError("index dir not found: " + self.index_dir)
        if handler is None and not os.path.exists(tdir):
            raise RuntimeError("tblaeq index dir not found: " + tdir)
        self.meta = load_meta(self.index_dir)
        self.records = load_records(self.index_dir, self.meta)
        self.handler = handler if handler is not None else QueryHandler(tdir, True)
        if handler is None:
            self.handler.prepare_for_query(policy if policy is not None else LevelPolicy.L0)
        if self.handler.info()["D"] != KNN_DIM:
            raise RuntimeError("the T-BLAEQ index of a file index must be 4-dimensional")
        # How far a record's slots reach below and above its key (exact range candidates).
        key = record_keys_us(self.records)
        ts = self.records.timestamp_us
        self.slot_spread_us = ((int(max(0, np.max(key - ts.min(1)))), int(max(0, np.max(ts.max(1) - key))))
                               if len(key) else (0, 0))

    def query(self, requests: Sequence[Request], mode=None) -> List[ServiceResult]:
        """Answers every request; a request whose arguments the reference would reject carries the
        reference's message in `error` and no matches."""
        from . import Mode, QueryType
        mode = Mode.EXACT if mode is None else mode
        out: List[Optional[ServiceResult]] = [None] * len(requests)
        checked = []
        for i, r in enumerate(requests):
            try:
                seqs, v = _check_request(r)
                checked.append((i, seqs, v))
            except ValueError as e:
                out[i] = ServiceResult(error=str(e))
        cands = {}
        rng = [(i, s, v) for i, s, v in checked if requests[i].mode == "range"]
        if rng:
            if mode == Mode.EXACT:
                # The boxes whose union is exactly the keys of the request's interval widened by the
                # slots' spread (and the sequence range). Index vectors are integers (limbs + 1,
                # sequence numbers) and the index's decoded coordinates differ from them by rounding
                # only (far below 0.25): boxes widened by a quarter hold exactly the records whose
                # stored vector lies in them.
                below, above = self.slot_spread_us
                per = [interval_boxes_us(max(0, timestamp_to_us(requests[i].start) - above),
                                         timestamp_to_us(requests[i].end) + below, sq[0], sq[-1])
                       for i, sq, _ in rng]
                boxes = np.stack([b for bs in per for b in bs])
                boxes[:, :KNN_DIM] -= 0.25
                boxes[:, KNN_DIM:] += 0.25
                owner = np.repeat(np.arange(len(rng)), [len(bs) for bs in per])
            else:
                boxes = np.stack([v for _, _, v in rng])
                owner = np.arange(len(rng))
            res = self.handler.query_batch(QueryType.RANGE, np.ascontiguousarray(boxes), mode)
            offs, ids = res.offsets.numpy(), (res.ids.numpy() if res.total else np.zeros(0, np.uint64))
            parts = [[] for _ in rng]
            for b, j in enumerate(owner):
                parts[j].append(ids[offs[b]:offs[b + 1]])
            for j, (i, _, _) in enumerate(rng):
                c = np.concatenate(parts[j]) if parts[j] else np.zeros(0, np.uint64)
                if mode == Mode.EXACT and len(c):
                    c = np.unique(c)
                    if int(c[-1]) < len(self.records.item_no):  # else refine reports the missing records
                        t = self.records.timestamp_us[c.astype(np.int64)]
                        lo, hi = timestamp_to_us(requests[i].start), timestamp_to_us(requests[i].end)
                        c = c[np.any((t >= lo) & (t <= hi), axis=1)]
                cands[i] = c
        knn = [(i, s, v) for i, s, v in checked if requests[i].mode == "knn"]
        if knn and mode == Mode.EXACT:
            pts = np.ascontiguousarray(np.stack([v for _, _, v in knn]))
            ks = np.array([requests[i].knn_k for i, _, _ in knn], np.uint32)
            res = self.handler.query_batch(QueryType.POINT, pts, Mode.EXACT, K=ks)
            offs, ids = res.offsets.numpy(), (res.ids.numpy() if res.total else np.zeros(0, np.uint64))
            for j, (i, _, _) in enumerate(knn):
                cands[i] = ids[offs[j]:offs[j + 1]]
        elif knn:
            # The reference's KNN candidates: per-level plugin steps (bound, sort, STEP) of one query.
            L = self.handler.info()["intervals"]
            for i, _, v in knn:
                grid = self.handler.coarsest_grid()
                for lvl in range(L):
                    grid = self.handler.run_level(lvl, grid, QueryType.POINT, point=v, K=requests[i].knn_k)
                cands[i] = self.handler.grid_arrays(grid)[0].copy()
        for i, seqs, _ in checked:
            out[i] = refine(self.records, requests[i], seqs, cands[i])
        return out

    def dump_payloads(self, result: ServiceResult, dump_dir: str) -> List[str]:
        """Writes each match's payload bytes to its own file (names as the reference's dump,
        IndexJsonTblaeqQuery.cu:84-93); returns the paths."""
        os.makedirs(dump_dir, exist_ok=True)
        ext = {TYPE_IMAGE: ".png", TYPE_LIDAR_360: ".npy", TYPE_LIVOX_AVIA: ".npy",
               TYPE_RADAR_ENCHANCE_PCL: ".npy", TYPE_COORD: ".coord.bin"}
        paths = []
        for m in result.matches:
            ts = ("%.6f" % m.timestamp).replace(".", "_")
            name = (f"match_{m.rank:04d}_item{m.item_no:08d}_slot{m.slot:03d}_seq{m.seq:04d}_dtype{m.dtype}_{ts}"
                    f"{ext.get(m.dtype, '.bin')}")
            src = os.path.join(self.index_dir, m.data_file)
            if not os.path.exists(src):
                raise RuntimeError("data file not found: " + src)
            size = os.path.getsize(src)
            if m.payload_offset > size or m.payload_size > size - m.payload_offset:
                raise RuntimeError(f"payload range exceeds data file length: file={src} "
                                   f"abs_start={m.payload_offset} size={m.payload_size} file_size={size}")
            with open(src, "rb") as f:
                f.seek(m.payload_offset)
                data = f.read(m.payload_size)
            p = os.path.join(dump_dir, name)
            with open(p, "wb") as f:
                f.write(data)
            paths.append(p)
        return paths
