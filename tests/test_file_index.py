"""The JSONL + payload refine service on the CPU (t-blaeq_b200/file_index.py).

A small dataset (timestamped payload files in seqNNNN/<type>/ folders plus a coordinate CSV) is
built by the reference's own tool (oracle/_ref/IndexJsonTblaeqTool build, compiled from the
reference sources; its build runs on the CPU). Checked here without a GPU:
* the service reads the tool's meta.json and JSONL main index, and its timestamp arithmetic
  (microseconds, 21-bit limbs) reproduces every index vector and avg_timestamp_us the tool wrote;
* the refine step equals a line-by-line restatement of the reference's selection and ordering
  rules (IndexJsonTblaeqQuery.cu:216-290) for knn and range requests over all records;
* argument errors carry the reference's messages;
* payload dumps return the bytes of the source files.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO

TOOL = os.path.join(REPO, "oracle", "_ref", "IndexJsonTblaeqTool")
T0 = 1.7e9


def make_dataset(base, n_files=(40, 30, 25), n_coords=60, seed=0, height=3, ratios="4,4"):
    """Writes a synthetic dataset under base/root (+ base/coords.csv) and builds it with the
    reference's tool into base/idx. Returns (index_root, {payload file name: bytes})."""
    rng = np.random.default_rng(seed)
    root = os.path.join(base, "root")
    payloads = {}
    for (seq, folder, ext), n in zip([("seq0001", "Image", ".png"), ("seq0001", "lidar_360", ".npy"),
                                      ("seq0002", "Image", ".png")], n_files):
        d = os.path.join(root, seq, folder)
        os.makedirs(d, exist_ok=True)
        for t in np.sort(rng.uniform(T0, T0 + 100, n)):
            name = f"{t:.6f}{ext}"
            data = rng.integers(0, 255, int(rng.integers(1, 64))).astype(np.uint8).tobytes()
            with open(os.path.join(d, name), "wb") as f:
                f.write(data)
            payloads[name] = data
    csv = os.path.join(base, "coords.csv")
    with open(csv, "w") as f:
        f.write("Sequence,Timestamp,Position,Classification\n")
        for i in range(n_coords):
            f.write(f'seq000{1 + i % 2},{T0 + rng.uniform(0, 100):.6f},"[{rng.normal():.3f}, {rng.normal():.3f}, '
                    f'{rng.normal():.3f}]",{i % 5}\n')
    idx = os.path.join(base, "idx")
    subprocess.run([TOOL, "build", root, csv, idx, "--height", str(height), "--ratios", ratios, "--force-cpu"],
                   check=True, stdout=subprocess.DEVNULL, timeout=600)
    return idx, payloads


@pytest.fixture(scope="module")
def dataset(tmp_path_factory):
    if not os.path.exists(TOOL):
        pytest.skip("reference tool not built (make -C oracle ref needs the reference sources)")
    return make_dataset(str(tmp_path_factory.mktemp("fi")))


@pytest.fixture(scope="module")
def fi(tb):
    import importlib
    return importlib.import_module("tblaeq_b200.file_index")


def test_reads_the_reference_layout_and_reproduces_its_timestamp_vectors(fi, dataset):
    idx, _ = dataset
    d = os.path.join(idx, "file_index")
    meta = fi.load_meta(d)
    rec = fi.load_records(d, meta)
    assert meta.group_size == 1 and len(rec.item_no) == 40 + 30 + 25 + 60
    import json
    lines = [json.loads(x) for x in open(os.path.join(d, "index.jsonl")) if x.strip()]
    for o in lines:
        assert fi.timestamp_to_us(o["avg_timestamp"]) == o["avg_timestamp_us"]
        assert list(fi.split_timestamp_3d(o["avg_timestamp"])) == o["index_vector"][:3]
        assert o["index_vector"][3] == o["seq"]
    assert meta.binary_index_record_size == fi.binary_index_record_size(1, 32) == 99


def _reference_refine(rec, req, cands):
    """Restatement of the reference's refine loops (IndexJsonTblaeqQuery.cu:216-290), record by
    record and slot by slot, over the candidate records sorted by item_no."""
    import importlib
    fi = importlib.import_module("tblaeq_b200.file_index")
    recs = sorted(set(int(c) for c in cands))
    N = rec.group_size
    seqs = sorted(set(req.seqs))
    out = []
    if req.mode == "knn":
        target = fi.timestamp_to_us(req.timestamp)
        for ri, r in enumerate(recs):
            if rec.seq[r] != seqs[0]:
                continue
            for s in range(N):
                if not req.include_padding and rec.sizes[r, s] == 0:
                    continue
                t = int(rec.timestamp_us[r, s])
                out.append((abs(t - target), t, ri, s, r))
        out.sort()
        return [(r, s, d) for d, t, ri, s, r in out[:req.knn_k]]
    lo, hi = fi.timestamp_to_us(req.start), fi.timestamp_to_us(req.end)
    for ri, r in enumerate(recs):
        if int(rec.seq[r]) not in seqs:
            continue
        for s in range(N):
            if not req.include_padding and rec.data_offsets[r, s + 1] == rec.data_offsets[r, s]:
                continue
            t = int(rec.timestamp_us[r, s])
            if lo <= t <= hi:
                out.append((t, ri, s, r))
    out.sort()
    if req.range_limit:
        out = out[:req.range_limit]
    return [(r, s, 0) for t, ri, s, r in out]


def test_refine_equals_the_reference_rules(fi, dataset):
    idx, _ = dataset
    d = os.path.join(idx, "file_index")
    rec = fi.load_records(d, fi.load_meta(d))
    rng = np.random.default_rng(3)
    allc = np.arange(len(rec.item_no), dtype=np.uint64)
    for t in range(40):
        sub = allc[rng.random(len(allc)) < 0.6] if t % 3 else allc
        if t % 2 == 0:
            req = fi.Request(mode="knn", timestamp=T0 + rng.uniform(-5, 105), seqs=[1 + t % 2],
                             knn_k=int(rng.integers(1, 30)))
        else:
            a, b = np.sort(T0 + rng.uniform(-5, 105, 2))
            req = fi.Request(mode="range", start=a, end=b, seqs=[1, 2] if t % 4 == 1 else [2],
                             range_limit=int(rng.integers(0, 3)) * 7)
        seqs, _ = fi._check_request(req)
        got = fi.refine(rec, req, seqs, sub)
        want = _reference_refine(rec, req, sub)
        assert [(m.item_no, m.slot, m.diff_us) for m in got.matches] == [(int(r), s, dd) for r, s, dd in want], t
        assert got.candidate_count == got.record_count == len(sub)
        for m in got.matches:
            assert m.payload_offset == int(rec.index_copy_offset[m.item_no]) + 99 + int(rec.data_offsets[m.item_no, 0])
            assert m.payload_size == int(rec.sizes[m.item_no, m.slot])


def test_argument_errors_carry_the_reference_messages(fi):
    cases = [(fi.Request(mode="knn", seqs=[1]), "--timestamp is required for knn mode"),
             (fi.Request(mode="knn", timestamp=T0, seqs=[1, 2]), "--seq must specify exactly one value for knn mode"),
             (fi.Request(mode="knn", timestamp=T0, seqs=[1], knn_k=0), "--knn-k must be > 0 for knn mode"),
             (fi.Request(mode="range", start=T0, seqs=[1]), "--start and --end are required for range mode"),
             (fi.Request(mode="range", start=T0, end=T0 + 1), "--seq is required for range mode"),
             (fi.Request(mode="range", start=T0 + 1, end=T0, seqs=[1]), "--end must be >= --start"),
             (fi.Request(mode="other"), "unsupported mode: other")]
    for req, msg in cases:
        with pytest.raises(ValueError) as e:
            fi._check_request(req)
        assert str(e.value) == msg


def test_payload_dump_returns_the_source_bytes(fi, dataset, tmp_path):
    idx, payloads = dataset
    d = os.path.join(idx, "file_index")
    rec = fi.load_records(d, fi.load_meta(d))

    class _View:  # the service without a T-BLAEQ handle: dump only reads the main index and data files
        index_dir = d
        records = rec
    req = fi.Request(mode="range", start=T0 - 1, end=T0 + 101, seqs=[1, 2])
    res = fi.refine(rec, req, [1, 2], np.arange(len(rec.item_no)))
    paths = fi.FileIndexService.dump_payloads(_View(), res, str(tmp_path / "dump"))
    assert len(paths) == len(res.matches) > 0
    by_ts = {("%.6f" % float(k.rsplit(".", 1)[0])): v for k, v in payloads.items()}
    checked = 0
    for m, p in zip(res.matches, paths):
        data = open(p, "rb").read()
        assert len(data) == m.payload_size
        if m.dtype != fi.TYPE_COORD:
            assert data == by_ts["%.6f" % m.timestamp]
            checked += 1
    assert checked == 40 + 30 + 25


def test_interval_boxes_cover_exactly_the_interval(fi):
    """The boxes of an interval hold exactly the timestamps in it, whichever limbs the end points
    share (checked against every microsecond of short intervals and random ones across limbs)."""
    rng = np.random.default_rng(9)
    m = (1 << 21) - 1

    def inside(us, boxes):
        v = np.array([((us >> 42) & m) + 1, ((us >> 21) & m) + 1, (us & m) + 1, 1.0])
        return sum(bool(np.all(b[:4] <= v) and np.all(v <= b[4:])) for b in boxes)

    for s_us, e_us in [(5 << 21, (5 << 21) + 10), ((7 << 21) - 3, (7 << 21) + 3), ((1 << 42) - 2, (1 << 42) + 2),
                       (123, 123)]:
        boxes = fi.interval_boxes(s_us / 1e6, e_us / 1e6, 1, 1)
        lo_us, hi_us = fi.timestamp_to_us(s_us / 1e6), fi.timestamp_to_us(e_us / 1e6)
        for us in range(lo_us - 5, hi_us + 6):
            assert inside(us, boxes) == (1 if lo_us <= us <= hi_us else 0), (s_us, e_us, us)
    for _ in range(200):
        a = float(rng.uniform(T0, T0 + 50))
        b = a + float(np.exp(rng.uniform(np.log(1e-5), np.log(1e5))))
        boxes = fi.interval_boxes(a, b, 1, 1)
        lo_us, hi_us = fi.timestamp_to_us(a), fi.timestamp_to_us(b)
        for us in list(rng.integers(lo_us, hi_us + 1, 20)) + [lo_us, hi_us, lo_us - 1, hi_us + 1]:
            assert inside(int(us), boxes) == (1 if lo_us <= us <= hi_us else 0)
