"""The JSONL + payload refine service on the GPU against the reference's own service.

The dataset is built by the reference's tool (oracle/_ref/IndexJsonTblaeqTool build, CPU). The
reference's refine service itself, run_query_service (src/file_index/IndexJsonTblaeqQuery.cu:294-380),
answers every request through oracle/_ref/file_index_harness on the same GPU; the B200 service
answers all of them in two batched traversals:
* in ref-parity mode the matches are identical to the reference's, request for request (rank,
  record, slot, sequence, type, timestamp, difference, payload offset and size, data file), and so
  are the candidate, record and slot counts;
* in exact mode the coarse candidates are exactly the records holding a slot whose timestamp lies
  in the request's interval (range) or the K nearest points of the T-BLAEQ index (KNN: the FP64
  brute force over its decoded points, id tie-break), and the refined matches equal the refine of
  those candidates; range requests without a match limit never lose a match against ref-parity
  mode (with a limit, each mode keeps the earliest of its own matches).

A request on which the reference's harness process dies is recorded with its exit status and the
harness restarts after it; the parity test names such requests and compares all the others.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO
from test_file_index import T0, make_dataset

pytestmark = pytest.mark.gpu

HARNESS = os.path.join(REPO, "oracle", "_ref", "file_index_harness")
TOOL = os.path.join(REPO, "oracle", "_ref", "IndexJsonTblaeqTool")


def _requests(fi, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for t in range(n):
        if t % 2 == 0:
            out.append(fi.Request(mode="knn", timestamp=float(T0 + rng.uniform(-2, 102)), seqs=[1 + (t // 2) % 2],
                                  knn_k=int([1, 5, 20, 60][t % 4])))
        else:
            a = T0 + rng.uniform(-2, 100)
            b = a + float(np.exp(rng.uniform(np.log(0.01), np.log(80))))
            out.append(fi.Request(mode="range", start=float(a), end=float(b), seqs=[[1], [2], [1, 2]][t % 3],
                                  range_limit=[0, 0, 10][t % 3], include_padding=bool(t % 5 == 0)))
    return out


def _parse_reference(out):
    """Complete requests of a harness output file (the harness flushes after each request)."""
    res, cur, want = [], None, 0
    for line in open(out):
        f = line.split()
        if f[0] == "R":
            cur = {"counts": tuple(int(x) for x in f[1:4]), "matches": []}
            want = int(f[4])
            res.append(cur)
        elif f[0] == "M":
            cur["matches"].append((int(f[1]), int(f[2]), int(f[3]), int(f[4]), int(f[5]), float(f[6]), int(f[7]),
                                   int(f[8]), int(f[9]), f[10]))
        else:
            res.append({"error": line[2:].strip()})
    if cur is not None and len(cur["matches"]) != want:
        res.pop()  # cut off inside its last request
    return res


def _run_reference(idx, reqs, tmp):
    """The reference service's answer to each request, or {"crashed": status, "stderr": tail} for a
    request on which the harness process died."""
    res = []
    while len(res) < len(reqs):
        path = os.path.join(tmp, "req.txt")
        with open(path, "w") as f:
            for r in reqs[len(res):]:
                if r.mode == "knn":
                    f.write(f"knn {r.timestamp!r} {r.knn_k} {int(r.include_padding)} {r.seqs[0]}\n")
                else:
                    f.write(f"range {r.start!r} {r.end!r} {r.range_limit} {int(r.include_padding)} {len(r.seqs)} "
                            + " ".join(str(s) for s in r.seqs) + "\n")
        out = os.path.join(tmp, "out.txt")
        p = subprocess.run([HARNESS, idx, path, out], timeout=600, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
        got = _parse_reference(out)
        res.extend(got)
        if p.returncode == 0:
            assert len(res) == len(reqs)
            break
        res.append({"crashed": p.returncode, "stderr": p.stderr.decode(errors="replace")[-300:]})
    return res


@pytest.fixture(scope="module")
def service(tb, tmp_path_factory, cuda):
    if not (os.path.exists(TOOL) and os.path.exists(HARNESS)):
        pytest.skip("reference tool not built (make -C oracle ref needs the reference sources)")
    import importlib
    fi = importlib.import_module("tblaeq_b200.file_index")
    base = str(tmp_path_factory.mktemp("fi_gpu"))
    idx, _ = make_dataset(base, n_files=(400, 300, 250), n_coords=2000, seed=5, height=3, ratios="10,10")
    return fi, idx, fi.FileIndexService(idx), base


def test_ref_parity_matches_the_reference_service(service):
    fi, idx, svc, base = service
    reqs = _requests(fi, 48, 1)
    ref = _run_reference(idx, reqs, base)
    got = svc.query(reqs, mode=svc_mode(svc, "REF_PARITY"))
    assert len(ref) == len(got)
    crashed = [(q, reqs[q], r) for q, r in enumerate(ref) if "crashed" in r]
    for c in crashed:
        print("the reference harness died on request", c)
    assert len(crashed) <= len(reqs) // 4
    n_matches = 0
    for q, (r, g) in enumerate(zip(ref, got)):
        if "crashed" in r:
            continue
        assert "error" not in r and g.error is None, (q, r, g.error)
        assert (g.candidate_count, g.record_count, g.slot_count) == r["counts"], q
        mine = [(m.rank, m.item_no, m.seq, m.dtype, m.slot, m.timestamp, m.diff_us, m.payload_offset, m.payload_size,
                 m.data_file) for m in g.matches]
        assert mine == r["matches"], q
        n_matches += len(mine)
    assert n_matches > 100


def svc_mode(svc, name):
    import tblaeq_b200 as tb
    return getattr(tb.Mode, name)


def test_exact_mode_equals_brute_force_candidates(service, oracle_mod):
    fi, idx, svc, base = service
    reqs = _requests(fi, 48, 2)
    got = svc.query(reqs, mode=svc_mode(svc, "EXACT"))
    par = svc.query(reqs, mode=svc_mode(svc, "REF_PARITY"))
    vecs = svc.records.index_vector
    ids = svc.records.item_no
    dec_pts, dec_ids = oracle_mod.decoded_points(oracle_mod.load_index(os.path.join(idx, "tblaeq_index")))
    gained = 0
    for q, r in enumerate(reqs):
        seqs, v = fi._check_request(r)
        if r.mode == "range":
            # Records holding a slot with a timestamp in [start, end], sequences in range.
            ts = svc.records.timestamp_us
            s_us, e_us = fi.timestamp_to_us(r.start), fi.timestamp_to_us(r.end)
            inside = np.any((ts >= s_us) & (ts <= e_us), axis=1)
            cand = ids[inside & (vecs[:, 3] >= seqs[0]) & (vecs[:, 3] <= seqs[-1])]
        else:
            b = oracle_mod.brute_query(dec_pts, dec_ids, oracle_mod.KNN, v[None, :], K=r.knn_k)
            cand = b.ids
        want = fi.refine(svc.records, r, seqs, cand)
        assert got[q].candidate_count == want.candidate_count, q
        assert [(m.item_no, m.slot) for m in got[q].matches] == [(m.item_no, m.slot) for m in want.matches], q
        if r.mode == "range" and r.range_limit == 0:
            assert set((m.item_no, m.slot) for m in par[q].matches) <= set((m.item_no, m.slot) for m in got[q].matches)
            gained += len(got[q].matches) - len(par[q].matches)
    print(f"range matches the reference's candidates missed and exact mode found: {gained}")


def test_bad_requests_are_reported_per_request(service):
    fi, idx, svc, base = service
    reqs = [fi.Request(mode="knn", seqs=[1]), fi.Request(mode="range", start=T0, end=T0 + 10, seqs=[1])]
    got = svc.query(reqs)
    assert got[0].error == "--timestamp is required for knn mode"
    assert got[1].error is None and len(got[1].matches) > 0
