"""Ref-parity against the reference's own CUDA build, run on the same GPU.

oracle/_ref/ref_harness is the reference T-BLAEQ compiled from its sources (oracle/Makefile) plus a
small driver that calls QueryHandler::performSingle{Range,KNN}Query(saveFineMesh=true) one query at a
time and dumps the candidate ids. The B200 build in ref-parity mode must return the same id sets and
the same per-level grid sizes; the CPU oracle must agree as well, which pins the oracle.

When TBLAEQ_GOLDEN_OUT names a directory, the reference's outputs (per-query candidate counts,
SHA-256 of the sorted ids, per-level grid sizes) are also written there as .npz fixtures; committed
under tests/golden/, they pin the CPU oracle without a GPU (test_golden_fixtures.py).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO, oracle_from_handler

pytestmark = pytest.mark.gpu

HARNESS = os.path.join(REPO, "oracle", "_ref", "ref_harness")


def _read_harness(path):
    raw = open(path, "rb").read()
    nq, intervals = np.frombuffer(raw, np.uint64, 2, 0)
    off = 16
    out = []
    for _ in range(int(nq)):
        lv = np.frombuffer(raw, np.uint64, int(intervals), off); off += 8 * int(intervals)
        us = np.frombuffer(raw, np.float64, 1, off)[0]; off += 8
        n = int(np.frombuffer(raw, np.uint64, 1, off)[0]); off += 8
        ids = np.frombuffer(raw, np.uint64, n, off); off += 8 * n
        out.append((lv.copy(), float(us), ids.copy()))
    return out


CASES = [
    # name, N, D, ratios, seed, sigma divisor, query kind, n queries, K
    ("small_range", 500000, 5, (80, 40, 20), 20260330, 2.2, "range", 60, 0),
    ("small_knn", 500000, 5, (80, 40, 20), 20260330, 2.2, "knn", 30, 10),
    ("d8_range", 200000, 8, (100, 50, 20), 1, 3.0, "range", 60, 0),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_reference_cuda_build_agrees(tb, wl, oracle_mod, tmp_path, cuda, case):
    if not os.path.exists(HARNESS):
        pytest.skip("reference build not present (make -C oracle ref needs the reference sources)")
    name, N, D, ratios, seed, sdiv, kind, nq, K = case
    h = tb.QueryHandler.generate(N, D, 1.0, 100.0, False, 4, ratios, seed, sdiv)
    idx_dir = str(tmp_path / "idx")
    h.save_index(idx_dir)
    if kind == "range":
        Q = wl.range_boxes(h, nq, seed=100 + seed % 1000, half_width=0.05)
        qtype, t = tb.QueryType.RANGE, 0
    else:
        Q = wl.knn_points(h, nq, seed=200 + seed % 1000, noise=0.01)
        qtype, t = tb.QueryType.POINT, 1
    qfile = str(tmp_path / "q.txt")
    tb.save_query_file(qfile, qtype, Q, D)
    out = str(tmp_path / "ref.bin")
    subprocess.run([HARNESS, idx_dir, qfile, str(t), str(K), "L0", out], check=True, timeout=600,
                   stdout=subprocess.DEVNULL)
    ref = _read_harness(out)
    o = oracle_mod.load_index(idx_dir)
    orc = oracle_mod.ref_query(o, oracle_mod.RANGE if kind == "range" else oracle_mod.KNN, Q, K=K)
    for q in range(nq):
        lv, us, ids = ref[q]
        assert np.array_equal(ids, orc.query(q)), f"oracle vs reference CUDA, query {q}"
        assert np.array_equal(lv, orc.level_sizes[q])
    h.prepare_for_query(tb.LevelPolicy.L0)
    if kind == "range":
        r = h.query_batch(qtype, Q, tb.Mode.REF_PARITY)
        offs = r.offsets.numpy()
        got = r.ids.numpy()
        for q in range(nq):
            assert np.array_equal(np.sort(got[offs[q]:offs[q + 1]]), ref[q][2]), f"B200 vs reference, query {q}"
    else:
        # The B200 KNN plugin (IQueryStrategy::runLevel, POINT) level by level against the reference
        # CUDA build directly: the same per-level grid sizes and the same final candidate ids.
        for q in range(nq):
            grid = h.coarsest_grid()
            sizes = []
            for l in range(h.info()["intervals"]):
                grid = h.run_level(l, grid, tb.QueryType.POINT, point=Q[q], K=K)
                sizes.append(grid.nnz)
            got, _ = h.grid_arrays(grid)
            assert np.array_equal(np.array(sizes, np.uint64), ref[q][0]), f"B200 plugin vs reference, query {q}"
            assert np.array_equal(np.sort(got), ref[q][2]), f"B200 plugin vs reference, query {q}"
    gold = os.environ.get("TBLAEQ_GOLDEN_OUT")
    if gold:
        os.makedirs(gold, exist_ok=True)
        import hashlib
        digests = np.array([np.frombuffer(hashlib.sha256(np.sort(r[2]).astype("<u8").tobytes()).digest(), np.uint8)
                            for r in ref])
        np.savez_compressed(os.path.join(gold, f"ref_cuda_{name}.npz"), queries=Q, K=K,
                            params=np.array([N, D, *ratios, seed], np.uint64), sigma_divisor=sdiv,
                            counts=np.array([len(r[2]) for r in ref], np.uint64), digests=digests,
                            levels=np.stack([r[0] for r in ref]).astype(np.uint64),
                            query_us=np.array([r[1] for r in ref]))
