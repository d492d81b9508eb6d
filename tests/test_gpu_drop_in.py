"""The drop-in proof, from both sides.

* The reference's own engine drives the B200 library: oracle/_ref/b200_drop_in is the reference's
  QueryHandler / QueryEngine (compiled from its sources) with one expression changed, the L0 case of
  PolicyScheduler::makeForLevel, which returns the reference-side adapter B200Strategy
  (oracle/ref_shim/b200/B200Strategy.cuh) over tblaeq_level. Its performSingleRangeQuery /
  performSingleKNNQuery results (candidate ids and every level's grid size) equal the unmodified
  reference build's (oracle/_ref/ref_harness, policy L0) query for query, and every level of every
  query ran in the B200 library.
* The B200 library's C++ facade is the reference's query API: a C++ caller (tests/cpp/facade_check.cpp)
  of QueryHandler::performQuery / performSingle*Query gets the reference's candidate sets in
  ref-parity mode and the FP64 brute force's answers in exact mode.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

REF = os.path.join(REPO, "oracle", "_ref", "ref_harness")
DROP_IN = os.path.join(REPO, "oracle", "_ref", "b200_drop_in")


def _read(path):
    raw = open(path, "rb").read()
    nq, intervals = (int(x) for x in np.frombuffer(raw, np.uint64, 2, 0))
    off, out = 16, []
    for _ in range(nq):
        lv = np.frombuffer(raw, np.uint64, intervals, off); off += 8 * intervals
        off += 8
        c = int(np.frombuffer(raw, np.uint64, 1, off)[0]); off += 8
        out.append((lv.copy(), np.frombuffer(raw, np.uint64, c, off).copy())); off += 8 * c
    return out


@pytest.fixture(scope="module")
def index(tb, wl, tmp_path_factory, cuda):
    if not (os.path.exists(REF) and os.path.exists(DROP_IN)):
        pytest.skip("reference build not present (make -C oracle ref needs the reference sources)")
    d = tmp_path_factory.mktemp("dropin")
    h = tb.QueryHandler.generate(300000, 5, 1.0, 100.0, False, 4, (60, 30, 15), 77, 2.2)
    idx = str(d / "idx")
    h.save_index(idx)
    Q = wl.range_boxes(h, 40, seed=5, half_width=0.05)
    P = wl.knn_points(h, 20, seed=6, noise=0.01)
    # The reference derives a label from the query file's name (the text after the last '_' of the
    # whole path, src/utils/Utils.cu:18-35) and aborts when that text holds a '-' that is not
    # "<int>-<int>": name the files so that it reads "range" / "knn".
    fq, fp = str(d / "q_range.txt"), str(d / "q_knn.txt")
    tb.save_query_file(fq, tb.QueryType.RANGE, Q, 5)
    tb.save_query_file(fp, tb.QueryType.POINT, P, 5)
    return d, idx, fq, fp, Q, P


@pytest.mark.parametrize("kind", ["range", "knn"])
def test_reference_engine_drives_the_b200_library(index, kind):
    d, idx, fq, fp, Q, P = index
    qf, t, K = (fq, "0", "0") if kind == "range" else (fp, "1", "10")
    a, b = str(d / f"ref_{kind}.bin"), str(d / f"b200_{kind}.bin")
    subprocess.run([REF, idx, qf, t, K, "L0", a], check=True, timeout=600, stdout=subprocess.DEVNULL)
    subprocess.run([DROP_IN, idx, qf, t, K, "L0", b], check=True, timeout=600, stdout=subprocess.DEVNULL)
    ref, got = _read(a), _read(b)
    assert len(ref) == len(got) == (40 if kind == "range" else 20)
    for q, ((lr, ir), (lg, ig)) in enumerate(zip(ref, got)):
        assert np.array_equal(lr, lg), q
        assert np.array_equal(ir, ig), q
    assert int(open(b + ".levels").read()) == len(ref) * 3  # every level of every query ran in the library
    assert sum(len(i) for _, i in ref) > 1000


def test_cpp_facade_is_the_reference_query_api(index, oracle_mod, tmp_path):
    d, idx, fq, fp, Q, P = index
    exe = str(tmp_path / "facade_check")
    csrc = os.path.join(REPO, "t-blaeq_b200", "csrc")
    lib_dir = os.path.join(REPO, "t-blaeq_b200")
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-x", "cu", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", csrc, "-I", os.path.join(REPO, "include"), os.path.join(REPO, "tests", "cpp", "facade_check.cpp"),
                    "-o", exe, "-L", lib_dir, "-l:libtblaeq_b200.so", "-Xlinker", "-rpath=" + lib_dir],
                   check=True, timeout=600)
    o = oracle_mod.load_index(idx)
    pts, ids = oracle_mod.decoded_points(o)
    for kind, qf, t, K, rows in (("range", fq, "0", 0, Q), ("knn", fp, "1", 10, P)):
        out = str(tmp_path / f"{kind}.txt")
        subprocess.run([exe, idx, qf, t, str(K), out], check=True, timeout=600)
        lines = [ln.split("|") for ln in open(out)]
        ref = _read(str(d / f"ref_{kind}.bin")) if os.path.exists(str(d / f"ref_{kind}.bin")) else None
        if ref is None:
            a = str(tmp_path / f"ref_{kind}.bin")
            subprocess.run([REF, idx, qf, t, str(K), "L0", a], check=True, timeout=600, stdout=subprocess.DEVNULL)
            ref = _read(a)
        brute = oracle_mod.brute_query(pts, ids, oracle_mod.RANGE if kind == "range" else oracle_mod.KNN, rows, K=K)
        n = len(rows)
        assert len(lines) == 2 * n
        for head, tail in lines:
            mode, q, *lv = (int(x) for x in head.split())
            got = np.array([int(x) for x in tail.split()], np.uint64)
            if mode == 0:  # ref-parity: the reference's candidate set and level sizes
                assert np.array_equal(np.sort(got), ref[q][1]), (kind, q)
                assert np.array_equal(np.array(lv, np.uint64), ref[q][0]), (kind, q)
            else:          # exact: the FP64 brute force
                want = brute.query(q)
                assert np.array_equal(np.sort(got) if kind == "range" else got, want), (kind, q)
