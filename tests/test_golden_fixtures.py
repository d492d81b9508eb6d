"""The CPU oracle pinned against the reference's own CUDA build (CPU only).

tests/golden/ref_cuda_*.npz were written by tests/test_gpu_reference.py (TBLAEQ_GOLDEN_OUT) from
oracle/_ref/ref_harness -- the reference T-BLAEQ compiled from source, run on a B200 one query at a
time through QueryHandler::performSingle{Range,KNN}Query(saveFineMesh=true). Each fixture holds the
queries, and per query the candidate count, the SHA-256 of the sorted candidate ids and the grid size
after every level. The index is regenerated here with the B200 build's generator, whose bytes are
pinned to the reference's --gen-index by test_index_format.py.
"""
import glob
import hashlib
import os

import numpy as np
import pytest

from conftest import oracle_from_handler

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_cuda_*.npz")))


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[9:-4] for p in FIXTURES])
def test_oracle_reproduces_reference_cuda_candidates(tb, oracle_mod, tmp_path, path):
    z = np.load(path)
    N, D, r0, r1, r2, seed = (int(v) for v in z["params"])
    h = tb.QueryHandler.generate(N, D, 1.0, 100.0, False, 4, (r0, r1, r2), seed, float(z["sigma_divisor"]))
    o = oracle_from_handler(oracle_mod, h, tmp_path)
    Q = z["queries"]
    K = int(z["K"])
    qtype = oracle_mod.KNN if K > 0 else oracle_mod.RANGE
    res = oracle_mod.ref_query(o, qtype, Q, K=K)
    assert np.array_equal(np.diff(res.offsets), z["counts"])
    assert np.array_equal(res.level_sizes, z["levels"])
    for q in range(len(Q)):
        dig = np.frombuffer(hashlib.sha256(np.sort(res.query(q)).astype("<u8").tobytes()).digest(), np.uint8)
        assert np.array_equal(dig, z["digests"][q]), q
