"""bench.py's reader of the reference harness dump and the reference CLI's mean, on the CPU."""
import numpy as np
import pytest

import bench


def _dump(queries, intervals=3):
    """A dump in the harness layout: per query level sizes, microseconds, candidate ids."""
    parts = [np.array([len(queries), intervals], np.uint64).tobytes()]
    for us, ids in queries:
        parts.append(np.arange(intervals, dtype=np.uint64).tobytes())
        parts.append(np.array([us], np.float64).tobytes())
        parts.append(np.array([len(ids)], np.uint64).tobytes())
        parts.append(np.asarray(ids, np.uint64).tobytes())
    return b"".join(parts)


def test_reads_times_and_candidates():
    raw = _dump([(120.5, [3, 1, 2]), (80.0, []), (400.0, [7]), (100.0, [9, 8])])
    us, cands = bench.read_harness_times(raw)
    assert us == [120.5, 80.0, 400.0, 100.0] and cands == 6
    # The reference CLI drops the fastest and the slowest query: mean of 100 and 120.5.
    assert bench.reference_mean_us(us) == pytest.approx(110.25)
    assert bench.reference_mean_us([5.0, 7.0]) == pytest.approx(6.0)


def test_rejects_a_truncated_dump():
    raw = _dump([(1.0, [1, 2, 3])])
    with pytest.raises(ValueError):
        bench.read_harness_times(raw[:-8])


def test_reference_arm_draws_the_same_workload(tb, wl, oracle_mod, tmp_path):
    """The reference arm reads its index with the oracle's reader and draws boxes and points from the
    oracle's decoded coordinates; they must be the product arm's inputs exactly."""
    h = tb.QueryHandler.generate(30000, 8, 1.0, 100.0, False, 4, (20, 10, 5), 1, 3.0)
    d = str(tmp_path / "idx")
    h.save_index(d)
    view = bench.OracleWorkloadView(oracle_mod, oracle_mod.load_index(d))
    assert view.info()["N"] == 30000 and view.info()["D"] == 8
    a = wl.range_boxes(view, 64, seed=42, log_uniform=(0.001, 0.1))
    b = wl.range_boxes(h, 64, seed=42, log_uniform=(0.001, 0.1))
    assert np.array_equal(a, b)
    assert np.array_equal(wl.knn_points(view, 32, seed=1234, noise=0.02), wl.knn_points(h, 32, seed=1234, noise=0.02))


def test_query_file_writer_matches_the_package(tb, tmp_path):
    rows = np.random.default_rng(0).uniform(-5, 5, (7, 6))
    bench.write_query_file(str(tmp_path / "a.txt"), rows, 3)
    tb.save_query_file(str(tmp_path / "b.txt"), tb.QueryType.RANGE, rows, 3)
    assert open(tmp_path / "a.txt").read() == open(tmp_path / "b.txt").read()


def test_knn_workload_mix():
    k = bench.knn_k(6)
    assert k.tolist() == [20, 100, 20, 100, 20, 100] and k.dtype == np.uint32
