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
