"""The C-ABI library loads and exports every entry point include/tblaeq.h declares (CPU only),
and host-side logic that needs no GPU: scheduler byte math, argument validation, query files."""
import ctypes
import os
import re

import numpy as np
import pytest


def _declared_functions(header):
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tblaeq_[a-z_0-9]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(tb):
    lib = ctypes.CDLL(tb.LIB_PATH)
    names = _declared_functions(tb.HEADER_PATH)
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version(tb):
    assert tb.lib().tblaeq_abi_version() == tb.ABI_VERSION == 3


def test_header_is_plain_c_and_links(tb, tmp_path):
    """A C caller (the reference's cgo/ctypes-style bindings see the same thing): the header compiles
    as strict C99, and a program linked against the library agrees on the ABI version."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    src = tmp_path / "abi.c"
    src.write_text('#include "tblaeq.h"\n'
                   "int main(void) { return tblaeq_abi_version() == TBLAEQ_ABI_VERSION ? 0 : 1; }\n")
    exe = tmp_path / "abi"
    lib_dir = os.path.dirname(tb.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                    "-I", os.path.dirname(tb.HEADER_PATH), str(src), "-o", str(exe),
                    "-L", lib_dir, "-l:" + os.path.basename(tb.LIB_PATH), "-Wl,-rpath," + lib_dir], check=True)
    assert subprocess.run([str(exe)]).returncode == 0


def test_null_arguments_are_rejected(tb):
    lib = tb.lib()
    assert lib.tblaeq_open(None, None) == 1
    assert lib.tblaeq_info(None, None) == 1
    assert lib.tblaeq_prepare(None, None, 0) == 1
    assert b"null" in lib.tblaeq_last_error()


def test_query_before_prepare_is_a_state_error(tb):
    h = tb.QueryHandler.generate(2000, 3, 1.0, 100.0, False, 4, (10, 10, 10), 1, 3.0)
    with pytest.raises(tb.TblaeqError) as e:
        h.query_batch(tb.QueryType.RANGE, np.zeros((1, 6)))
    assert e.value.code == 7
    with pytest.raises(tb.TblaeqError) as e:
        h.coarsest_grid()
    assert e.value.code == 7


def test_bad_policy_list(tb):
    h = tb.QueryHandler.generate(2000, 3, 1.0, 100.0, False, 4, (10, 10, 10), 1, 3.0)
    with pytest.raises(tb.TblaeqError) as e:
        h.prepare_for_query([tb.LevelPolicy.L0])
    assert e.value.code == 1


def _restated_recommend(info_sizes, D, free):
    """PolicyScheduler::recommend (src/core/MemoryPolicy.cu:100-177) restated for the test."""
    sizes = info_sizes  # finest -> coarsest
    intervals = len(sizes) - 1
    budget = int(free * 0.85)
    coarse_n = sizes[-1]
    permanent = coarse_n * 8 + coarse_n * D * 8 + sum(sizes[intervals - m] * 8 for m in range(1, intervals + 1))
    if budget <= permanent:
        return [3] * intervals
    budget -= permanent
    out = []
    for l in range(intervals):
        nnz = sizes[intervals - (l + 1)]
        col = sizes[intervals - l]
        pv, rad, sp = nnz * D * 8, col * 8, 3 * nnz * 8
        c0 = pv + rad + sp + pv
        c2 = 2 * pv + sp
        if budget >= c0:
            out.append(0)
            budget -= c0
        elif budget >= c2:
            out.append(2)
        else:
            out.append(3)
    return out


@pytest.mark.parametrize("free", [10 ** 3, 10 ** 5, 2 * 10 ** 6, 8 * 10 ** 6, 3 * 10 ** 7, 10 ** 10])
def test_scheduler_matches_reference_byte_math(tb, free):
    h = tb.QueryHandler.generate(50000, 4, 1.0, 100.0, False, 4, (10, 10, 10), 1, 3.0)
    info = h.info()
    got = [int(p) for p in h.recommend(free)]
    assert got == _restated_recommend(info["meshSizes"], info["D"], free)


def test_scheduler_degrades_level_by_level(tb):
    h = tb.QueryHandler.generate(50000, 4, 1.0, 100.0, False, 4, (10, 10, 10), 1, 3.0)
    assert [int(p) for p in h.recommend(10 ** 10)] == [0, 0, 0]
    mixed = [int(p) for p in h.recommend(5 * 10 ** 6)]
    assert mixed[0] == 0 and mixed[-1] in (2, 3)
    assert [int(p) for p in h.recommend(10)] == [3, 3, 3]


def test_query_file_roundtrip(tb, tmp_path):
    rng = np.random.default_rng(0)
    rows = rng.uniform(1, 100, (7, 10))
    p = tmp_path / "q.txt"
    tb.save_query_file(str(p), tb.QueryType.RANGE, rows, 5)
    back, _ = tb.load_query_file(str(p), tb.QueryType.RANGE)
    assert np.array_equal(back, rows)
    bad = tmp_path / "bad.txt"
    bad.write_text("2 3\n1 2 3\n")
    with pytest.raises(ValueError):
        tb.load_query_file(str(bad), tb.QueryType.RANGE)


def test_alloc_failure_hook_is_clean_on_cpu(tb):
    # Without a GPU the first device allocation happens in prepare; the hook must not leak state.
    tb.lib().tblaeq_debug_fail_alloc_after(1)
    tb.lib().tblaeq_debug_fail_alloc_after(0)
    assert tb.lib().tblaeq_live_device_bytes() == 0


def test_noalloc_rejects_a_grid_of_another_dimension(tb):
    """tblaeq_level_range_noalloc checks the grid's dimension against the index before anything
    else runs (a narrower grid would otherwise be read as nnz * D doubles): no GPU is needed."""
    h = tb.QueryHandler.generate(2000, 3, 1.0, 100.0, False, 4, (10, 10, 10), 1, 3.0)
    lib = tb.lib()
    lib.tblaeq_level_range_noalloc.restype = ctypes.c_int
    g = tb.Grid(1, 2, 1, None, None)  # dim 2 against D = 3
    lo = (ctypes.c_double * 3)(0, 0, 0)
    hi = (ctypes.c_double * 3)(1, 1, 1)
    n = ctypes.c_uint64(7)
    code = lib.tblaeq_level_range_noalloc(h._h, ctypes.c_uint64(0), ctypes.byref(g), lo, hi,
                                          None, None, ctypes.c_uint64(0), ctypes.byref(n))
    assert code == 1
    assert b"dimension mismatch" in lib.tblaeq_last_error()
    # The right dimension on an unprepared handle reaches the state check instead.
    g.dim = 3
    code = lib.tblaeq_level_range_noalloc(h._h, ctypes.c_uint64(0), ctypes.byref(g), lo, hi,
                                          None, None, ctypes.c_uint64(0), ctypes.byref(n))
    assert code == 7


def test_tuning_cache_round_trip(tb, tmp_path):
    """The autotuner's cache file: versioned, one line per key, entries added and replaced, other
    keys kept, a file of another format ignored and then replaced."""
    path = str(tmp_path / "tuning.txt")
    assert tb.tuning_lookup(path, "gpu|N=1") is None            # no file yet
    tb.tuning_store(path, "gpu|N=1", [0, 1, 0, 0], [100, 75, 50, 25])
    tb.tuning_store(path, "gpu|N=2", [1, 1, 0], [25, 25, 100])
    assert tb.tuning_lookup(path, "gpu|N=1") == ([0, 1, 0, 0], [100, 75, 50, 25])
    assert tb.tuning_lookup(path, "gpu|N=2") == ([1, 1, 0], [25, 25, 100])
    tb.tuning_store(path, "gpu|N=1", [1, 0, 0, 1], [50, 50, 50, 50])  # replaced, the other kept
    assert tb.tuning_lookup(path, "gpu|N=1") == ([1, 0, 0, 1], [50, 50, 50, 50])
    assert tb.tuning_lookup(path, "gpu|N=2") == ([1, 1, 0], [25, 25, 100])
    lines = open(path).read().splitlines()
    assert lines[0] == "tblaeq-tuning-cache 1" and len(lines) == 3
    assert tb.tuning_lookup(path, "gpu|N=3") is None
    with open(path, "w") as f:
        f.write("some-other-format 7\ngpu|N=1\t4\t0:100,0:100,0:100,0:100\n")
    assert tb.tuning_lookup(path, "gpu|N=1") is None             # another format is not read
    tb.tuning_store(path, "gpu|N=9", [0, 0], [100, 100])
    assert open(path).read().splitlines()[0] == "tblaeq-tuning-cache 1"
    with pytest.raises(tb.TblaeqError):
        tb.tuning_store(path, "bad\tkey", [0], [100])


def test_launch_counts_need_no_gpu(tb):
    """The launch counter is a process-wide count, readable before any device work; the graph's
    kernel count needs a prepared handle and rejects a null one before touching the device."""
    n = tb.kernel_launches()
    assert isinstance(n, int) and n >= 0
    assert tb.kernel_launches() == n  # nothing launched in between
    lib = tb.lib()
    k, nodes = ctypes.c_uint64(7), ctypes.c_uint64(7)
    assert tb.ERR_NAMES[lib.tblaeq_graph_launches(None, ctypes.byref(k), ctypes.byref(nodes))] == "INVALID"
    assert (k.value, nodes.value) == (7, 7)
