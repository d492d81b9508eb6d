"""The allocation-free per-level range step (tblaeq_level_range_noalloc) against tblaeq_level.

Callers that cannot allocate device memory while they query -- a process that reserved its whole
memory budget at start-up, or one whose rules forbid allocation between start-up and shutdown --
use tblaeq_level_range_noalloc: it writes into buffers the caller owns and keeps its scratch in a
fixed device array. Its results must equal the allocating entry point's, bit for bit (ids in the
reference's order and the rebuilt coordinates), on consecutive calls, because every call reuses the
same scratch array. This file is collected last so a failure here leaves every other test run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

D = 5
MAX_GRID = 16384


@pytest.fixture(scope="module")
def env(tb, cuda):
    import torch
    h = tb.QueryHandler.generate(200000, D, 1.0, 100.0, False, 4, (40, 20, 10), 23, 2.2)
    h.prepare_for_query(tb.LevelPolicy.L0)
    lib = tb.lib()
    lib.tblaeq_level_range_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(tb.Grid),
                                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                               ctypes.POINTER(ctypes.c_uint64)]
    lib.tblaeq_level_range_noalloc.restype = ctypes.c_int
    cap = 1 << 18
    out_ids = torch.empty(cap, dtype=torch.int64, device="cuda")
    out_vals = torch.empty(cap * D, dtype=torch.float64, device="cuda")
    return h, lib, out_ids, out_vals, cap


def _noalloc(tb, h, lib, l, grid, lo, hi, out_ids, out_vals, cap):
    n = ctypes.c_uint64()
    lo = np.ascontiguousarray(lo, dtype=np.float64)
    hi = np.ascontiguousarray(hi, dtype=np.float64)
    code = lib.tblaeq_level_range_noalloc(h._h, l, ctypes.byref(grid), lo.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          hi.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out_ids.data_ptr(),
                                          out_vals.data_ptr(), cap, ctypes.byref(n))
    return code, int(n.value)


def _boxes(h, n, seed):
    rng = np.random.default_rng(seed)
    pts, _ = h.decode_points(rng.integers(0, 200000, n))
    hw = rng.uniform(2.0, 12.0, (n, D))
    return pts - hw, pts + hw


def test_noalloc_matches_level_step_on_consecutive_calls(tb, env):
    h, lib, out_ids, out_vals, cap = env
    los, his = _boxes(h, 3, 1)
    calls = 0
    for q in range(3):  # several queries in a row: every call reuses the same scratch array
        grid = h.coarsest_grid()
        for l in range(3):
            if grid.nnz > MAX_GRID:
                break
            code, n = _noalloc(tb, h, lib, l, grid, los[q], his[q], out_ids, out_vals, cap)
            assert code == 0, lib.tblaeq_last_error()
            ref = h.run_level(l, grid, tb.QueryType.RANGE, lo=los[q], hi=his[q])
            ref_ids, ref_vals = h.grid_arrays(ref)
            assert n == ref.nnz
            got_ids = out_ids[:n].cpu().numpy().astype(np.uint64)
            got_vals = out_vals[:n * D].cpu().numpy().reshape(n, D)
            assert np.array_equal(got_ids, ref_ids)      # same ids, same order
            assert np.array_equal(got_vals, ref_vals)    # bit-identical coordinates
            calls += 1
            grid = ref
    assert calls >= 4


def test_noalloc_allocates_no_device_memory(tb, env):
    """The property the entry point exists for: after one warm-up call (which looks up the scratch
    array's device address), calls allocate nothing. The library's device allocation count stays
    unchanged, and with the allocation-failure hook armed (the next allocation fails) the calls
    still succeed."""
    h, lib, out_ids, out_vals, cap = env
    los, his = _boxes(h, 4, 3)
    grid = h.coarsest_grid()
    code, _ = _noalloc(tb, h, lib, 0, grid, los[0], his[0], out_ids, out_vals, cap)
    assert code == 0, lib.tblaeq_last_error()
    live = lib.tblaeq_live_device_bytes()
    lib.tblaeq_debug_fail_alloc_after(1)
    try:
        for q in range(4):
            code, n = _noalloc(tb, h, lib, 0, grid, los[q], his[q], out_ids, out_vals, cap)
            assert code == 0, lib.tblaeq_last_error()
            assert lib.tblaeq_live_device_bytes() == live
    finally:
        lib.tblaeq_debug_fail_alloc_after(0)
    assert lib.tblaeq_live_device_bytes() == live


def test_noalloc_limits(tb, env):
    h, lib, out_ids, out_vals, cap = env
    los, his = _boxes(h, 1, 2)
    grid = h.coarsest_grid()
    big = grid
    for l in range(3):  # a box holding everything: the last grid has every point
        big = h.run_level(l, big, tb.QueryType.RANGE, lo=los[0] - 1e3, hi=his[0] + 1e3)
    assert big.nnz > MAX_GRID
    code, _ = _noalloc(tb, h, lib, 2, big, los[0], his[0], out_ids, out_vals, cap)
    assert code == 1  # beyond the fixed grid limit: rejected before any work
    code, _ = _noalloc(tb, h, lib, 0, grid, los[0] - 1e3, his[0] + 1e3, out_ids, out_vals, 4)
    assert code == 5  # output larger than the caller's buffers
    code, n = _noalloc(tb, h, lib, 0, grid, los[0], his[0], out_ids, out_vals, cap)
    assert code == 0 and n > 0  # and the next call is clean again


def test_noalloc_timeout_then_clean_call(tb, env):
    """A look-back wait that runs out inside the allocation-free step (test hook: one work tile
    never publishes) fails the call with TBLAEQ_ERR_TIMEOUT; the next call clears the shared
    array's control words and matches tblaeq_level again."""
    h, lib, out_ids, out_vals, cap = env
    los, his = _boxes(h, 1, 5)
    lo, hi = los[0] - 1e3, his[0] + 1e3  # every cluster survives
    grid = h.run_level(0, h.coarsest_grid(), tb.QueryType.RANGE, lo=lo, hi=hi)  # 250 nodes of mesh 1
    lib.tblaeq_debug_lookback_timeout(1, 2000)
    try:
        code, _ = _noalloc(tb, h, lib, 1, grid, lo, hi, out_ids, out_vals, cap)  # 5,000 children
        assert code == 6, lib.tblaeq_last_error()
    finally:
        lib.tblaeq_debug_lookback_timeout(2**64 - 1, 0)
    code, n = _noalloc(tb, h, lib, 1, grid, lo, hi, out_ids, out_vals, cap)
    assert code == 0, lib.tblaeq_last_error()
    ref = h.run_level(1, grid, tb.QueryType.RANGE, lo=lo, hi=hi)
    ref_ids, ref_vals = h.grid_arrays(ref)
    assert n == ref.nnz > 256
    assert np.array_equal(out_ids[:n].cpu().numpy().astype(np.uint64), ref_ids)
    assert np.array_equal(out_vals[:n * D].cpu().numpy().reshape(n, D), ref_vals)
