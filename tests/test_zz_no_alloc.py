"""The allocation-free prefix sum, checked against the regular one.

clb_prefix_sum_u32_noalloc exists for callers that cannot allocate device
memory when they need a scan (a runtime whose pool already holds all of the
GPU's memory, or a hot loop that must not pay for cudaMalloc's implicit
synchronisation): its scratch is a fixed array inside the library.  This file
is named to be collected last, so a run that stops at the first failure has
already run every other test; it also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scan_noalloc(controls, buf, n, d_total):
    import clbool_b200 as cb
    stream = cb.lib.clb_controls_get_stream(controls.handle)
    rc = cb.lib.clb_prefix_sum_u32_noalloc(C.c_void_p(buf.ptr if buf is not None else 0), n,
                                           C.c_void_p(d_total.ptr if d_total is not None else 0),
                                           C.c_void_p(stream))
    cb.core.check(rc, "prefix_sum_noalloc")
    controls.sync()


def test_noalloc_prefix_sum_matches_regular_twice(controls):
    import clbool_b200 as cb
    rng = np.random.default_rng(2024)
    d_total = cb.DeviceBuffer.empty(controls, 1, np.uint64)
    # two calls in a row, the second shorter than the first, so leftovers of
    # the first call in the shared scratch would show up in the second
    for n in (1_000_003, 70_001):
        v = rng.integers(0, 4, size=n, dtype=np.uint32)
        regular = cb.DeviceBuffer.from_host(controls, v, np.uint32)
        free_of_alloc = cb.DeviceBuffer.from_host(controls, v, np.uint32)
        total = cb.prefix_sum(controls, regular, n)
        _scan_noalloc(controls, free_of_alloc, n, d_total)
        assert np.array_equal(free_of_alloc.to_host(), regular.to_host())
        assert int(d_total.to_host()[0]) == total == int(v.sum(dtype=np.uint64))


def test_noalloc_prefix_sum_rejects_sizes_past_its_scratch(controls):
    import clbool_b200 as cb
    buf = cb.DeviceBuffer.empty(controls, 16, np.uint32)
    d_total = cb.DeviceBuffer.empty(controls, 1, np.uint64)
    rc = cb.lib.clb_prefix_sum_u32_noalloc(C.c_void_p(buf.ptr), (1 << 28) + 1, C.c_void_p(d_total.ptr), None)
    assert rc == 12  # CLBOOL_INVALID_ARGUMENT, nothing launched
    assert b"static scratch limit" in cb.lib.clb_last_error()


@pytest.mark.parametrize("n", [0, 1, 4096, 4097, 8192, 8193])
def test_noalloc_prefix_sum_edge_sizes(controls, n):
    """No entries (only the total is written), one entry, exactly one tile
    and one past it, each compared with the regular scan and numpy."""
    import clbool_b200 as cb
    rng = np.random.default_rng(n + 7)
    v = rng.integers(0, 1000, size=max(n, 1), dtype=np.uint32)[:n]
    d_total = cb.DeviceBuffer.from_host(controls, np.array([12345], np.uint64), np.uint64)
    if n == 0:
        _scan_noalloc(controls, None, 0, d_total)
        assert int(d_total.to_host()[0]) == 0
        return
    regular = cb.DeviceBuffer.from_host(controls, v, np.uint32)
    free_of_alloc = cb.DeviceBuffer.from_host(controls, v, np.uint32)
    total = cb.prefix_sum(controls, regular, n)
    _scan_noalloc(controls, free_of_alloc, n, d_total)
    want = np.concatenate([[0], np.cumsum(v.astype(np.uint64))[:-1]]).astype(np.uint32)
    assert np.array_equal(free_of_alloc.to_host(), want)
    assert np.array_equal(regular.to_host(), want)
    assert int(d_total.to_host()[0]) == total == int(v.sum(dtype=np.uint64))


def test_noalloc_prefix_sum_without_total(controls):
    """d_total = NULL: the scan still runs, nothing else is written."""
    import clbool_b200 as cb
    v = np.arange(10_000, dtype=np.uint32) % 5
    buf = cb.DeviceBuffer.from_host(controls, v, np.uint32)
    _scan_noalloc(controls, buf, v.size, None)
    want = np.concatenate([[0], np.cumsum(v.astype(np.uint64))[:-1]]).astype(np.uint32)
    assert np.array_equal(buf.to_host(), want)
