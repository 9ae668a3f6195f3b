"""Primitives on the GPU vs the oracle and the golden vectors: prefix_sum
(test_procedures.cpp:9-14), coo::sort_arrays (test_procedures.cpp:2-7), the
matrix_coo dedupe constructor (test_procedures.cpp:20-31) and the
DCSR <-> CSR <-> COO conversions (test/test_conversions.cpp)."""
import numpy as np
import pytest

import oracle as O
from util import dcsr_digest, from_device, golden, pairs_dcsr, sha, to_device

pytestmark = pytest.mark.gpu
G = golden()


def test_prefix_sum_vectors(controls):
    import clbool_b200 as cb
    for case in G["prefix_sum"]:
        v = O.fill_random_buffer(case["n"], 3)
        buf = cb.DeviceBuffer.from_host(controls, v, np.uint32)
        total = cb.prefix_sum(controls, buf, case["n"])
        assert total == case["total"]
        assert sha(buf.to_host(), np.uint32) == case["scan"]


@pytest.mark.parametrize("n", [1, 2, 4095, 4096, 4097, 8193, 1_000_003])
def test_prefix_sum_sizes_u64(controls, n):
    import clbool_b200 as cb
    rng = np.random.default_rng(n)
    v = rng.integers(0, 1 << 40, size=n, dtype=np.uint64)
    buf = cb.DeviceBuffer.from_host(controls, v, np.uint64)
    total = cb.prefix_sum(controls, buf, n)
    ref = np.concatenate([np.zeros(1, np.uint64), np.cumsum(v, dtype=np.uint64)[:-1]])
    assert total == int(v.sum(dtype=np.uint64))
    assert np.array_equal(buf.to_host(), ref)


@pytest.mark.parametrize("n,offset", [(4097, 0), (8192, 0), (8193, 0), (8193, 2), (12_289, 1), (16_384, 0),
                                      (1_000_003, 0), (1_000_003, 3), ((1 << 26) + 5, 0), ((1 << 26) + 5, 1)])
def test_prefix_sum_u32_tiles(controls, n, offset):
    """u32 scans in place through the C ABI around the 8192-entry tile
    (one tile, one tile plus one entry, ragged last tiles), on arrays that do
    not start on a 16-byte boundary (element loads instead of vectors), with
    entries up to 2^32 - 1 (the scan wraps modulo 2^32 like the reference's
    u32 output; the returned total is the exact 64-bit sum)."""
    import ctypes

    import clbool_b200 as cb
    rng = np.random.default_rng(n + offset)
    v = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    pad = np.full(offset, 7, np.uint32)
    buf = cb.DeviceBuffer.from_host(controls, np.concatenate([pad, v, pad]), np.uint32)
    tot = ctypes.c_uint64()
    rc = cb.lib.clb_prefix_sum_u32(controls.handle, ctypes.c_void_p(buf.ptr + 4 * offset), n, ctypes.byref(tot))
    assert rc == 0, cb.lib.clb_last_error()
    inc = np.cumsum(v, dtype=np.uint64)
    assert tot.value == int(inc[-1])
    got = buf.to_host()
    assert np.array_equal(got[:offset], pad) and np.array_equal(got[offset + n:], pad)
    want = np.concatenate([np.zeros(1, np.uint64), inc[:-1]]).astype(np.uint32)
    assert np.array_equal(got[offset:offset + n], want)


def test_bitonic_sort_vectors(controls):
    import clbool_b200 as cb
    for case in G["bitonic_sort"]:
        r, c = O.fill_random_matrix(case["n"])
        rb = cb.DeviceBuffer.from_host(controls, r, np.uint32)
        cbuf = cb.DeviceBuffer.from_host(controls, c, np.uint32)
        cb.coo.sort_arrays(controls, rb, cbuf, case["n"])
        assert sha(rb.to_host(), np.uint32) == case["rows"] and sha(cbuf.to_host(), np.uint32) == case["cols"]


def test_sort_grid_like_reference(controls):
    """test_procedures.cpp:2-7: sizes 0..4985 step 15 against std::sort."""
    import clbool_b200 as cb
    for n in range(15, 4986, 15 * 37):
        r, c = O.fill_random_matrix(n)
        rb = cb.DeviceBuffer.from_host(controls, r, np.uint32)
        cbuf = cb.DeviceBuffer.from_host(controls, c, np.uint32)
        cb.coo.sort_arrays(controls, rb, cbuf, n)
        wr, wc = O.sort_pairs(r, c)
        assert np.array_equal(rb.to_host(), wr) and np.array_equal(cbuf.to_host(), wc), n


@pytest.mark.parametrize("n,hi", [(10_374_663, 1043), (3_000_000, 1 << 31), (100_000, 1 << 32)])
def test_sort_large_and_wide(controls, n, hi):
    import clbool_b200 as cb
    rng = np.random.default_rng(n)
    r = rng.integers(0, hi, size=n, dtype=np.uint64).astype(np.uint32)
    c = rng.integers(0, hi, size=n, dtype=np.uint64).astype(np.uint32)
    rb = cb.DeviceBuffer.from_host(controls, r, np.uint32)
    cbuf = cb.DeviceBuffer.from_host(controls, c, np.uint32)
    cb.coo.sort_arrays(controls, rb, cbuf, n)
    key = np.sort((r.astype(np.uint64) << np.uint64(32)) | c)
    assert np.array_equal(rb.to_host(), (key >> np.uint64(32)).astype(np.uint32))
    assert np.array_equal(cbuf.to_host(), (key & np.uint64(0xFFFFFFFF)).astype(np.uint32))


def test_coo_constructor_dedupe(controls):
    import clbool_b200 as cb
    g = G["coo_constructor"]
    m = cb.matrix_coo.from_host(controls, g["rows"], g["cols"], g["n"], g["n"], len(g["rows"]), True, False)
    assert m.nnz() == len(g["rows"]) - 2 == g["nnz_after"]
    h = cb.matrix_coo_from_gpu(controls, m)
    assert h.rows.tolist() == g["out_rows"] and h.cols.tolist() == g["out_cols"]


def test_coo_constructor_unsorted_with_duplicates(controls):
    import clbool_b200 as cb
    r, c = O.fill_random_matrix(200_000, 700)
    m = cb.matrix_coo.from_host(controls, r, c, 700, 700, len(r), sorted=False, noDuplicates=False)
    wr, wc = O.unique_pairs(*O.sort_pairs(r, c))
    h = cb.matrix_coo_from_gpu(controls, m)
    assert np.array_equal(h.rows, wr) and np.array_equal(h.cols, wc)


@pytest.mark.parametrize("size,k", [(0, 0), (1, 5), (200, 3), (3000, 29), (29300, 60)])
def test_dcsr_csr_roundtrips(controls, size, k):
    """test/src/conversions.cpp:49-84: DCSR->CSR equals CSR built on the host
    and CSR->DCSR equals DCSR built on the host."""
    import clbool_b200 as cb
    a = pairs_dcsr(size, k)
    A = to_device(controls, a)
    csr = cb.dcsr_to_csr(controls, A)
    want = O.dcsr_to_csr(a)
    h = cb.matrix_csr_from_gpu(controls, csr)
    if len(a.cols):
        assert np.array_equal(h.rpt, want.rpt) and np.array_equal(h.cols, want.cols)
        assert csr.cols_gpu() is A.cols_gpu()  # shallow for cols
    back = cb.csr_to_dcsr(controls, csr)
    assert dcsr_digest(from_device(controls, back)) == dcsr_digest(a)
    coo = cb.dcsr_to_coo_deep(controls, A)
    hc = cb.matrix_coo_from_gpu(controls, coo)
    oc = O.dcsr_to_coo(a)
    assert np.array_equal(hc.rows, oc.rows) and np.array_equal(hc.cols, oc.cols)
    d2 = cb.coo_to_dcsr_shallow(controls, coo)
    assert dcsr_digest(from_device(controls, d2)) == dcsr_digest(a)


def test_dcsr_to_csr_rejects_rows_past_nrows(controls):
    """A stored row index >= nrows cannot be kept by a CSR of nrows rows;
    the reference raises CLBOOL_INVALID_VALUE (matrices_conversions.cpp:268)."""
    import clbool_b200 as cb
    a = O.coo_to_dcsr(O.Coo(5, 5, np.array([1, 1, 5], np.uint32), np.array([0, 4, 2], np.uint32)))
    with pytest.raises(cb.ClBoolException) as e:
        cb.dcsr_to_csr(controls, to_device(controls, a))
    assert e.value.status_name == "CLBOOL_INVALID_VALUE"


def test_workload_matches_oracle(controls):
    import clbool_b200 as cb
    a = pairs_dcsr(3000, 40)
    buf, total = cb.dcsr.workload(controls, to_device(controls, a), to_device(controls, a))
    want = O.workload(a, a)
    assert total == int(want.sum())
    assert np.array_equal(buf.to_host(len(a.rows)).astype(np.uint64), want)

