"""The headline workload at its full size: R-MAT scale 20 (edge factor 16,
a/b/c/d = .57/.19/.19/.05, seed 1), C = A*A -- 2.09e10 products and 9.7e9
output columns, beyond what the oracle computes in a test.  The forms are
checked through properties that hold at any size:
  * the learned single pass, the ESC single pass and the exact two-pass form
    (dcsr::matrix_multiplication_hash, src/dcsr/dcsr.hpp:32-36) give
    bit-identical C, compared on the device;
  * C's row lengths equal the symbolic pass's counts (clb_dcsr_row_nnz);
  * every row of C is strictly increasing (sorted, no duplicates);
  * 256 seeded rows of A against the full right operand equal the oracle's
    rows of the product.
Device memory: C is 39 GB; the peak (two-pass C held while the ESC form
runs with its upper-bound slots) is about 160 GB of the B200's 180 GB."""
import ctypes

import numpy as np
import pytest

import oracle as O

SCALE = 20
CHUNK = 1 << 28  # elements per device comparison


class _Cai:
    """A device array seen by torch without a copy (__cuda_array_interface__)."""

    def __init__(self, ptr: int, n: int, dtype):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": np.dtype(dtype).str,
                                         "data": (int(ptr), False), "version": 3}


def _view(buf, n, dtype):
    """Signed view (torch compares signed integers; u32 columns < 2^31 and u64
    offsets < 2^63 keep their order, and equality is bitwise either way)."""
    import torch
    signed = {np.dtype(np.uint32): np.int32, np.dtype(np.uint64): np.int64}[np.dtype(dtype)]
    return torch.as_tensor(_Cai(buf.ptr, n, signed), device="cuda")


def _same_on_device(x, y, what):
    assert (x.nnz(), x.nzr()) == (y.nnz(), y.nzr()), what
    for get, n, dt in ((lambda m: m.rpt_gpu(), x.nzr() + 1, np.uint64), (lambda m: m.rows_gpu(), x.nzr(), np.uint32),
                       (lambda m: m.cols_gpu(), x.nnz(), np.uint32)):
        a, b = _view(get(x), n, dt), _view(get(y), n, dt)
        for s in range(0, n, CHUNK):
            assert bool((a[s:s + CHUNK] == b[s:s + CHUNK]).all()), f"{what}: differs in [{s}, {s + CHUNK})"


@pytest.fixture(scope="module")
def rmat20():
    from clbool_b200 import gen
    r, c = gen.rmat(SCALE, seed=1)  # sorted, duplicate-free
    n = 1 << SCALE
    return O.coo_to_dcsr(O.Coo(n, n, r, c))


@pytest.mark.gpu
def test_rmat20_forms_identical_and_sound(controls, rmat20):
    import torch

    import clbool_b200 as cb
    from clbool_b200 import sizing
    from util import to_device

    a = rmat20
    A = to_device(controls, a)
    st = {}
    C2 = cb.dcsr.matrix_multiplication_hash(controls, None, A, A, stats=st)
    assert st["products"] == 20921347870 and C2.nnz() > 9_000_000_000, st

    sizer = sizing.RowSizer.load(controls)
    C1 = sizing.matrix_multiplication_learned(controls, None, A, A, sizer)
    controls.sync()
    _same_on_device(C1, C2, "learned vs two-pass")
    del C1
    C3 = cb.dcsr.matrix_multiplication(controls, None, A, A)
    controls.sync()
    _same_on_device(C3, C2, "ESC vs two-pass")
    del C3

    # row lengths = the symbolic counts
    rpt = C2.rpt_gpu().to_host(C2.nzr() + 1).astype(np.int64)
    crows = C2.rows_gpu().to_host(C2.nzr())
    sym = sizing.row_nnz(controls, A, A).to_host(len(a.rows)).astype(np.int64)
    lens = np.zeros(len(a.rows), np.int64)
    pos = np.searchsorted(a.rows, crows)
    assert np.array_equal(a.rows[pos], crows)
    lens[pos] = np.diff(rpt)
    assert np.array_equal(lens, sym)

    # strictly increasing inside every row: a non-increase may only sit at a row start
    cols = _view(C2.cols_gpu(), C2.nnz(), np.uint32)
    starts = torch.as_tensor(rpt[1:-1], device="cuda")
    for s in range(0, C2.nnz() - 1, CHUNK):
        e = min(s + CHUNK + 1, C2.nnz())
        bad = torch.nonzero(cols[s + 1:e] <= cols[s:e - 1]).flatten() + (s + 1)
        assert bool(torch.isin(bad, starts).all()), "a row of C is not strictly increasing"

    # 256 seeded rows against the oracle
    rng = np.random.default_rng(11)
    pick = np.sort(rng.choice(len(a.rows), 256, replace=False))
    lens_a = np.diff(a.rpt.astype(np.int64))
    sub_rpt = np.concatenate([[0], np.cumsum(lens_a[pick])]).astype(np.uint64)
    sub_cols = np.concatenate([a.cols[int(a.rpt[i]):int(a.rpt[i + 1])] for i in pick])
    want = O.spgemm(O.Dcsr(a.nrows, a.ncols, sub_rpt, a.rows[pick], sub_cols), a)
    got_rows = np.searchsorted(crows, want.rows)
    assert np.array_equal(crows[got_rows], want.rows)
    lib = cb.lib
    for k, g in enumerate(got_rows):
        lo, hi = int(rpt[g]), int(rpt[g + 1])
        seg = np.empty(hi - lo, np.uint32)
        assert lib.clb_memcpy_d2h(controls.handle, seg.ctypes.data_as(ctypes.c_void_p),
                                  ctypes.c_void_p(C2.cols_gpu().ptr + 4 * lo), 4 * (hi - lo)) == 0
        assert np.array_equal(seg, want.cols[int(want.rpt[k]):int(want.rpt[k + 1])]), f"row {want.rows[k]}"
