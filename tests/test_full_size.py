"""The headline workload at its full size: R-MAT scale 20 (edge factor 16,
a/b/c/d = .57/.19/.19/.05, seed 1), C = A*A -- 2.09e10 products and 9.7e9
output columns, beyond what the oracle computes in a test -- and its second
operation, the CSR addition C + A.  The forms are checked through
properties that hold at any size:
  * the learned single pass, the ESC single pass and the exact two-pass form
    (dcsr::matrix_multiplication_hash, src/dcsr/dcsr.hpp:32-36) give
    bit-identical C, compared on the device;
  * C's row lengths equal the symbolic pass's counts (clb_dcsr_row_nnz);
  * every row of C is strictly increasing (sorted, no duplicates);
  * 640 seeded rows of A against the full right operand equal the oracle's
    rows of the product: 512 drawn in proportion to their products (the
    bitmap rows carry 98.7% of them) and 128 uniformly;
  * C + A (csr::matrix_addition, src/csr/csr_addition.cpp:26-168): every
    row strictly increasing, nnz(C + A) >= nnz(C), and the same 640 rows
    equal the oracle's union of the rows of C and A.
Device memory: C is 39 GB; the peak (two-pass C held while the ESC form
runs with its upper-bound slots) is about 160 GB of the B200's 180 GB."""
import ctypes

import numpy as np
import pytest

import oracle as O
from util import assert_rows_match, rows_strictly_increasing, same_on_device, sub_rows, weighted_pick

SCALE = 20


@pytest.fixture(scope="module")
def rmat20():
    from clbool_b200 import gen
    r, c = gen.rmat(SCALE, seed=1)  # sorted, duplicate-free
    n = 1 << SCALE
    return O.coo_to_dcsr(O.Coo(n, n, r, c))


@pytest.fixture(scope="module")
def sample20(rmat20):
    """640 stored rows of A (512 by products, 128 uniform) and the oracle's
    rows of A*A for them."""
    a = rmat20
    pick = weighted_pick(O.workload(a, a), 512, seed=11, uniform=128)
    sa = sub_rows(a, pick)
    return sa, O.spgemm(sa, a)


@pytest.mark.gpu
def test_rmat20_forms_identical_and_sound(controls, rmat20, sample20):
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
    same_on_device(C1, C2, "learned vs two-pass")
    del C1
    C3 = cb.dcsr.matrix_multiplication(controls, None, A, A)
    controls.sync()
    same_on_device(C3, C2, "ESC vs two-pass")
    del C3
    C4 = cb.dcsr.matrix_multiplication_tuned(controls, None, A, A, cb.dcsr.tuning("two_pass_kept"))
    controls.sync()
    same_on_device(C4, C2, "two-pass keeping its bitmaps vs two-pass")
    del C4

    # row lengths = the symbolic counts
    rpt = C2.rpt_gpu().to_host(C2.nzr() + 1).astype(np.int64)
    crows = C2.rows_gpu().to_host(C2.nzr())
    sym = sizing.row_nnz(controls, A, A).to_host(len(a.rows)).astype(np.int64)
    lens = np.zeros(len(a.rows), np.int64)
    pos = np.searchsorted(a.rows, crows)
    assert np.array_equal(a.rows[pos], crows)
    lens[pos] = np.diff(rpt)
    assert np.array_equal(lens, sym)

    rows_strictly_increasing(C2, rpt, "C = A*A")
    # the sampled rows against the oracle (heavy rows weighted in)
    _, want = sample20
    assert_rows_match(controls, C2, want, "C = A*A")


@pytest.mark.gpu
def test_rmat20_csr_addition_c_plus_a(controls, rmat20, sample20):
    import clbool_b200 as cb
    from clbool_b200 import sizing
    from util import to_device

    a = rmat20
    n = a.nrows
    A = to_device(controls, a)
    C = sizing.matrix_multiplication_learned(controls, None, A, A, sizing.RowSizer.load(controls))
    Cc, Ac = cb.dcsr_to_csr(controls, C), cb.dcsr_to_csr(controls, A)
    nnz_c = C.nnz()
    del C
    S = cb.csr.matrix_addition(controls, None, Cc, Ac)
    controls.sync()
    assert S.nnz() >= nnz_c and S.nnz() <= nnz_c + len(a.cols)
    srpt = S.rpt_gpu().to_host(n + 1).astype(np.int64)
    rows_strictly_increasing(S, srpt, "C + A")

    # sampled rows: the oracle's union of the row of A*A and the row of A
    sa, want_c = sample20
    want = O.csr_add(O.dcsr_to_csr(want_c), O.dcsr_to_csr(sa))
    lib = cb.lib
    for r in sa.rows:
        lo, hi = int(srpt[r]), int(srpt[r + 1])
        seg = np.empty(hi - lo, np.uint32)
        assert lib.clb_memcpy_d2h(controls.handle, seg.ctypes.data_as(ctypes.c_void_p),
                                  ctypes.c_void_p(S.cols_gpu().ptr + 4 * lo), 4 * (hi - lo)) == 0
        assert np.array_equal(seg, want.cols[int(want.rpt[r]):int(want.rpt[r + 1])]), f"C + A row {r}"
