"""clb_dcsr_spgemm_to_host: C = A*B delivered into host arrays in row blocks
(the copy of one block overlapped with the product of the next).  The
result must be the oracle's product whatever the block count, for the
learned form and the tuned (exact) form."""
import numpy as np
import pytest

import oracle as O
from util import pairs_dcsr, to_device


def _rmat(scale):
    from clbool_b200 import gen
    r, c = gen.rmat(scale, seed=scale)
    n = 1 << scale
    return O.coo_to_dcsr(O.Coo(n, n, r, c))


def _run(controls, a, b, sizer, blocks, rows_cap=None, cols_cap=None):
    from clbool_b200 import sizing
    want = O.spgemm(a, b)
    rows_cap = len(want.rows) if rows_cap is None else rows_cap
    cols_cap = len(want.cols) if cols_cap is None else cols_cap
    h_rpt = np.zeros(rows_cap + 1, np.uint64)
    h_rows = np.zeros(max(rows_cap, 1), np.uint32)
    h_cols = np.zeros(max(cols_cap, 1), np.uint32)
    st = {}
    nzr, nnz = sizing.matrix_multiplication_to_host(controls, to_device(controls, a), to_device(controls, b), h_rpt,
                                                    h_rows, h_cols, rows_cap, cols_cap, sizer=sizer, blocks=blocks,
                                                    stats=st)
    return want, nzr, nnz, h_rpt, h_rows, h_cols, st


@pytest.mark.gpu
@pytest.mark.parametrize("blocks", [1, 3, 8])
@pytest.mark.parametrize("learned", [True, False])
def test_to_host_matches_oracle(controls, blocks, learned):
    from clbool_b200 import sizing
    sizer = sizing.RowSizer.load(controls) if learned else None
    for a, b, what in ((_rmat(12), None, "rmat12"), (pairs_dcsr(2000, 30), None, "pairs2000")):
        b = a if b is None else b
        want, nzr, nnz, h_rpt, h_rows, h_cols, st = _run(controls, a, b, sizer, blocks)
        assert (nzr, nnz) == (len(want.rows), len(want.cols)), what
        assert np.array_equal(h_rpt[:nzr + 1], np.asarray(want.rpt, np.uint64)), what
        assert np.array_equal(h_rows[:nzr], want.rows), what
        assert np.array_equal(h_cols[:nnz], want.cols), what
        assert st["products"] == int(O.workload(a, b).astype(np.int64).sum()), what


@pytest.mark.gpu
def test_to_host_small_arrays_and_empty(controls):
    import clbool_b200 as cb
    from clbool_b200 import ClBoolException
    a = _rmat(10)
    with pytest.raises(ClBoolException, match="host arrays too small"):
        _run(controls, a, a, None, 4, cols_cap=10)
    z = O.Dcsr(64, 64, np.zeros(1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    want, nzr, nnz, h_rpt, _, _, _ = _run(controls, z, pairs_dcsr(64, 3), None, 4)
    assert (nzr, nnz) == (0, 0) and h_rpt[0] == 0
