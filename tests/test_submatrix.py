"""dcsr::submatrix and dcsr::reduce on the GPU vs the oracle and the golden
vectors recorded from the reference (test_operations.cpp:52-106,
operations.cpp:84-166; README example test_operations.cpp:309-310)."""
import numpy as np
import pytest

import oracle as O
from util import assert_dcsr_equal, dcsr_digest, from_device, golden, pairs_dcsr, to_device

pytestmark = pytest.mark.gpu
G = golden()


def sub(ctl, a, i, j, nr, nc):
    import clbool_b200 as cb
    return from_device(ctl, cb.dcsr.submatrix(ctl, None, to_device(ctl, a), i, j, nr, nc))


def red(ctl, a):
    import clbool_b200 as cb
    return from_device(ctl, cb.dcsr.reduce(ctl, None, to_device(ctl, a)))


def test_readme_example(controls):
    g = G["readme"]
    a = O.coo_to_dcsr(O.Coo(5, 5, np.array(g["a"]["rows"], np.uint32), np.array(g["a"]["cols"], np.uint32)))
    r = red(controls, a)
    assert r.rows.tolist() == g["reduce"]["rows"] and r.cols.tolist() == g["reduce"]["cols"]
    assert r.rpt.tolist() == g["reduce"]["rpt"] and r.ncols == 1
    s = sub(controls, a, 0, 2, 3, 2)
    assert s.rpt.tolist() == g["submatrix_0_2_3_2"]["rpt"] and s.rows.tolist() == g["submatrix_0_2_3_2"]["rows"]
    assert s.cols.tolist() == g["submatrix_0_2_3_2"]["cols"] and (s.nrows, s.ncols) == (3, 2)


@pytest.mark.parametrize("case", G["submatrix_reduce"], ids=lambda c: f"s{c['size']}k{c['k']}")
def test_golden_grid(controls, case):
    a = pairs_dcsr(case["size"], case["k"])
    s = sub(controls, a, case["i"], case["j"], case["nrows"], case["ncols"])
    assert dcsr_digest(s) == case["submatrix"]
    assert dcsr_digest(red(controls, a)) == case["reduce"]


def test_random_ranges(controls):
    rng = np.random.default_rng(77)
    for size, k in ((997, 11), (3000, 40), (20000, 60)):
        a = pairs_dcsr(size, k)
        for _ in range(6):
            i1, i2, i3, i4 = (int(x) for x in rng.integers(0, size + 1, 4))
            i, nr, j, nc = min(i1, i2), abs(i1 - i2), min(i3, i4), abs(i3 - i4)
            assert_dcsr_equal(sub(controls, a, i, j, nr, nc), O.submatrix(a, i, j, nr, nc), f"{size} {i} {j}")


def test_edge_cases(controls):
    import clbool_b200 as cb
    a = pairs_dcsr(500, 8)
    # whole matrix, empty ranges, ranges past the end, wide keys
    assert_dcsr_equal(sub(controls, a, 0, 0, 500, 500), a, "whole")
    for i, j, nr, nc in ((0, 0, 0, 10), (0, 0, 10, 0), (600, 0, 50, 50), (0, 600, 50, 50),
                         (490, 490, 1 << 33, 1 << 33), (0, 0, 1, 1)):
        s = sub(controls, a, i, j, nr, nc)
        assert_dcsr_equal(s, O.submatrix(a, i, j, nr, nc), f"{i} {j} {nr} {nc}")
        assert (s.nrows, s.ncols) == (nr, nc)
    z = O.coo_to_dcsr(O.Coo(40, 40, np.zeros(0, np.uint32), np.zeros(0, np.uint32)))
    assert len(sub(controls, z, 0, 0, 10, 10).cols) == 0
    r = red(controls, z)
    assert len(r.cols) == 0 and (r.nrows, r.ncols) == (40, 1)
    # output aliasing the input, as dcsr_reduce.cpp:17 allows
    A = to_device(controls, a)
    cb.dcsr.reduce(controls, A, A)
    assert_dcsr_equal(from_device(controls, A), O.reduce(a), "reduce in place")
    with pytest.raises(cb.ClBoolException) as e:
        cb.dcsr.submatrix(controls, None, to_device(controls, a), 1 << 33, 0, 1, 1)
    assert e.value.status_name == "CLBOOL_INVALID_VALUE"
