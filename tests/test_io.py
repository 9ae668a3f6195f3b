"""Binary DCSR files with a checksum (clbool_b200/io.py and clbool::io in
include/clbool/clbool.hpp; the C++ side is exercised by test_host_layer)."""
import numpy as np
import pytest

from util import assert_dcsr_equal, from_device, pairs_dcsr, to_device

def test_dcsr_file_roundtrip_and_checksum(tmp_path):
    """Binary DCSR files (clbool_b200/io.py): round trip, empty matrix,
    corruption and truncation detected.  Host only."""
    from clbool_b200 import io
    a = pairs_dcsr(700, 9)
    p = str(tmp_path / "a.dcsr")
    io.save(p, a.nrows, a.ncols, a.rpt, a.rows, a.cols)
    nrows, ncols, rpt, rows, cols = io.load(p)
    assert (nrows, ncols) == (a.nrows, a.ncols)
    assert np.array_equal(rpt, a.rpt) and np.array_equal(rows, a.rows) and np.array_equal(cols, a.cols)
    e = str(tmp_path / "e.dcsr")
    io.save(e, 10, 20, np.zeros(1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    assert io.load(e)[:2] == (10, 20) and io.load(e)[4].size == 0
    raw = bytearray(open(p, "rb").read())
    raw[100] ^= 1
    bad = str(tmp_path / "bad.dcsr")
    open(bad, "wb").write(bytes(raw))
    with pytest.raises(Exception, match="checksum"):
        io.load(bad)
    open(bad, "wb").write(bytes(open(p, "rb").read()[:-40]))
    with pytest.raises(Exception):
        io.load(bad)


@pytest.mark.gpu
def test_dcsr_file_device_roundtrip(controls, tmp_path):
    from clbool_b200 import io
    a = pairs_dcsr(1200, 15)
    p = str(tmp_path / "a.dcsr")
    io.save_device(controls, p, to_device(controls, a))
    assert_dcsr_equal(from_device(controls, io.load_device(controls, p)), a, "file round trip")
