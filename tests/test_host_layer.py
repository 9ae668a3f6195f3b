"""The C++ host layer (include/clbool/clbool.hpp) used the way the reference's
own example test uses clbool.hpp (test/test_operations.cpp:279-319): the
compiled check program must run clean on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "clbool_b200", "cpp", "host_layer_check")


@pytest.mark.gpu
def test_cpp_host_layer(tmp_path):
    if not os.path.exists(BIN):
        subprocess.run(["make", "-s", "-C", os.path.dirname(BIN)], check=True)
    path = os.path.join(tmp_path, "readme_a.dcsr")
    r = subprocess.run([BIN, path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "host layer OK" in r.stdout
    # the file the C++ layer wrote reads back in Python (same format and checksum)
    from clbool_b200 import io
    nrows, ncols, rpt, rows, cols = io.load(path)
    assert (nrows, ncols) == (5, 5)
    assert rpt.tolist() == [0, 3, 5, 6] and rows.tolist() == [0, 2, 4] and cols.tolist() == [0, 1, 4, 2, 3, 2]


def test_cpp_host_layer_compiles():
    """No GPU needed: the header-only layer compiles against the C ABI."""
    r = subprocess.run(["make", "-s", "-C", os.path.dirname(BIN)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
