"""The C++ host layer (include/clbool/clbool.hpp) used the way the reference's
own example test uses clbool.hpp (test/test_operations.cpp:279-319): the
compiled check program must run clean on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "clbool_b200", "cpp", "host_layer_check")


@pytest.mark.gpu
def test_cpp_host_layer():
    if not os.path.exists(BIN):
        subprocess.run(["make", "-s", "-C", os.path.dirname(BIN)], check=True)
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "host layer OK" in r.stdout


def test_cpp_host_layer_compiles():
    """No GPU needed: the header-only layer compiles against the C ABI."""
    r = subprocess.run(["make", "-s", "-C", os.path.dirname(BIN)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
