"""The C-ABI library loads and exports every entry point declared in
include/*.h (no GPU needed: nothing here launches a kernel)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names |= set(re.findall(r"CLB_API\s+[\w\s\*]+?\b(clb_\w+)\s*\(", src))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared()
    assert "clb_dcsr_spgemm_hash" in names and len(names) > 20


def test_library_exports_every_declared_symbol():
    import clbool_b200 as cb
    lib = ctypes.CDLL(cb.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_status_strings_mirror_reference_order():
    import clbool_b200 as cb
    names = [cb.lib.clb_status_string(i).decode() for i in range(15)]
    assert names[0] == "CLBOOL_SUCCESS"
    assert names[1:] == ["CLBOOL_NO_SUCH_PROGRAM", "CLBOOL_CREATE_KERNEL_ERROR", "CLBOOL_BUILD_PROGRAM_ERROR",
                         "CLBOOL_INCOMPLETE_KERNEL", "CLBOOL_RUN_KERNEL_FAILURE", "CLBOOL_EVENT_WAITING_ERROR",
                         "CLBOOL_CREATE_BUFFER_ERROR", "CLBOOL_COPY_BUFFER_ERROR", "CLBOOL_READ_BUFFER_ERROR",
                         "CLBOOL_WRITE_BUFFER_ERROR", "CLBOOL_CREATE_CONTROLS_ERROR", "CLBOOL_INVALID_ARGUMENT",
                         "CLBOOL_INVALID_VALUE", "CLBOOL_INITIALIZATION_ERROR"]


def test_invalid_device_raises_like_reference():
    """test_errors.cpp:7-25: an invalid device id raises clbool::Exception."""
    import clbool_b200 as cb
    with pytest.raises(cb.ClBoolException) as e:
        cb.create_controls(0, 10_000)
    assert e.value.status_name == "CLBOOL_CREATE_CONTROLS_ERROR"
    with pytest.raises(cb.ClBoolException):
        cb.create_controls(7, 0)
