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


OPERATIONS = ["clb_dcsr_spgemm_hash", "clb_dcsr_spgemm_esc", "clb_dcsr_spgemm_learned", "clb_dcsr_spgemm_tuned",
              "clb_dcsr_spgemm_batched", "clb_dcsr_spgemm_to_host", "clb_spgemm_batched_plan", "clb_spgemm_autotune",
              "clb_dcsr_workload", "clb_coo_add", "clb_csr_add", "clb_dcsr_kronecker", "clb_dcsr_transpose",
              "clb_dcsr_submatrix", "clb_dcsr_reduce", "clb_coo_sort", "clb_coo_to_dcsr", "clb_dcsr_to_coo",
              "clb_dcsr_to_csr", "clb_csr_to_dcsr", "clb_prefix_sum_u32"]


def _signature(name):
    src = "".join(open(h).read() for h in glob.glob(os.path.join(ROOT, "include", "*.h")))
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    m = re.search(r"CLB_API\s+int\s+" + name + r"\s*\(([^)]*)\)\s*;", src)
    assert m, name
    return [" ".join(p.split()) for p in m.group(1).split(",")]


def _null_args(params):
    """NULL for every pointer, zero for every scalar, typed as declared."""
    types, values = [], []
    for p in params:
        if "*" in p:
            types.append(ctypes.c_void_p)
            values.append(None)
            continue
        t = p.rsplit(" ", 1)[0].replace("const ", "")
        ct = {"uint64_t": ctypes.c_uint64, "uint32_t": ctypes.c_uint32, "int": ctypes.c_int,
              "float": ctypes.c_float, "double": ctypes.c_double}[t]
        types.append(ct)
        values.append(ct(0))
    return types, values


@pytest.mark.parametrize("name", OPERATIONS)
def test_operations_reject_null_arguments(name):
    """Every operation checks its arguments on the host before any device
    work: NULL controls or matrices give CLBOOL_INVALID_ARGUMENT (the status
    the reference raises for bad arguments, src/core/error.hpp:130-151) and a
    message, never a crash (no GPU needed)."""
    import clbool_b200 as cb
    lib = ctypes.CDLL(cb.LIB_PATH)
    fn = getattr(lib, name)
    types, values = _null_args(_signature(name))
    fn.argtypes = types
    fn.restype = ctypes.c_int
    assert fn(*values) == 12, name  # CLBOOL_INVALID_ARGUMENT
    lib.clb_last_error.restype = ctypes.c_char_p
    assert lib.clb_last_error().decode(), name
