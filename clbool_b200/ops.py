"""Operations of the hot path over the C ABI, with the reference's names,
argument order ``(controls, matrix_out, a, b)`` and error behaviour.

Reference surface (clBool sources):
  dcsr::matrix_multiplication_hash / matrix_multiplication   src/dcsr/dcsr.hpp:27-36
  dcsr::kronecker_product / transpose                        src/dcsr/dcsr.hpp:17-21,38-41
  coo::matrix_addition                                       src/coo/coo.hpp:9-14
  csr::matrix_addition                                       src/csr/csr.hpp:12
  coo::sort_arrays                                           src/coo/coo_initialization.hpp:9
  prefix_sum / fill_with                                     src/common/cl_operations.hpp:9-16
  conversions                                                src/common/matrices_conversions.hpp:9-26

Every call runs on the CUDA library; there is no host fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import clb_coo, clb_csr, clb_dcsr, clb_spgemm_stats, lib
from .core import (ClBoolException, Controls, DeviceBuffer, check, matrix_coo, matrix_coo_cpu, matrix_csr,
                   matrix_csr_cpu, matrix_dcsr, matrix_dcsr_cpu)


def _require(name: str):
    f = getattr(lib, name, None)
    if f is None:
        raise ClBoolException(65, f"{name} is not in this build of libclbool_b200.so")
    return f


# ------------------------------------------------------------- primitives --
def prefix_sum(controls: Controls, array: DeviceBuffer, array_size: int) -> int:
    """Exclusive scan of `array_size` entries in place; returns the total."""
    total = C.c_uint64()
    f = lib.clb_prefix_sum_u64 if array.dtype == np.uint64 else lib.clb_prefix_sum_u32
    check(f(controls.handle, C.c_void_p(array.ptr), int(array_size), C.byref(total)), "prefix_sum")
    return int(total.value)


def fill_with(controls: Controls, array: DeviceBuffer, size: int, value: int) -> None:
    check(lib.clb_fill_u32(controls.handle, C.c_void_p(array.ptr), int(size), int(value)), "fill_with")


def fill_with_zeroes(controls: Controls, array: DeviceBuffer, size: int) -> None:
    fill_with(controls, array, size, 0)


def _coo_sort(controls: Controls, rows: DeviceBuffer, cols: DeviceBuffer, n: int) -> None:
    check(_require("clb_coo_sort")(controls.handle, C.c_void_p(rows.ptr), C.c_void_p(cols.ptr), int(n)),
          "sort_arrays")


def _coo_reduce_duplicates(controls: Controls, m: matrix_coo) -> matrix_coo:
    out = clb_coo()
    s = m.c_struct()
    check(_require("clb_coo_reduce_duplicates")(controls.handle, C.byref(s), C.byref(out)), "reduce_duplicates")
    return matrix_coo.adopt(controls, out)


# ------------------------------------------------------------ conversions --
def coo_to_dcsr_shallow(controls: Controls, a: matrix_coo) -> matrix_dcsr:
    if a.empty():
        return matrix_dcsr.zeros(a.nrows(), a.ncols())
    out = clb_dcsr()
    s = a.c_struct()
    check(lib.clb_coo_to_dcsr(controls.handle, C.byref(s), C.byref(out), 0), "coo_to_dcsr_shallow")
    return matrix_dcsr.adopt(controls, out, cols_owner=a.cols_gpu())


def dcsr_to_coo_shallow(controls: Controls, a: matrix_dcsr) -> matrix_coo:
    if a.empty():
        return matrix_coo.zeros(a.nrows(), a.ncols())
    out = clb_coo()
    s = a.c_struct()
    check(lib.clb_dcsr_to_coo(controls.handle, C.byref(s), C.byref(out), 0), "dcsr_to_coo_shallow")
    return matrix_coo.adopt(controls, out, cols_owner=a.cols_gpu())


def dcsr_to_coo_deep(controls: Controls, a: matrix_dcsr) -> matrix_coo:
    if a.empty():
        return matrix_coo.zeros(a.nrows(), a.ncols())
    out = clb_coo()
    s = a.c_struct()
    check(lib.clb_dcsr_to_coo(controls.handle, C.byref(s), C.byref(out), 1), "dcsr_to_coo_deep")
    return matrix_coo.adopt(controls, out)


def dcsr_to_csr(controls: Controls, m: matrix_dcsr) -> matrix_csr:
    """Shallow for cols (matrices_conversions.hpp:25-26)."""
    if m.empty():
        return matrix_csr.zeros(m.nrows(), m.ncols())
    out = clb_csr()
    s = m.c_struct()
    check(lib.clb_dcsr_to_csr(controls.handle, C.byref(s), C.byref(out)), "dcsr_to_csr")
    return matrix_csr.adopt(controls, out, cols_owner=m.cols_gpu())


def csr_to_dcsr(controls: Controls, m: matrix_csr) -> matrix_dcsr:
    """Shallow for cols (matrices_conversions.hpp:23-24)."""
    if m.empty():
        return matrix_dcsr.zeros(m.nrows(), m.ncols())
    out = clb_dcsr()
    s = m.c_struct()
    check(lib.clb_csr_to_dcsr(controls.handle, C.byref(s), C.byref(out)), "csr_to_dcsr")
    return matrix_dcsr.adopt(controls, out, cols_owner=m.cols_gpu())


def matrix_dcsr_from_cpu(controls: Controls, m: matrix_dcsr_cpu, size: int, ncols: int | None = None) -> matrix_dcsr:
    """matrix_dcsr_from_cpu (matrices_conversions.cpp:93-108): square `size`
    unless `ncols` is given."""
    nc = size if ncols is None else ncols
    if len(m.cols) == 0:
        return matrix_dcsr.zeros(size, nc)
    return matrix_dcsr(DeviceBuffer.from_host(controls, m.rpt, np.uint64),
                       DeviceBuffer.from_host(controls, m.rows, np.uint32),
                       DeviceBuffer.from_host(controls, m.cols, np.uint32),
                       size, nc, len(m.cols), len(m.rows))


def matrix_dcsr_from_gpu(controls: Controls, m: matrix_dcsr) -> matrix_dcsr_cpu:
    if m.empty():
        return matrix_dcsr_cpu()
    return matrix_dcsr_cpu(m.rpt_gpu().to_host(m.nzr() + 1), m.rows_gpu().to_host(m.nzr()),
                           m.cols_gpu().to_host(m.nnz()))


def matrix_coo_from_gpu(controls: Controls, m: matrix_coo) -> matrix_coo_cpu:
    if m.empty():
        return matrix_coo_cpu()
    return matrix_coo_cpu(m.rows_gpu().to_host(m.nnz()), m.cols_gpu().to_host(m.nnz()))


def matrix_csr_from_gpu(controls: Controls, m: matrix_csr) -> matrix_csr_cpu:
    if m.empty():
        return matrix_csr_cpu(None, None, m.nrows(), m.ncols())
    return matrix_csr_cpu(m.rpt_gpu().to_host(m.nrows() + 1), m.cols_gpu().to_host(m.nnz()), m.nrows(), m.ncols())


def csr_from_cpu(controls: Controls, m: matrix_csr_cpu) -> matrix_csr:
    if len(m.cols) == 0:
        return matrix_csr.zeros(m.nrows, m.ncols)
    return matrix_csr(DeviceBuffer.from_host(controls, m.rpt, np.uint64),
                      DeviceBuffer.from_host(controls, m.cols, np.uint32), m.nrows, m.ncols, len(m.cols))


def csr_cpu_from_pairs(rows, cols, m: int, n: int) -> matrix_csr_cpu:
    """csr_cpu_from_pairs (matrices_conversions.cpp:158-177), host only: rows
    must be sorted."""
    r = np.asarray(rows, dtype=np.uint32)
    rpt = np.zeros(m + 1, dtype=np.uint64)
    if r.size:
        np.cumsum(np.bincount(r, minlength=m)[:m], out=rpt[1:])
    return matrix_csr_cpu(rpt, np.asarray(cols, dtype=np.uint32), m, n)


# -------------------------------------------------------------- operations --
def workload(controls: Controls, a: matrix_dcsr, b: matrix_dcsr):
    """Products per A row (count_workload) -> (DeviceBuffer uint32[nzr_A], total)."""
    total = C.c_uint64()
    sa, sb = a.c_struct(), b.c_struct()
    buf = DeviceBuffer.empty(controls, max(a.nzr(), 1), np.uint32)
    check(lib.clb_dcsr_workload(controls.handle, C.byref(sa), C.byref(sb), C.c_void_p(buf.ptr), C.byref(total)),
          "count_workload")
    return buf, int(total.value)


def _spgemm(fn_name: str, controls, matrix_out, a, b, stats):
    out = clb_dcsr()
    st = clb_spgemm_stats()
    sa, sb = a.c_struct(), b.c_struct()
    check(_require(fn_name)(controls.handle, C.byref(sa), C.byref(sb), C.byref(out), C.byref(st)), fn_name)
    res = matrix_dcsr.adopt(controls, out)
    if stats is not None:
        stats.update(st.as_dict())
    if matrix_out is None:
        return res
    return matrix_out._assign(res)


def matrix_multiplication_hash(controls: Controls, matrix_out: matrix_dcsr | None, a: matrix_dcsr, b: matrix_dcsr,
                               stats: dict | None = None) -> matrix_dcsr:
    """dcsr::matrix_multiplication_hash: C = A*B (boolean), exact two-pass."""
    return _spgemm("clb_dcsr_spgemm_hash", controls, matrix_out, a, b, stats)


def matrix_multiplication(controls: Controls, matrix_out: matrix_dcsr | None, a: matrix_dcsr, b: matrix_dcsr,
                          stats: dict | None = None) -> matrix_dcsr:
    """dcsr::matrix_multiplication (ESC/merge form)."""
    return _spgemm("clb_dcsr_spgemm_esc", controls, matrix_out, a, b, stats)


def coo_matrix_addition(controls: Controls, matrix_out: matrix_coo | None, a: matrix_coo, b: matrix_coo) -> matrix_coo:
    out = clb_coo()
    sa, sb = a.c_struct(), b.c_struct()
    check(_require("clb_coo_add")(controls.handle, C.byref(sa), C.byref(sb), C.byref(out)), "coo::matrix_addition")
    res = matrix_coo.adopt(controls, out)
    return res if matrix_out is None else matrix_out._assign(res)


def csr_matrix_addition(controls: Controls, c: matrix_csr | None, a: matrix_csr, b: matrix_csr) -> matrix_csr:
    out = clb_csr()
    sa, sb = a.c_struct(), b.c_struct()
    check(_require("clb_csr_add")(controls.handle, C.byref(sa), C.byref(sb), C.byref(out)), "csr::matrix_addition")
    res = matrix_csr.adopt(controls, out)
    return res if c is None else c._assign(res)


def csr_matrix_addition_batched(controls: Controls, pairs) -> list[matrix_csr]:
    """[A_k + B_k for (A_k, B_k) in pairs] (CSR, boolean) in one set of
    launches (clb_csr_add_batched)."""
    pairs = list(pairs)
    n = len(pairs)
    if n == 0:
        return []
    A, B, out = (clb_csr * n)(), (clb_csr * n)(), (clb_csr * n)()
    for k, (a, b) in enumerate(pairs):
        A[k], B[k] = a.c_struct(), b.c_struct()
    check(_require("clb_csr_add_batched")(controls.handle, n, A, B, out), "csr::matrix_addition_batched")
    return [matrix_csr.adopt(controls, out[k]) for k in range(n)]


def kronecker_product(controls: Controls, matrix_c: matrix_dcsr | None, matrix_a: matrix_dcsr,
                      matrix_b: matrix_dcsr) -> matrix_dcsr:
    out = clb_dcsr()
    sa, sb = matrix_a.c_struct(), matrix_b.c_struct()
    check(_require("clb_dcsr_kronecker")(controls.handle, C.byref(sa), C.byref(sb), C.byref(out)),
          "dcsr::kronecker_product")
    res = matrix_dcsr.adopt(controls, out)
    return res if matrix_c is None else matrix_c._assign(res)


def transpose(controls: Controls, matrix_out: matrix_dcsr | None, matrix_in: matrix_dcsr) -> matrix_dcsr:
    out = clb_dcsr()
    s = matrix_in.c_struct()
    check(_require("clb_dcsr_transpose")(controls.handle, C.byref(s), C.byref(out)), "dcsr::transpose")
    res = matrix_dcsr.adopt(controls, out)
    return res if matrix_out is None else matrix_out._assign(res)


def submatrix(controls: Controls, matrix_out: matrix_dcsr | None, matrix_in: matrix_dcsr, i: int, j: int, nrows: int,
              ncols: int) -> matrix_dcsr:
    """dcsr::submatrix: rows [i, i+nrows), columns [j, j+ncols), re-indexed."""
    out = clb_dcsr()
    s = matrix_in.c_struct()
    check(lib.clb_dcsr_submatrix(controls.handle, C.byref(s), int(i), int(j), int(nrows), int(ncols), C.byref(out)),
          "dcsr::submatrix")
    res = matrix_dcsr.adopt(controls, out)
    return res if matrix_out is None else matrix_out._assign(res)


def reduce(controls: Controls, matrix_out: matrix_dcsr | None, matrix_in: matrix_dcsr) -> matrix_dcsr:
    """dcsr::reduce: row-wise OR as an nrows x 1 matrix."""
    out = clb_dcsr()
    s = matrix_in.c_struct()
    check(lib.clb_dcsr_reduce(controls.handle, C.byref(s), C.byref(out)), "dcsr::reduce")
    res = matrix_dcsr.adopt(controls, out)
    return res if matrix_out is None else matrix_out._assign(res)


def sort_arrays(controls: Controls, rows_gpu: DeviceBuffer, cols_gpu: DeviceBuffer, n: int) -> None:
    _coo_sort(controls, rows_gpu, cols_gpu, n)
