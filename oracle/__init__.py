"""Parity oracle for the boolean sparse hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` import this package, and only to check results or to time the
CPU baseline.  The product library never calls it.

Two back ends, both plain host code:

* ``liboracle.so`` (``clb_oracle.c``): a CPU restatement of clBool's
  algorithm with 64-bit offsets and OpenMP; each C function cites the
  reference file:line it follows.
* ``_ref/libclbool_ref.so``: the reference's own CPU functions
  (``coo_utils::matrix_multiplication_cpu`` and friends), compiled from the
  reference sources by ``oracle/Makefile``.  It pins the restatement and is
  the reference arm's CPU implementation.  Absent when the reference sources
  were never available to build it.

Matrices cross this module as small namedtuples of numpy arrays with the
field names of the reference's host containers (``cpu_matrices.hpp``):
``Dcsr(nrows, ncols, rpt, rows, cols)``, ``Coo(nrows, ncols, rows, cols)``,
``Csr(nrows, ncols, rpt, cols)``; ``rpt`` is uint64, indices uint32.
"""
from __future__ import annotations

import ctypes as C
import os
from collections import namedtuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libclbool_ref.so")

Dcsr = namedtuple("Dcsr", "nrows ncols rpt rows cols")
Coo = namedtuple("Coo", "nrows ncols rows cols")
Csr = namedtuple("Csr", "nrows ncols rpt cols")

u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)


class _OrcDcsr(C.Structure):
    _fields_ = [("nrows", C.c_uint64), ("ncols", C.c_uint64), ("nnz", C.c_uint64), ("nzr", C.c_uint64),
                ("rpt", u64p), ("rows", u32p), ("cols", u32p)]


def _p32(a):
    return a.ctypes.data_as(u32p)


def _p64(a):
    return a.ctypes.data_as(u64p)


def build():
    """Compile liboracle.so (and _ref when CLBOOL_REFERENCE_SRC names the
    reference's source tree)."""
    import subprocess
    ref = os.environ.get("CLBOOL_REFERENCE_SRC", "")
    subprocess.run(["make", "-s", "-C", HERE, "all"] + ([f"REF={ref}"] if ref else []), check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_threads.restype = C.c_int
        L.orc_fill_random_buffer.argtypes = [u32p, C.c_uint32, C.c_uint32]
        L.orc_fill_random_matrix.argtypes = [u32p, u32p, C.c_uint32, C.c_uint32]
        for name in ("orc_gen_coo_pairs", "orc_gen_coo_inclusive"):
            f = getattr(L, name)
            f.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(u32p), C.POINTER(u32p)]
            f.restype = C.c_uint64
        L.orc_sort_pairs.argtypes = [u32p, u32p, C.c_uint64]
        L.orc_unique_pairs.argtypes = [u32p, u32p, C.c_uint64]
        L.orc_unique_pairs.restype = C.c_uint64
        L.orc_prefix_sum_u32.argtypes = [u32p, C.c_uint64]
        L.orc_prefix_sum_u32.restype = C.c_uint64
        L.orc_prefix_sum_u64.argtypes = [u64p, C.c_uint64]
        L.orc_prefix_sum_u64.restype = C.c_uint64
        L.orc_coo_to_dcsr.argtypes = [u32p, C.c_uint64, C.POINTER(u64p), C.POINTER(u32p)]
        L.orc_coo_to_dcsr.restype = C.c_uint64
        L.orc_dcsr_to_coo_rows.argtypes = [u64p, u32p, C.c_uint64, u32p]
        L.orc_dcsr_to_csr_rpt.argtypes = [u64p, u32p, C.c_uint64, C.c_uint64, u64p]
        L.orc_csr_to_dcsr.argtypes = [u64p, C.c_uint64, C.POINTER(u64p), C.POINTER(u32p)]
        L.orc_csr_to_dcsr.restype = C.c_uint64
        L.orc_csr_rpt_from_coo.argtypes = [u32p, C.c_uint64, C.c_uint64, u64p]
        L.orc_workload.argtypes = [C.POINTER(_OrcDcsr), C.POINTER(_OrcDcsr), u64p]
        L.orc_spgemm.argtypes = [C.POINTER(_OrcDcsr), C.POINTER(_OrcDcsr), C.POINTER(_OrcDcsr)]
        L.orc_spgemm.restype = C.c_int
        L.orc_spgemm_row_nnz.argtypes = [C.POINTER(_OrcDcsr), C.POINTER(_OrcDcsr), u64p]
        L.orc_spgemm_row_nnz.restype = C.c_int
        L.orc_coo_add.argtypes = [u32p, u32p, C.c_uint64, u32p, u32p, C.c_uint64, C.POINTER(u32p), C.POINTER(u32p)]
        L.orc_coo_add.restype = C.c_uint64
        L.orc_csr_add.argtypes = [u64p, u32p, u64p, u32p, C.c_uint64, u64p, C.POINTER(u32p)]
        L.orc_csr_add.restype = C.c_uint64
        L.orc_kronecker.argtypes = [C.POINTER(_OrcDcsr), C.POINTER(_OrcDcsr), C.POINTER(_OrcDcsr)]
        L.orc_transpose.argtypes = [C.POINTER(_OrcDcsr), C.POINTER(_OrcDcsr)]
        L.orc_submatrix.argtypes = [C.POINTER(_OrcDcsr), C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                                    C.POINTER(_OrcDcsr)]
        L.orc_reduce.argtypes = [C.POINTER(_OrcDcsr), C.POINTER(_OrcDcsr)]
        L.orc_mlp_num_params.restype = C.c_int
        f32p = C.POINTER(C.c_float)
        f64p = C.POINTER(C.c_double)
        L.orc_mlp_grad.argtypes = [f32p, f32p, f32p, C.c_uint64, f64p, f64p, f64p]
        _lib = L
    return _lib


def set_threads(n: int = 0) -> int:
    return lib().orc_set_threads(n)


def _take(ptr, n, dtype):
    """Copy n elements out of a malloc'ed C array and free it."""
    if n:
        out = np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)
    else:
        out = np.zeros(0, dtype=dtype)
    lib().orc_free(C.cast(ptr, C.c_void_p))
    return out


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def _to_orc(m: Dcsr, keep: list):
    rpt, rows, cols = _c64(m.rpt), _c32(m.rows), _c32(m.cols)
    if rpt.size == 0:
        rpt = np.zeros(1, np.uint64)
    keep += [rpt, rows, cols]
    s = _OrcDcsr()
    s.nrows, s.ncols = int(m.nrows), int(m.ncols)
    s.nzr = rows.size
    s.nnz = cols.size
    s.rpt, s.rows, s.cols = _p64(rpt), _p32(rows), _p32(cols)
    return s


def _from_orc(s: _OrcDcsr) -> Dcsr:
    if s.nnz == 0:
        return Dcsr(int(s.nrows), int(s.ncols), np.zeros(1, np.uint64), np.zeros(0, np.uint32),
                    np.zeros(0, np.uint32))
    rpt = _take(s.rpt, s.nzr + 1, np.uint64)
    rows = _take(s.rows, s.nzr, np.uint32)
    cols = _take(s.cols, s.nnz, np.uint32)
    return Dcsr(int(s.nrows), int(s.ncols), rpt, rows, cols)


# ----------------------------------------------------------------- generators
def fill_random_buffer(n: int, maxv: int) -> np.ndarray:
    out = np.zeros(max(n, 1), np.uint32)
    lib().orc_fill_random_buffer(_p32(out), n, maxv)
    return out[:n]


def fill_random_matrix(n: int, max_size: int = 1024):
    r = np.zeros(max(n, 1), np.uint32)
    c = np.zeros(max(n, 1), np.uint32)
    lib().orc_fill_random_matrix(_p32(r), _p32(c), n, max_size)
    return r[:n], c[:n]


def generate_coo_pairs(pseudo_nnz: int, max_size: int):
    """generate_coo_pairs_cpu (coo_utils.cpp:204-218): sorted unique pairs."""
    r, c = u32p(), u32p()
    n = lib().orc_gen_coo_pairs(pseudo_nnz, max_size, C.byref(r), C.byref(c))
    return _take(r, n, np.uint32), _take(c, n, np.uint32)


def generate_coo_inclusive(pseudo_nnz: int, max_size: int):
    """generate_coo_cpu (coo_utils.cpp:220-239)."""
    r, c = u32p(), u32p()
    n = lib().orc_gen_coo_inclusive(pseudo_nnz, max_size, C.byref(r), C.byref(c))
    return _take(r, n, np.uint32), _take(c, n, np.uint32)


# ------------------------------------------------------------- conversions
def coo_to_dcsr(m: Coo) -> Dcsr:
    rows = _c32(m.rows)
    if rows.size == 0:
        return Dcsr(m.nrows, m.ncols, np.zeros(1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    rp, rr = u64p(), u32p()
    nzr = lib().orc_coo_to_dcsr(_p32(rows), rows.size, C.byref(rp), C.byref(rr))
    return Dcsr(m.nrows, m.ncols, _take(rp, nzr + 1, np.uint64), _take(rr, nzr, np.uint32), _c32(m.cols).copy())


def dcsr_to_coo(m: Dcsr) -> Coo:
    cols = _c32(m.cols)
    rows = np.zeros(max(cols.size, 1), np.uint32)
    if cols.size:
        lib().orc_dcsr_to_coo_rows(_p64(_c64(m.rpt)), _p32(_c32(m.rows)), len(m.rows), _p32(rows))
    return Coo(m.nrows, m.ncols, rows[:cols.size], cols.copy())


def dcsr_to_csr(m: Dcsr) -> Csr:
    out = np.zeros(m.nrows + 1, np.uint64)
    if len(m.cols):
        lib().orc_dcsr_to_csr_rpt(_p64(_c64(m.rpt)), _p32(_c32(m.rows)), len(m.rows), m.nrows, _p64(out))
    return Csr(m.nrows, m.ncols, out, _c32(m.cols).copy())


def csr_to_dcsr(m: Csr) -> Dcsr:
    rpt = _c64(m.rpt)
    if len(m.cols) == 0:
        return Dcsr(m.nrows, m.ncols, np.zeros(1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    rp, rr = u64p(), u32p()
    nzr = lib().orc_csr_to_dcsr(_p64(rpt), m.nrows, C.byref(rp), C.byref(rr))
    return Dcsr(m.nrows, m.ncols, _take(rp, nzr + 1, np.uint64), _take(rr, nzr, np.uint32), _c32(m.cols).copy())


def coo_to_csr(m: Coo) -> Csr:
    """csr_cpu_from_pairs (matrices_conversions.cpp:158-177)."""
    out = np.zeros(m.nrows + 1, np.uint64)
    rows = _c32(m.rows)
    lib().orc_csr_rpt_from_coo(_p32(rows) if rows.size else None, rows.size, m.nrows, _p64(out))
    return Csr(m.nrows, m.ncols, out, _c32(m.cols).copy())


# ------------------------------------------------------------------ ops
def prefix_sum_u32(a: np.ndarray):
    """Exclusive scan in place semantics (cl_operations.cpp:4-88): (scanned, total)."""
    x = _c32(a).copy()
    total = lib().orc_prefix_sum_u32(_p32(x), x.size) if x.size else 0
    return x, int(total)


def sort_pairs(rows, cols):
    r, c = _c32(rows).copy(), _c32(cols).copy()
    if r.size:
        lib().orc_sort_pairs(_p32(r), _p32(c), r.size)
    return r, c


def unique_pairs(rows, cols):
    r, c = _c32(rows).copy(), _c32(cols).copy()
    n = lib().orc_unique_pairs(_p32(r), _p32(c), r.size) if r.size else 0
    return r[:n], c[:n]


def workload(a: Dcsr, b: Dcsr) -> np.ndarray:
    """Intermediate products per A row (count_workload.cl:30-53)."""
    keep = []
    sa, sb = _to_orc(a, keep), _to_orc(b, keep)
    out = np.zeros(max(len(a.rows), 1), np.uint64)
    if len(a.rows):
        lib().orc_workload(C.byref(sa), C.byref(sb), _p64(out))
    return out[:len(a.rows)]


def spgemm(a: Dcsr, b: Dcsr) -> Dcsr:
    """C = A*B over the boolean semiring (coo_utils.cpp:470-514 semantics)."""
    if a.ncols != b.nrows:
        raise ValueError("inner dimensions differ")
    keep = []
    sa, sb = _to_orc(a, keep), _to_orc(b, keep)
    sc = _OrcDcsr()
    rc = lib().orc_spgemm(C.byref(sa), C.byref(sb), C.byref(sc))
    if rc != 0:
        raise ValueError("oracle: B.ncols too wide for the bitmap accumulator")
    return _from_orc(sc)


def spgemm_row_nnz(a: Dcsr, b: Dcsr) -> np.ndarray:
    """Exact nnz of C's row for every A row (0 where no products)."""
    keep = []
    sa, sb = _to_orc(a, keep), _to_orc(b, keep)
    out = np.zeros(max(len(a.rows), 1), np.uint64)
    if len(a.rows):
        rc = lib().orc_spgemm_row_nnz(C.byref(sa), C.byref(sb), _p64(out))
        if rc != 0:
            raise ValueError("oracle: B.ncols too wide")
    return out[:len(a.rows)]


def coo_add(a: Coo, b: Coo) -> Coo:
    """std::merge + std::unique (coo_utils.cpp:315-324)."""
    ar, ac, br, bc = _c32(a.rows), _c32(a.cols), _c32(b.rows), _c32(b.cols)
    r, c = u32p(), u32p()
    z = np.zeros(1, np.uint32)
    n = lib().orc_coo_add(_p32(ar if ar.size else z), _p32(ac if ac.size else z), ar.size,
                          _p32(br if br.size else z), _p32(bc if bc.size else z), br.size, C.byref(r), C.byref(c))
    return Coo(a.nrows, a.ncols, _take(r, n, np.uint32), _take(c, n, np.uint32))


def csr_add(a: Csr, b: Csr) -> Csr:
    rpt = np.zeros(a.nrows + 1, np.uint64)
    z = np.zeros(1, np.uint32)
    ac, bc = _c32(a.cols), _c32(b.cols)
    out = u32p()
    n = lib().orc_csr_add(_p64(_c64(a.rpt)), _p32(ac if ac.size else z), _p64(_c64(b.rpt)),
                          _p32(bc if bc.size else z), a.nrows, _p64(rpt), C.byref(out))
    return Csr(a.nrows, a.ncols, rpt, _take(out, n, np.uint32))


def kronecker(a: Dcsr, b: Dcsr) -> Dcsr:
    keep = []
    sa, sb = _to_orc(a, keep), _to_orc(b, keep)
    sc = _OrcDcsr()
    lib().orc_kronecker(C.byref(sa), C.byref(sb), C.byref(sc))
    return _from_orc(sc)


def transpose(a: Dcsr) -> Dcsr:
    keep = []
    sa = _to_orc(a, keep)
    sc = _OrcDcsr()
    lib().orc_transpose(C.byref(sa), C.byref(sc))
    return _from_orc(sc)


def submatrix(a: Dcsr, i: int, j: int, nrows: int, ncols: int) -> Dcsr:
    """Rows [i, i+nrows), columns [j, j+ncols) of A, re-indexed (empty rows
    dropped); cpu_matrix_operations.cpp:6-52."""
    keep = []
    sa = _to_orc(a, keep)
    sc = _OrcDcsr()
    lib().orc_submatrix(C.byref(sa), i, j, nrows, ncols, C.byref(sc))
    return _from_orc(sc)


def reduce(a: Dcsr) -> Dcsr:
    """Row-wise OR: one entry (column 0) per stored row; dcsr_reduce.cpp:5-31."""
    keep = []
    sa = _to_orc(a, keep)
    sc = _OrcDcsr()
    lib().orc_reduce(C.byref(sa), C.byref(sc))
    return _from_orc(sc)


def union(mats) -> Dcsr:
    """Boolean sum of DCSR matrices of one shape (restates
    coo_utils::matrix_addition_cpu, coo_utils.cpp:315-324, folded)."""
    m0 = mats[0]
    rows, cols = [], []
    for m in mats:
        if len(m.cols):
            rows.append(np.repeat(np.asarray(m.rows, np.uint32), np.diff(np.asarray(m.rpt, np.int64))))
            cols.append(np.asarray(m.cols, np.uint32))
    if not rows:
        return coo_to_dcsr(Coo(m0.nrows, m0.ncols, np.zeros(0, np.uint32), np.zeros(0, np.uint32)))
    r, c = unique_pairs(*sort_pairs(np.concatenate(rows), np.concatenate(cols)))
    return coo_to_dcsr(Coo(m0.nrows, m0.ncols, r, c))


def closure(labels, max_iters: int = 64):
    """Bounded fixpoint C_{t+1} = C_t v sum_i C_t L_i from C_0 = v_i L_i;
    returns (C, nnz per iteration).  Not in the reference."""
    C = union(labels)
    hist = [len(C.cols)]
    for _ in range(max_iters):
        Cn = union([C] + [spgemm(C, L) for L in labels])
        hist.append(len(Cn.cols))
        stable = len(Cn.cols) == len(C.cols)
        C = Cn
        if stable:
            break
    return C, hist


def row_features(a: Dcsr, b: Dcsr) -> np.ndarray:
    """Six features of every A row of A*B (float64, shape [nzr_A, 6]), the
    inputs of the row-size predictor: log2(1+|A_i|), log2(1+P_i),
    log2(1+max |B_k|), log2(1+min nonzero |B_k|) -- k over the columns of A_i,
    all divided by 16 -- then A.rows[i] / A.nrows and
    log2(B.nrows * B.ncols / nnz(B)) / 16.  Not in the reference."""
    nzr = len(a.rows) if len(a.cols) else 0
    out = np.zeros((nzr, 6), np.float64)
    if nzr == 0:
        return out
    blen = np.zeros(max(int(a.ncols), 1), np.int64)
    if len(b.cols):
        brpt = np.asarray(b.rpt, np.int64)
        keep = np.asarray(b.rows, np.int64) < blen.size
        blen[np.asarray(b.rows, np.int64)[keep]] = np.diff(brpt)[keep]
    arpt = np.asarray(a.rpt, np.int64)
    lens = blen[np.asarray(a.cols, np.int64)]
    seg = np.repeat(np.arange(nzr), np.diff(arpt))
    P = np.bincount(seg, weights=lens, minlength=nzr)
    mx = np.zeros(nzr)
    np.maximum.at(mx, seg, lens)
    mn = np.full(nzr, np.inf)
    nzl = lens > 0
    np.minimum.at(mn, seg[nzl], lens[nzl])
    mn[np.isinf(mn)] = 0
    out[:, 0] = np.log2(1.0 + np.diff(arpt)) / 16
    out[:, 1] = np.log2(1.0 + P) / 16
    out[:, 2] = np.log2(1.0 + mx) / 16
    out[:, 3] = np.log2(1.0 + mn) / 16
    out[:, 4] = np.asarray(a.rows, np.float64) / float(a.nrows) if a.nrows else 0.0
    nnzb = len(b.cols)
    out[:, 5] = np.log2(float(b.nrows) * float(b.ncols) / nnzb) / 16 if nnzb else 0.0
    return out


def mlp_grad(params, features, targets):
    """FP64 loss, gradient and predictions of the row-size predictor
    (6 -> 64 -> 64 -> 1, ReLU, BF16-rounded weights, MSE)."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    f = np.ascontiguousarray(features, dtype=np.float32).reshape(-1)
    t = np.ascontiguousarray(targets, dtype=np.float32)
    n = t.size
    g = np.zeros(lib().orc_mlp_num_params(), np.float64)
    pr = np.zeros(max(n, 1), np.float64)
    loss = C.c_double()
    f32p = C.POINTER(C.c_float)
    f64p = C.POINTER(C.c_double)
    lib().orc_mlp_grad(p.ctypes.data_as(f32p), f.ctypes.data_as(f32p), t.ctypes.data_as(f32p), n,
                       g.ctypes.data_as(f64p), C.byref(loss), pr.ctypes.data_as(f64p))
    return float(loss.value), g, pr[:n]


# ------------------------------------------------------- reference library
class Ref:
    """The reference's own CPU functions (built into _ref/ by the Makefile)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        L.ref_free.argtypes = [C.c_void_p]
        L.ref_gen_coo_pairs.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(u32p), C.POINTER(u32p)]
        L.ref_gen_coo_pairs.restype = C.c_uint64
        L.ref_gen_coo_cpu.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(u32p), C.POINTER(u32p)]
        L.ref_gen_coo_cpu.restype = C.c_uint64
        L.ref_fill_random_buffer.argtypes = [u32p, C.c_uint32, C.c_uint32]
        L.ref_fill_random_matrix.argtypes = [u32p, u32p, C.c_uint32, C.c_uint32]
        L.ref_pairs_to_dcsr.argtypes = [u32p, u32p, C.c_uint32, C.POINTER(u32p), C.POINTER(u32p), C.POINTER(u32p)]
        L.ref_pairs_to_dcsr.restype = C.c_uint32
        dc = [u32p, u32p, u32p, C.c_uint32, C.c_uint32]
        L.ref_spgemm.argtypes = dc + dc + [C.POINTER(u32p), C.POINTER(u32p), C.POINTER(u32p), C.POINTER(C.c_uint32)]
        L.ref_spgemm.restype = C.c_uint32
        L.ref_workload.argtypes = dc + dc + [u32p]
        L.ref_coo_add.argtypes = [u32p, u32p, C.c_uint32, u32p, u32p, C.c_uint32, C.POINTER(u32p), C.POINTER(u32p)]
        L.ref_coo_add.restype = C.c_uint64
        L.ref_csr_from_pairs.argtypes = [u32p, u32p, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(u32p),
                                         C.POINTER(u32p)]
        L.ref_kronecker_pairs.argtypes = [u32p, u32p, C.c_uint32, u32p, u32p, C.c_uint32, C.c_uint32, C.c_uint32,
                                          C.POINTER(u32p), C.POINTER(u32p)]
        L.ref_kronecker_pairs.restype = C.c_uint64
        L.ref_submatrix.argtypes = [u32p, u32p, u32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.c_uint32, C.POINTER(u32p), C.POINTER(u32p), C.POINTER(u32p),
                                    C.POINTER(C.c_uint32)]
        L.ref_submatrix.restype = C.c_uint32
        L.ref_reduce.argtypes = [u32p, u32p, u32p, C.c_uint32, C.c_uint32, C.POINTER(u32p), C.POINTER(u32p),
                                 C.POINTER(u32p)]
        L.ref_reduce.restype = C.c_uint32
        L.ref_random_matrices.argtypes = [C.c_int, C.c_uint32, C.c_uint32] + \
            [C.POINTER(u32p)] * 3 + [u32p] + [C.POINTER(u32p)] * 3 + [u32p]
        self.L = L

    def _take(self, ptr, n, dtype=np.uint32):
        out = np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True) if n else np.zeros(0, dtype)
        self.L.ref_free(C.cast(ptr, C.c_void_p))
        return out

    @staticmethod
    def _arr(a):
        a = _c32(a)
        return a if a.size else np.zeros(1, np.uint32)

    def generate_coo_pairs(self, pseudo_nnz, max_size):
        r, c = u32p(), u32p()
        n = self.L.ref_gen_coo_pairs(pseudo_nnz, max_size, C.byref(r), C.byref(c))
        return self._take(r, n), self._take(c, n)

    def generate_coo_cpu(self, pseudo_nnz, max_size):
        r, c = u32p(), u32p()
        n = self.L.ref_gen_coo_cpu(pseudo_nnz, max_size, C.byref(r), C.byref(c))
        return self._take(r, n), self._take(c, n)

    def fill_random_buffer(self, n, maxv):
        out = np.zeros(max(n, 1), np.uint32)
        self.L.ref_fill_random_buffer(_p32(out), n, maxv)
        return out[:n]

    def fill_random_matrix(self, n, max_size=1024):
        r = np.zeros(max(n, 1), np.uint32)
        c = np.zeros(max(n, 1), np.uint32)
        self.L.ref_fill_random_matrix(_p32(r), _p32(c), n, max_size)
        return r[:n], c[:n]

    def pairs_to_dcsr(self, rows, cols, nrows, ncols) -> Dcsr:
        rp, rr, cc = u32p(), u32p(), u32p()
        n = len(rows)
        nzr = self.L.ref_pairs_to_dcsr(_p32(self._arr(rows)), _p32(self._arr(cols)), n, C.byref(rp), C.byref(rr),
                                       C.byref(cc))
        rpt = self._take(rp, nzr + 1 if n else 0).astype(np.uint64)
        if rpt.size == 0:
            rpt = np.zeros(1, np.uint64)
        return Dcsr(nrows, ncols, rpt, self._take(rr, nzr), self._take(cc, n))

    def _dc(self, m: Dcsr):
        rpt = self._arr(np.asarray(m.rpt, dtype=np.uint64).astype(np.uint32))
        return [_p32(rpt), _p32(self._arr(m.rows)), _p32(self._arr(m.cols)), len(m.rows), len(m.cols)], rpt

    def spgemm(self, a: Dcsr, b: Dcsr) -> Dcsr:
        keep = [self._arr(a.rows), self._arr(a.cols), self._arr(b.rows), self._arr(b.cols)]
        ra = self._arr(np.asarray(a.rpt, dtype=np.uint64).astype(np.uint32))
        rb = self._arr(np.asarray(b.rpt, dtype=np.uint64).astype(np.uint32))
        rp, rr, cc, nzr = u32p(), u32p(), u32p(), C.c_uint32()
        nnz = self.L.ref_spgemm(_p32(ra), _p32(keep[0]), _p32(keep[1]), len(a.rows), len(a.cols),
                                _p32(rb), _p32(keep[2]), _p32(keep[3]), len(b.rows), len(b.cols),
                                C.byref(rp), C.byref(rr), C.byref(cc), C.byref(nzr))
        rpt = self._take(rp, nzr.value + 1).astype(np.uint64)
        return Dcsr(a.nrows, b.ncols, rpt, self._take(rr, nzr.value), self._take(cc, nnz))

    def workload(self, a: Dcsr, b: Dcsr) -> np.ndarray:
        keep = [self._arr(a.rows), self._arr(a.cols), self._arr(b.rows), self._arr(b.cols)]
        ra = self._arr(np.asarray(a.rpt, dtype=np.uint64).astype(np.uint32))
        rb = self._arr(np.asarray(b.rpt, dtype=np.uint64).astype(np.uint32))
        out = np.zeros(max(len(a.rows), 1), np.uint32)
        self.L.ref_workload(_p32(ra), _p32(keep[0]), _p32(keep[1]), len(a.rows), len(a.cols),
                            _p32(rb), _p32(keep[2]), _p32(keep[3]), len(b.rows), len(b.cols), _p32(out))
        return out[:len(a.rows)]

    def coo_add(self, a: Coo, b: Coo) -> Coo:
        r, c = u32p(), u32p()
        n = self.L.ref_coo_add(_p32(self._arr(a.rows)), _p32(self._arr(a.cols)), len(a.rows),
                               _p32(self._arr(b.rows)), _p32(self._arr(b.cols)), len(b.rows), C.byref(r), C.byref(c))
        return Coo(a.nrows, a.ncols, self._take(r, n), self._take(c, n))

    def csr_from_pairs(self, rows, cols, nrows, ncols) -> Csr:
        rp, cc = u32p(), u32p()
        n = len(rows)
        self.L.ref_csr_from_pairs(_p32(self._arr(rows)), _p32(self._arr(cols)), n, nrows, ncols, C.byref(rp),
                                  C.byref(cc))
        return Csr(nrows, ncols, self._take(rp, nrows + 1).astype(np.uint64), self._take(cc, n))

    def random_matrices(self, which: str, max_size: int, seed: int):
        """generate_random_matrices_esc / _large (coo_utils.cpp:13-132) -> (A, B)
        as Dcsr (arrays exactly as the reference builds them)."""
        ptrs = [u32p() for _ in range(6)]
        sa = (C.c_uint32 * 3)()
        sb = (C.c_uint32 * 3)()
        self.L.ref_random_matrices(1 if which == "large" else 0, max_size, seed, C.byref(ptrs[0]), C.byref(ptrs[1]),
                                   C.byref(ptrs[2]), sa, C.byref(ptrs[3]), C.byref(ptrs[4]), C.byref(ptrs[5]), sb)
        a = [self._take(ptrs[i], sa[i]) for i in range(3)]
        b = [self._take(ptrs[3 + i], sb[i]) for i in range(3)]
        A = Dcsr(max_size, max_size, a[0].astype(np.uint64), a[1], a[2])
        B = Dcsr(max_size, max_size, b[0].astype(np.uint64), b[1], b[2])
        return A, B

    def submatrix(self, a: Dcsr, i, j, nrows, ncols) -> Dcsr:
        keep = [self._arr(a.rows), self._arr(a.cols)]
        ra = self._arr(np.asarray(a.rpt, dtype=np.uint64).astype(np.uint32))
        rp, rr, cc, nzr = u32p(), u32p(), u32p(), C.c_uint32()
        nnz = self.L.ref_submatrix(_p32(ra), _p32(keep[0]), _p32(keep[1]), len(a.rows), len(a.cols), i, j, nrows,
                                   ncols, C.byref(rp), C.byref(rr), C.byref(cc), C.byref(nzr))
        # an empty result comes back without row pointers
        rpt = self._take(rp, nzr.value + 1).astype(np.uint64) if nnz else np.zeros(1, np.uint64)
        return Dcsr(nrows, ncols, rpt, self._take(rr, nzr.value), self._take(cc, nnz))

    def reduce(self, a: Dcsr) -> Dcsr:
        keep = [self._arr(a.rows), self._arr(a.cols)]
        ra = self._arr(np.asarray(a.rpt, dtype=np.uint64).astype(np.uint32))
        rp, rr, cc = u32p(), u32p(), u32p()
        n = self.L.ref_reduce(_p32(ra), _p32(keep[0]), _p32(keep[1]), len(a.rows), len(a.cols), C.byref(rp),
                              C.byref(rr), C.byref(cc))
        return Dcsr(a.nrows, 1, self._take(rp, n + 1).astype(np.uint64), self._take(rr, n), self._take(cc, n))

    def kronecker_pairs(self, a: Coo, b: Coo, b_nrows, b_ncols) -> Coo:
        r, c = u32p(), u32p()
        n = self.L.ref_kronecker_pairs(_p32(self._arr(a.rows)), _p32(self._arr(a.cols)), len(a.rows),
                                       _p32(self._arr(b.rows)), _p32(self._arr(b.cols)), len(b.rows),
                                       b_nrows, b_ncols, C.byref(r), C.byref(c))
        return Coo(a.nrows * b_nrows, a.ncols * b_ncols, self._take(r, n), self._take(c, n))


def ref_available() -> bool:
    return os.path.exists(REF_SO)
