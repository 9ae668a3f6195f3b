"""Tuned and batched boolean SpGEMM (no counterpart in the reference).

``matrix_multiplication_batched(controls, pairs)`` computes C_k = A_k * B_k for
a list of independent pairs in one pass: the library stacks the pairs
block-diagonally, runs one set of accumulator launches over all of them, and
splits the product per pair.  ``autotune`` times the accumulator tunings on a
batch and returns the fastest; every tuning gives the same C.
"""
from __future__ import annotations

import ctypes as C

from ._capi import clb_dcsr, clb_spgemm_stats, clb_spgemm_tuning, lib
from .core import ClBoolException, Controls, check, matrix_dcsr


def tuning(form: str | int = "two_pass", warp_max: int = 0, bitmap_min: int = 0, bitmap_threads: int = 0,
           small_lanes: int = 0, wide_rows: str = "") -> clb_spgemm_tuning:
    """A tuning; zero fields take the library defaults."""
    t = clb_spgemm_tuning()
    lib.clb_spgemm_tuning_default(C.byref(t))
    t.form = {"two_pass": 0, "single_pass": 1}.get(form, form) if isinstance(form, str) else int(form)
    if warp_max:
        t.warp_max = warp_max
    if bitmap_min:
        t.bitmap_min = bitmap_min
    if bitmap_threads:
        t.bitmap_threads = bitmap_threads
    if small_lanes:
        t.small_lanes = small_lanes
    if wide_rows:
        t.wide_rows = {"cluster": 1, "chunks": 2}[wide_rows]
    return t


def matrix_multiplication_tuned(controls: Controls, matrix_out: matrix_dcsr | None, a: matrix_dcsr, b: matrix_dcsr,
                                tune: clb_spgemm_tuning | None = None, stats: dict | None = None) -> matrix_dcsr:
    out, st = clb_dcsr(), clb_spgemm_stats()
    sa, sb = a.c_struct(), b.c_struct()
    check(lib.clb_dcsr_spgemm_tuned(controls.handle, C.byref(sa), C.byref(sb), C.byref(tune) if tune else None,
                                    C.byref(out), C.byref(st)), "matrix_multiplication_tuned")
    res = matrix_dcsr.adopt(controls, out)
    if stats is not None:
        stats.update(st.as_dict())
    return res if matrix_out is None else matrix_out._assign(res)


def _arrays(pairs):
    n = len(pairs)
    if n == 0:
        return 0, None, None, []
    A = (clb_dcsr * n)()
    B = (clb_dcsr * n)()
    for k, (a, b) in enumerate(pairs):
        A[k] = a.c_struct()
        B[k] = b.c_struct()
    return n, A, B, pairs  # `pairs` keeps the device buffers alive


def matrix_multiplication_batched(controls: Controls, pairs, tune: clb_spgemm_tuning | None = None,
                                  stats: dict | None = None) -> list[matrix_dcsr]:
    """[A_k * B_k for (A_k, B_k) in pairs] in one pass."""
    n, A, B, _keep = _arrays(list(pairs))
    if n == 0:
        return []
    out = (clb_dcsr * n)()
    st = clb_spgemm_stats()
    check(lib.clb_dcsr_spgemm_batched(controls.handle, n, A, B, out, C.byref(tune) if tune else None, C.byref(st)),
          "matrix_multiplication_batched")
    if stats is not None:
        stats.update(st.as_dict())
    return [matrix_dcsr.adopt(controls, out[k]) for k in range(n)]


def autotune(controls: Controls, pairs, max_tried: int = 64):
    """(best tuning, [(tuning dict, ms), ...]) over the library's candidate tunings."""
    n, A, B, _keep = _arrays(list(pairs))
    if n == 0:
        raise ClBoolException(12, "autotune needs at least one pair")
    best = clb_spgemm_tuning()
    tried = (clb_spgemm_tuning * max_tried)()
    ms = (C.c_double * max_tried)()
    nt = C.c_uint32()
    check(lib.clb_spgemm_autotune(controls.handle, n, A, B, C.byref(best), tried, ms, max_tried, C.byref(nt)),
          "autotune")
    return best, [(tried[k].as_dict(), ms[k]) for k in range(min(nt.value, max_tried))]
