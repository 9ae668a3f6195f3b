"""Tuned and batched boolean SpGEMM (no counterpart in the reference).

``matrix_multiplication_batched(controls, pairs)`` computes C_k = A_k * B_k for
a list of independent pairs in one pass: the library stacks the pairs
block-diagonally, runs one set of accumulator launches over all of them, and
splits the product per pair.  ``autotune`` times the accumulator tunings on a
batch and returns the fastest; every tuning gives the same C.

``CapturedBatch`` is the same product with caller-sized buffers and no read
back to the host, so it can be recorded once into a CUDA graph (``Graph``) and
replayed while the pairs' device arrays keep their sizes and change their
contents -- the repeated small products of a fixpoint, say, without the
per-call host round trips.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import clb_dcsr, clb_spgemm_stats, clb_spgemm_tuning, lib
from .core import ClBoolException, Controls, DeviceBuffer, check, matrix_dcsr


def tuning(form: str | int = "two_pass", warp_max: int = 0, bitmap_min: int = 0, bitmap_threads: int = 0,
           small_lanes: int = 0, wide_rows: str = "") -> clb_spgemm_tuning:
    """A tuning; zero fields take the library defaults.  form: "two_pass",
    "single_pass" or "two_pass_kept" (the exact two-pass form whose symbolic
    pass keeps the bitmap rows' bitmaps for its numeric pass)."""
    t = clb_spgemm_tuning()
    lib.clb_spgemm_tuning_default(C.byref(t))
    t.form = ({"two_pass": 0, "single_pass": 1, "two_pass_kept": 2}.get(form, form) if isinstance(form, str)
              else int(form))
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


def matrix_multiplication_batched_learned(controls: Controls, pairs, sizer, margin_log2: float | None = None,
                                          slack: float | None = None, tune: clb_spgemm_tuning | None = None,
                                          stats: dict | None = None) -> list[matrix_dcsr]:
    """[A_k * B_k for (A_k, B_k) in pairs] in one pass sized by `sizer` (a
    sizing.RowSizer): the stacked pairs' bitmap rows get predicted slots, the
    rest exact bounds; rows over their slot spill or are recomputed exactly,
    so the result equals matrix_multiplication_batched's."""
    from .sizing import DEFAULT_MARGIN_LOG2, DEFAULT_SLACK
    n, A, B, _keep = _arrays(list(pairs))
    if n == 0:
        return []
    out = (clb_dcsr * n)()
    st = clb_spgemm_stats()
    check(lib.clb_dcsr_spgemm_batched_learned(
        controls.handle, n, A, B, out, sizer.handle,
        float(DEFAULT_MARGIN_LOG2 if margin_log2 is None else margin_log2),
        float(DEFAULT_SLACK if slack is None else slack), C.byref(tune) if tune else None, C.byref(st)),
        "matrix_multiplication_batched_learned")
    if stats is not None:
        stats.update(st.as_dict())
    return [matrix_dcsr.adopt(controls, out[k]) for k in range(n)]


def matrix_union(controls: Controls, mats, tune: clb_spgemm_tuning | None = None,
                 stats: dict | None = None) -> matrix_dcsr:
    """mats[0] v mats[1] v ... (boolean sum of DCSR matrices of one shape) in
    one pass: a product with the matrices stacked row-wise, whose rows merge
    the matrices' rows (clb_dcsr_union)."""
    mats = list(mats)
    n = len(mats)
    if n == 0:
        raise ClBoolException(12, "union of no matrices")
    M = (clb_dcsr * n)()
    for k, m in enumerate(mats):
        M[k] = m.c_struct()
    out, st = clb_dcsr(), clb_spgemm_stats()
    check(lib.clb_dcsr_union(controls.handle, n, M, C.byref(tune) if tune else None, C.byref(out), C.byref(st)),
          "matrix_union")
    if stats is not None:
        stats.update(st.as_dict())
    return matrix_dcsr.adopt(controls, out)


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


class Graph:
    """A CUDA graph recorded from the controls' stream (clb_graph_begin / end)."""

    def __init__(self, controls: Controls, fn):
        self.controls = controls
        self.handle = None
        check(lib.clb_graph_begin(controls.handle), "graph_begin")
        try:
            fn()
        finally:
            h = C.c_void_p()
            rc = lib.clb_graph_end(controls.handle, C.byref(h))
        check(rc, "graph_end")
        self.handle = h

    def launch(self) -> None:
        """Replays the graph on the controls' stream (no synchronisation)."""
        check(lib.clb_graph_launch(self.controls.handle, self.handle), "graph_launch")

    def close(self) -> None:
        if self.handle:
            lib.clb_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batched_plan(controls: Controls, pairs, sizer=None, margin_log2: float | None = None,
                 slack: float | None = None, tune: clb_spgemm_tuning | None = None):
    """(rows_need, slots_need) of CapturedBatch for the pairs' current
    contents: upper-bound slots, or the learned slots when `sizer` is given."""
    n, A, B, _keep = _arrays(list(pairs))
    rows, slots = C.c_uint64(), C.c_uint64()
    if sizer is None:
        check(lib.clb_spgemm_batched_plan(controls.handle, n, A, B, C.byref(rows), C.byref(slots)), "batched_plan")
    else:
        from .sizing import DEFAULT_MARGIN_LOG2, DEFAULT_SLACK
        check(lib.clb_spgemm_batched_plan_learned(
            controls.handle, n, A, B, sizer.handle, float(DEFAULT_MARGIN_LOG2 if margin_log2 is None else margin_log2),
            float(DEFAULT_SLACK if slack is None else slack), C.byref(tune) if tune else None, C.byref(rows),
            C.byref(slots)), "batched_plan_learned")
    return int(rows.value), int(slots.value)


class CapturedBatch:
    """C_k = A_k * B_k for fixed pairs, into buffers sized once: ``enqueue()``
    issues the product without any host read (so it may run inside
    ``Graph(controls, batch.enqueue)``); ``result()`` synchronises and returns
    the per-pair host arrays, raising when a capacity was too small.

    With a `sizer` (sizing.RowSizer) the slots are the learned ones
    (clb_dcsr_spgemm_batched_capture_learned) plus a spill arena of
    `arena_capacity` entries (default: a quarter of the slots, at least 2^20);
    a row that outgrows both is reported in the flags, and ``result()`` then
    recomputes the batch by the exact batched form (``fell_back`` is set)."""

    FLAG_NAMES = {1: "slot capacity", 2: "column capacity", 4: "device check", 8: "learned slot and arena"}
    EXACT_RETRY = 1 | 2 | 8  # flags a learned batch recovers from by the exact form

    def __init__(self, controls: Controls, pairs, slot_capacity: int | None = None,
                 cols_capacity: int | None = None, tune: clb_spgemm_tuning | None = None, sizer=None,
                 margin_log2: float | None = None, slack: float | None = None, arena_capacity: int | None = None):
        from .sizing import DEFAULT_MARGIN_LOG2, DEFAULT_SLACK
        self.controls = controls
        self.pairs = list(pairs)
        self.count, self._A, self._B, _ = _arrays(self.pairs)
        if self.count == 0:
            raise ClBoolException(12, "CapturedBatch needs at least one pair")
        self.sizer = sizer
        self.margin_log2 = float(DEFAULT_MARGIN_LOG2 if margin_log2 is None else margin_log2)
        self.slack = float(DEFAULT_SLACK if slack is None else slack)
        rows, slots = batched_plan(controls, self.pairs, sizer, self.margin_log2, self.slack, tune)
        self.slot_capacity = int(slots if slot_capacity is None else slot_capacity)
        self.arena_capacity = 0
        if sizer is not None:
            self.arena_capacity = int(max(self.slot_capacity // 4, 1 << 20) if arena_capacity is None
                                      else arena_capacity)
        self.cols_capacity = int(self.slot_capacity + self.arena_capacity if cols_capacity is None
                                 else cols_capacity)
        self.rows_capacity = rows
        self.tune = tune
        self.fell_back = False
        self.rpt = DeviceBuffer.empty(controls, rows + 1, np.uint64)
        self.rows = DeviceBuffer.empty(controls, max(rows, 1), np.uint32)
        self.cols = DeviceBuffer.empty(controls, max(self.cols_capacity, 1), np.uint32)
        self.res = DeviceBuffer.empty(controls, 2 + 2 * (self.count + 1), np.uint64)
        self.flags = DeviceBuffer.empty(controls, 1, np.uint32)

    def enqueue(self) -> None:
        tune = C.byref(self.tune) if self.tune else None
        out = (C.c_void_p(self.rpt.ptr), C.c_void_p(self.rows.ptr), C.c_void_p(self.cols.ptr), self.cols_capacity,
               C.c_void_p(self.res.ptr), C.c_void_p(self.flags.ptr))
        if self.sizer is None:
            check(lib.clb_dcsr_spgemm_batched_capture(self.controls.handle, self.count, self._A, self._B, tune,
                                                      self.slot_capacity, *out), "batched_capture")
        else:
            check(lib.clb_dcsr_spgemm_batched_capture_learned(
                self.controls.handle, self.count, self._A, self._B, self.sizer.handle, self.margin_log2, self.slack,
                tune, self.slot_capacity, self.arena_capacity, *out), "batched_capture_learned")

    def flags_now(self) -> int:
        """The flag word of the last enqueued call (synchronises)."""
        self.controls.sync()
        return int(self.flags.to_host(1)[0])

    def result(self):
        """[(rpt u64, rows u32, cols u32) per pair] on the host."""
        flags = self.flags_now()
        self.fell_back = False
        if flags and self.sizer is not None and not flags & ~self.EXACT_RETRY:
            # a learned slot (and the arena) was too small for some row: the
            # exact batched form gives the same product
            self.fell_back = True
            out = []
            for c in matrix_multiplication_batched(self.controls, self.pairs):
                if c.nnz() == 0:
                    out.append((np.zeros(1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint32)))
                    continue
                out.append((c.rpt_gpu().to_host(c.nzr() + 1).astype(np.uint64), c.rows_gpu().to_host(c.nzr()),
                            c.cols_gpu().to_host(c.nnz())))
            return out
        if flags:
            what = ", ".join(v for k, v in self.FLAG_NAMES.items() if flags & k)
            raise ClBoolException(5, f"captured batch incomplete ({what} exceeded or failed)")
        r = self.res.to_host()
        nzr, nnz, k = int(r[0]), int(r[1]), self.count
        rpt = self.rpt.to_host(nzr + 1).astype(np.uint64)
        rows = self.rows.to_host(nzr) if nzr else np.zeros(0, np.uint32)
        cols = self.cols.to_host(nnz) if nnz else np.zeros(0, np.uint32)
        out = []
        for i in range(k):
            r0, r1 = int(r[2 + i]), int(r[3 + i])
            j0, j1 = int(r[3 + k + i]), int(r[4 + k + i])
            out.append((rpt[r0:r1 + 1] - np.uint64(j0), rows[r0:r1], cols[j0:j1]))
        return out
