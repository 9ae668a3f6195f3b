"""Learned row sizing for the single-pass SpGEMM (no counterpart in the reference).

``RowSizer`` owns a row-size predictor on the device: an MLP 6 -> 64 -> 64 -> 1
(ReLU, BF16 weights, FP32 accumulation) that maps six features of an A row to
log2(1 + nnz(C row)) / 16.  Training (forward, backward, Adam) and inference
run in the library's CUDA kernels; this module only moves arrays and files.

``matrix_multiplication_learned`` is C = A*B with one numeric pass into
predicted capacities; a row over its slot goes to a spill arena in the same
pass (or, where its count comes too late, is recomputed by the exact
two-pass form), so the result is always identical to
``dcsr.matrix_multiplication_hash``.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from ._capi import clb_dcsr, clb_spgemm_stats, lib
from .core import ClBoolException, Controls, DeviceBuffer, check, matrix_dcsr

NUM_FEATURES = 6
FEATURE_SCALE = 1.0 / 16.0
# Trained on R-MAT A*A (scales 14-19); and on R-MAT plus power-law, uniform
# and closure-step products (for workloads whose rows collide less).
DEFAULT_CHECKPOINT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sizer_rmat.npz")
MIXED_CHECKPOINT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sizer_mixed.npz")
# Capacity = predicted size * 2^margin_log2 + slack (clamped to the exact bound).
DEFAULT_MARGIN_LOG2 = 0.25
DEFAULT_SLACK = 8.0


def num_params() -> int:
    return int(lib.clb_sizer_num_params())


def targets_from_row_nnz(row_nnz: np.ndarray) -> np.ndarray:
    """Training target of every row: log2(1 + nnz) / 16 (FP32)."""
    return (np.log2(1.0 + np.asarray(row_nnz, dtype=np.float64)) * FEATURE_SCALE).astype(np.float32)


def row_features(controls: Controls, a: matrix_dcsr, b: matrix_dcsr):
    """Features of every A row of A*B -> (DeviceBuffer f32[nzr*6], DeviceBuffer u32[nzr] products)."""
    n = max(a.nzr(), 1)
    feat = DeviceBuffer.empty(controls, n * NUM_FEATURES, np.float32)
    work = DeviceBuffer.empty(controls, n, np.uint32)
    sa, sb = a.c_struct(), b.c_struct()
    check(lib.clb_dcsr_row_features(controls.handle, C.byref(sa), C.byref(sb), C.c_void_p(feat.ptr),
                                    C.c_void_p(work.ptr)), "row_features")
    return feat, work


def row_nnz(controls: Controls, a: matrix_dcsr, b: matrix_dcsr) -> DeviceBuffer:
    """Exact nnz of every row of A*B (symbolic pass only), u32[nzr_A] on the device."""
    out = DeviceBuffer.empty(controls, max(a.nzr(), 1), np.uint32)
    sa, sb = a.c_struct(), b.c_struct()
    check(lib.clb_dcsr_row_nnz(controls.handle, C.byref(sa), C.byref(sb), C.c_void_p(out.ptr)), "row_nnz")
    return out


class RowSizer:
    """Device-resident row-size predictor with its Adam state."""

    def __init__(self, controls: Controls, seed: int = 1, params: np.ndarray | None = None):
        self.controls = controls
        h = C.c_void_p()
        check(lib.clb_sizer_create(controls.handle, int(seed), C.byref(h)), "sizer_create")
        self.handle = h
        if params is not None:
            self.set_params(params)

    def close(self) -> None:
        if self.handle:
            lib.clb_sizer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -------------------------------------------------------- parameters --
    def get_params(self) -> np.ndarray:
        out = np.empty(num_params(), np.float32)
        check(lib.clb_sizer_get_params(self.handle, out.ctypes.data_as(C.c_void_p), out.size), "sizer_get_params")
        return out

    def set_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        check(lib.clb_sizer_set_params(self.handle, p.ctypes.data_as(C.c_void_p), p.size), "sizer_set_params")

    def save(self, path: str, meta: dict | None = None) -> None:
        """Checkpoint: FP32 master weights plus a JSON metadata string."""
        np.savez(path, params=self.get_params(), meta=np.array(json.dumps(meta or {})))

    @classmethod
    def load(cls, controls: Controls, path: str = DEFAULT_CHECKPOINT) -> "RowSizer":
        with np.load(path) as z:
            params = z["params"]
        if params.size != num_params():
            raise ClBoolException(13, f"{path}: {params.size} parameters, expected {num_params()}")
        return cls(controls, params=params)

    @staticmethod
    def checkpoint_meta(path: str = DEFAULT_CHECKPOINT) -> dict:
        with np.load(path) as z:
            return json.loads(str(z["meta"]))

    # ---------------------------------------------------------- compute --
    def predict(self, features: DeviceBuffer, n: int) -> DeviceBuffer:
        out = DeviceBuffer.empty(self.controls, max(n, 1), np.float32)
        check(lib.clb_sizer_predict(self.handle, C.c_void_p(features.ptr), int(n), C.c_void_p(out.ptr)),
              "sizer_predict")
        return out

    def gradients(self, features: DeviceBuffer, targets: DeviceBuffer, n: int):
        """(loss, grads[num_params]) of the MSE over n rows w.r.t. the BF16-rounded weights."""
        g = np.empty(num_params(), np.float32)
        loss = C.c_float()
        check(lib.clb_sizer_gradients(self.handle, C.c_void_p(features.ptr), C.c_void_p(targets.ptr), int(n),
                                      g.ctypes.data_as(C.c_void_p), C.byref(loss)), "sizer_gradients")
        return float(loss.value), g

    def train(self, features: DeviceBuffer, targets: DeviceBuffer, n: int, epochs: int = 20, batch: int = 4096,
              lr: float = 1e-3, seed: int = 1) -> float:
        """Adam over n rows (device arrays); returns the loss of the last mini-batch."""
        loss = C.c_float()
        check(lib.clb_sizer_train(self.handle, C.c_void_p(features.ptr), C.c_void_p(targets.ptr), int(n),
                                  int(epochs), int(batch), float(lr), int(seed), C.byref(loss)), "sizer_train")
        return float(loss.value)


def matrix_multiplication_learned(controls: Controls, matrix_out: matrix_dcsr | None, a: matrix_dcsr,
                                  b: matrix_dcsr, sizer: RowSizer, margin_log2: float = DEFAULT_MARGIN_LOG2,
                                  slack: float = DEFAULT_SLACK, stats: dict | None = None,
                                  tune=None) -> matrix_dcsr:
    """C = A*B (boolean) in one numeric pass sized by `sizer`; exact.
    `tune` (optional, batched.tuning(...)) sets the accumulators."""
    out = clb_dcsr()
    st = clb_spgemm_stats()
    sa, sb = a.c_struct(), b.c_struct()
    check(lib.clb_dcsr_spgemm_learned(controls.handle, C.byref(sa), C.byref(sb), sizer.handle, float(margin_log2),
                                      float(slack), C.byref(tune) if tune is not None else None, C.byref(out),
                                      C.byref(st)), "matrix_multiplication_learned")
    res = matrix_dcsr.adopt(controls, out)
    if stats is not None:
        stats.update(st.as_dict())
    return res if matrix_out is None else matrix_out._assign(res)


def matrix_multiplication_to_host(controls: Controls, a: matrix_dcsr, b: matrix_dcsr, h_rpt, h_rows, h_cols,
                                  rows_capacity: int, cols_capacity: int, sizer: RowSizer | None = None,
                                  margin_log2: float = DEFAULT_MARGIN_LOG2, slack: float = DEFAULT_SLACK,
                                  blocks: int = 8, tune=None, stats: dict | None = None):
    """C = A*B written into host arrays (numpy arrays or raw addresses of
    page-locked buffers): row blocks of A are multiplied in turn (learned form
    when `sizer` is given, else the tuned form) while the previous block's
    rows are copied out.  Returns (nzr, nnz)."""
    def addr(x):
        return C.c_void_p(x.ctypes.data if isinstance(x, np.ndarray) else int(x))
    nzr, nnz = C.c_uint64(), C.c_uint64()
    st = clb_spgemm_stats()
    sa, sb = a.c_struct(), b.c_struct()
    check(lib.clb_dcsr_spgemm_to_host(controls.handle, C.byref(sa), C.byref(sb), sizer.handle if sizer else None,
                                      float(margin_log2), float(slack), C.byref(tune) if tune is not None else None,
                                      int(blocks), addr(h_rpt), addr(h_rows), addr(h_cols), int(rows_capacity),
                                      int(cols_capacity), C.byref(nzr), C.byref(nnz), C.byref(st)),
          "matrix_multiplication_to_host")
    if stats is not None:
        stats.update(st.as_dict())
    return int(nzr.value), int(nnz.value)
