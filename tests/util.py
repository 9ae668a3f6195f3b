"""Shared helpers of the test suite: moving matrices between the oracle's
host tuples and the library's device matrices, digests, comparisons."""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")


def golden() -> dict:
    with open(GOLDEN) as f:
        return json.load(f)["cases"]


def sha(a, dtype) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


def dcsr_digest(m) -> dict:
    nnz = len(m.cols)
    rpt = np.asarray(m.rpt, np.uint64) if nnz else np.zeros(0, np.uint64)
    return {"nnz": nnz, "nzr": len(m.rows) if nnz else 0, "rpt": sha(rpt, np.uint64),
            "rows": sha(m.rows if nnz else [], np.uint32), "cols": sha(m.cols, np.uint32)}


def coo_digest(rows, cols) -> dict:
    return {"nnz": len(rows), "rows": sha(rows, np.uint32), "cols": sha(cols, np.uint32)}


def csr_digest(c) -> dict:
    return {"nnz": len(c.cols), "rpt": sha(c.rpt, np.uint64), "cols": sha(c.cols, np.uint32)}


def pairs_dcsr(size: int, k: int, ncols: int | None = None) -> O.Dcsr:
    """The reference tests' input: generate_coo_pairs_cpu(size*k, size) as DCSR."""
    r, c = O.generate_coo_pairs(size * k, size)
    return O.coo_to_dcsr(O.Coo(size, size if ncols is None else ncols, r, c))


# ------------------------------------------------------------ device side --
def to_device(ctl, m: O.Dcsr):
    import clbool_b200 as cb
    return cb.matrix_dcsr_from_cpu(ctl, cb.matrix_dcsr_cpu(m.rpt, m.rows, m.cols), m.nrows, m.ncols)


def from_device(ctl, m) -> O.Dcsr:
    import clbool_b200 as cb
    h = cb.matrix_dcsr_from_gpu(ctl, m)
    if m.nnz() == 0:
        return O.Dcsr(m.nrows(), m.ncols(), np.zeros(1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    return O.Dcsr(m.nrows(), m.ncols(), h.rpt, h.rows, h.cols)


def assert_dcsr_equal(got: O.Dcsr, want: O.Dcsr, what: str = ""):
    assert got.nrows == want.nrows and got.ncols == want.ncols, f"{what}: shape"
    assert len(got.cols) == len(want.cols), f"{what}: nnz {len(got.cols)} != {len(want.cols)}"
    if len(want.cols) == 0:
        return
    assert np.array_equal(np.asarray(got.rows), np.asarray(want.rows)), f"{what}: rows differ"
    assert np.array_equal(np.asarray(got.rpt, np.uint64), np.asarray(want.rpt, np.uint64)), f"{what}: rpt differ"
    assert np.array_equal(np.asarray(got.cols), np.asarray(want.cols)), f"{what}: cols differ"
