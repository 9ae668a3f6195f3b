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


# ------------------------------------------------- checks at full sizes --
CHUNK = 1 << 28  # elements per device comparison


class _Cai:
    """A device array seen by torch without a copy (__cuda_array_interface__)."""

    def __init__(self, ptr: int, n: int, dtype):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": np.dtype(dtype).str,
                                         "data": (int(ptr), False), "version": 3}


def device_view(buf, n, dtype):
    """Signed torch view of a device buffer (torch compares signed integers;
    u32 columns < 2^31 and u64 offsets < 2^63 keep their order, and equality
    is bitwise either way)."""
    import torch
    signed = {np.dtype(np.uint32): np.int32, np.dtype(np.uint64): np.int64}[np.dtype(dtype)]
    return torch.as_tensor(_Cai(buf.ptr, n, signed), device="cuda")


def same_on_device(x, y, what):
    """Two device DCSR matrices hold identical arrays (compared on the GPU)."""
    assert (x.nnz(), x.nzr()) == (y.nnz(), y.nzr()), what
    for get, n, dt in ((lambda m: m.rpt_gpu(), x.nzr() + 1, np.uint64), (lambda m: m.rows_gpu(), x.nzr(), np.uint32),
                       (lambda m: m.cols_gpu(), x.nnz(), np.uint32)):
        if n == 0:
            continue
        a, b = device_view(get(x), n, dt), device_view(get(y), n, dt)
        for s in range(0, n, CHUNK):
            assert bool((a[s:s + CHUNK] == b[s:s + CHUNK]).all()), f"{what}: differs in [{s}, {s + CHUNK})"


def rows_strictly_increasing(m, rpt_host, what):
    """Every row of the device matrix m is strictly increasing: a
    non-increase of the column array may only sit at a row start."""
    import torch
    if m.nnz() < 2:
        return
    cols = device_view(m.cols_gpu(), m.nnz(), np.uint32)
    starts = torch.as_tensor(np.asarray(rpt_host[1:-1], np.int64), device="cuda")
    for s in range(0, m.nnz() - 1, CHUNK):
        e = min(s + CHUNK + 1, m.nnz())
        bad = torch.nonzero(cols[s + 1:e] <= cols[s:e - 1]).flatten() + (s + 1)
        assert bool(torch.isin(bad, starts).all()), f"{what}: a row is not strictly increasing"


def sub_rows(a: O.Dcsr, pick) -> O.Dcsr:
    """The stored rows `pick` (indices into a.rows, sorted) of a, same shape."""
    pick = np.asarray(pick, np.int64)
    arpt = np.asarray(a.rpt, np.int64)
    if pick.size and pick[-1] - pick[0] + 1 == pick.size:  # a contiguous block: slices
        lo, hi = int(pick[0]), int(pick[-1]) + 1
        return O.Dcsr(a.nrows, a.ncols, (arpt[lo:hi + 1] - arpt[lo]).astype(np.uint64),
                      np.asarray(a.rows)[lo:hi], np.asarray(a.cols)[arpt[lo]:arpt[hi]])
    lens = arpt[pick + 1] - arpt[pick]
    rpt = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    idx = np.repeat(arpt[pick] - rpt[:-1], lens) + np.arange(int(rpt[-1]), dtype=np.int64)
    return O.Dcsr(a.nrows, a.ncols, rpt.astype(np.uint64), np.asarray(a.rows)[pick], np.asarray(a.cols)[idx])


def weighted_pick(weights, count: int, seed: int, uniform: int = 0):
    """`count` stored rows drawn without replacement with probability
    proportional to `weights` (the rows that carry the work), plus `uniform`
    rows drawn uniformly; sorted, distinct."""
    w = np.asarray(weights, np.float64)
    rng = np.random.default_rng(seed)
    nz = np.flatnonzero(w > 0)
    k = min(count, nz.size)
    heavy = rng.choice(nz, size=k, replace=False, p=w[nz] / w[nz].sum()) if k else np.zeros(0, np.int64)
    light = rng.choice(w.size, size=min(uniform, w.size), replace=False) if uniform else np.zeros(0, np.int64)
    return np.unique(np.concatenate([heavy, light]).astype(np.int64))


def assert_rows_match(ctl, m, want: O.Dcsr, what: str):
    """Every stored row of `want` is a stored row of the device matrix m with
    the same columns (the rows are read one by one from the device)."""
    import ctypes

    import clbool_b200 as cb
    rpt = m.rpt_gpu().to_host(m.nzr() + 1).astype(np.int64)
    rows = m.rows_gpu().to_host(m.nzr())
    idx = np.searchsorted(rows, want.rows)
    assert np.all(idx < rows.size) and np.array_equal(rows[idx], want.rows), f"{what}: rows missing"
    for k, g in enumerate(idx):
        lo, hi = int(rpt[g]), int(rpt[g + 1])
        seg = np.empty(hi - lo, np.uint32)
        assert cb.lib.clb_memcpy_d2h(ctl.handle, seg.ctypes.data_as(ctypes.c_void_p),
                                     ctypes.c_void_p(m.cols_gpu().ptr + 4 * lo), 4 * (hi - lo)) == 0
        assert np.array_equal(seg, want.cols[int(want.rpt[k]):int(want.rpt[k + 1])]), f"{what}: row {want.rows[k]}"
