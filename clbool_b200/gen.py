"""Seeded synthetic workloads (host, numpy).

* ``rmat``: R-MAT graph (Chakrabarti et al. 2004): every edge descends
  ``scale`` levels of the adjacency matrix, picking quadrant (0,0), (0,1),
  (1,0), (1,1) with probabilities a, b, c, d.  Duplicates removed, self-loops
  kept, no vertex relabelling.
* ``poisson_rows``: every row draws its length from Poisson(lam) and its
  columns uniformly without replacement (sorted).
* ``power_law_rows``: row lengths from a discrete power law with a given
  exponent, mean and cap; columns uniform without replacement.

All generators return sorted unique COO pairs as uint32 arrays; use
``to_dcsr`` / ``to_csr`` for the other formats.
"""
from __future__ import annotations

import numpy as np


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1):
    n_edges = edge_factor << scale
    rng = np.random.default_rng(seed)
    src = np.zeros(n_edges, dtype=np.uint32)
    dst = np.zeros(n_edges, dtype=np.uint32)
    # quadrant thresholds on a uniform 32-bit draw
    ta, tab, tabc = (np.uint32(min(int(x * 2 ** 32), 2 ** 32 - 1)) for x in (a, a + b, a + b + c))
    for level in range(scale):
        u = rng.integers(0, 1 << 32, size=n_edges, dtype=np.uint32)
        sh = scale - 1 - level
        down = u >= tab                                 # quadrants (1,0), (1,1)
        right = ((u >= ta) & (u < tab)) | (u >= tabc)   # quadrants (0,1), (1,1)
        src |= down.view(np.uint8).astype(np.uint32) << sh
        dst |= right.view(np.uint8).astype(np.uint32) << sh
    key = (src.astype(np.uint64) << np.uint64(32)) | dst
    key.sort()
    key = key[np.concatenate([[True], key[1:] != key[:-1]])]
    return (key >> np.uint64(32)).astype(np.uint32), (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def _sorted_unique(a: np.ndarray) -> np.ndarray:
    a = np.sort(a)
    if a.size < 2:
        return a
    return a[np.concatenate([[True], a[1:] != a[:-1]])]


def _rows_without_replacement(lens: np.ndarray, ncols: int, rng: np.random.Generator):
    """Sorted COO with exactly lens[i] distinct columns in row i (uniform
    without replacement), vectorised: draw with replacement, drop duplicate
    (row, col) pairs, redraw the missing ones until every row is full."""
    lens = np.minimum(np.asarray(lens, dtype=np.int64), ncols)
    nrows = lens.size
    # rows longer than half the columns: drawn one by one without replacement
    dense = np.flatnonzero(lens * 2 > ncols)
    dkeys = [r * ncols + np.sort(rng.choice(ncols, size=int(lens[r]), replace=False)) for r in dense]
    sparse = lens.copy()
    sparse[dense] = 0
    rows = np.repeat(np.arange(nrows, dtype=np.int64), sparse)
    keys = _sorted_unique(rows * ncols + rng.integers(0, ncols, size=rows.size))
    for _ in range(200):
        have = np.bincount(keys // ncols, minlength=nrows)
        short = sparse - have
        if not short.any():
            break
        extra = np.repeat(np.arange(nrows, dtype=np.int64), short)
        keys = _sorted_unique(np.concatenate([keys, extra * ncols + rng.integers(0, ncols, size=extra.size)]))
    else:
        raise RuntimeError("row generation did not converge")
    if dkeys:
        keys = np.sort(np.concatenate([keys] + dkeys))
    return (keys // ncols).astype(np.uint32), (keys % ncols).astype(np.uint32)


def poisson_rows(nrows: int, ncols: int, lam: float = 8.0, seed: int = 1):
    rng = np.random.default_rng(seed)
    lens = rng.poisson(lam, size=nrows)
    return _rows_without_replacement(lens, ncols, rng)


def power_law_rows(nrows: int, ncols: int, exponent: float = 2.1, mean: float = 6.0, cap: int = 4096,
                   seed: int = 1):
    """Row lengths k >= 1 with P(k) ~ k^-exponent, truncated at `cap`, then
    scaled to the requested mean."""
    rng = np.random.default_rng(seed)
    k = np.arange(1, cap + 1, dtype=np.float64)
    p = k ** (-exponent)
    p /= p.sum()
    lens = rng.choice(k.astype(np.int64), size=nrows, p=p)
    scale = mean / max(lens.mean(), 1e-9)
    lens = np.clip(np.rint(lens * scale), 0, cap).astype(np.int64)
    return _rows_without_replacement(lens, ncols, rng)


def to_dcsr(rows: np.ndarray, cols: np.ndarray):
    """Sorted unique COO -> (rpt uint64[nzr+1], rows uint32[nzr], cols uint32[nnz])."""
    rows = np.asarray(rows, dtype=np.uint32)
    cols = np.asarray(cols, dtype=np.uint32)
    if rows.size == 0:
        return np.zeros(1, np.uint64), np.zeros(0, np.uint32), cols
    start = np.flatnonzero(np.concatenate([[True], rows[1:] != rows[:-1]]))
    rpt = np.concatenate([start, [rows.size]]).astype(np.uint64)
    return rpt, rows[start].copy(), cols


def to_csr(rows: np.ndarray, cols: np.ndarray, nrows: int):
    rows = np.asarray(rows, dtype=np.uint32)
    rpt = np.zeros(nrows + 1, dtype=np.uint64)
    if rows.size:
        np.cumsum(np.bincount(rows, minlength=nrows)[:nrows], out=rpt[1:])
    return rpt, np.asarray(cols, dtype=np.uint32)
