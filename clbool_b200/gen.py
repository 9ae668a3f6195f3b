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


def _rows_without_replacement(lens: np.ndarray, ncols: int, rng: np.random.Generator):
    lens = np.minimum(lens.astype(np.int64), ncols)
    total = int(lens.sum())
    rows = np.repeat(np.arange(lens.size, dtype=np.uint32), lens)
    cols = np.empty(total, dtype=np.uint32)
    off = 0
    # Rows are short relative to ncols: draw with replacement and redraw the
    # duplicates until every row has distinct columns.
    for i, L in enumerate(lens):
        if L == 0:
            continue
        if L * 4 > ncols:
            pick = rng.choice(ncols, size=L, replace=False)
        else:
            pick = np.unique(rng.integers(0, ncols, size=L + L // 4 + 4))
            while pick.size < L:
                pick = np.unique(np.concatenate([pick, rng.integers(0, ncols, size=L)]))
            pick = rng.permutation(pick)[:L]
        cols[off:off + L] = np.sort(pick)
        off += L
    return rows, cols


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
