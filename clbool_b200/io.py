"""Binary DCSR files with a checksum (host <-> file <-> device), so callers
can feed matrices without a generator; the file-side companion of the
reference's matrix_dcsr_from_cpu / matrix_dcsr_from_gpu
(src/common/matrices_conversions.cpp:93-139), which this module uses.

Layout (little endian):
    magic    8 bytes  b"CLBDCSR1"
    nrows    u64
    ncols    u64
    nnz      u64
    nzr      u64
    rpt      u64[nzr + 1]      (absent when nnz == 0)
    rows     u32[nzr]
    cols     u32[nnz]
    sha256   32 bytes over everything above

`include/clbool/clbool.hpp` reads and writes the same format
(clbool::io::save_dcsr / load_dcsr).
"""
from __future__ import annotations

import hashlib
import struct

import numpy as np

from .core import ClBoolException, Controls, matrix_dcsr, matrix_dcsr_cpu
from .ops import matrix_dcsr_from_cpu, matrix_dcsr_from_gpu

MAGIC = b"CLBDCSR1"


def save(path: str, nrows: int, ncols: int, rpt, rows, cols) -> None:
    """Writes a host DCSR (rpt may be u32 or u64)."""
    cols = np.ascontiguousarray(cols, dtype="<u4")
    rows = np.ascontiguousarray(rows, dtype="<u4")
    nnz, nzr = cols.size, rows.size if cols.size else 0
    body = MAGIC + struct.pack("<4Q", nrows, ncols, nnz, nzr)
    if nnz:
        rpt = np.ascontiguousarray(rpt, dtype="<u8")
        if rpt.size != nzr + 1 or int(rpt[-1]) != nnz:
            raise ClBoolException(13, "rpt does not match rows / cols")
        body += rpt.tobytes() + rows[:nzr].tobytes() + cols.tobytes()
    with open(path, "wb") as f:
        f.write(body + hashlib.sha256(body).digest())


def load(path: str):
    """(nrows, ncols, rpt u64, rows u32, cols u32); raises on a bad checksum."""
    with open(path, "rb") as f:
        data = f.read()
    if len(data) < 8 + 32 + 32 or data[:8] != MAGIC:
        raise ClBoolException(13, f"{path}: not a DCSR file")
    body, digest = data[:-32], data[-32:]
    if hashlib.sha256(body).digest() != digest:
        raise ClBoolException(13, f"{path}: checksum mismatch")
    nrows, ncols, nnz, nzr = struct.unpack_from("<4Q", body, 8)
    off = 40
    if nnz == 0:
        return nrows, ncols, np.zeros(1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint32)
    need = off + 8 * (nzr + 1) + 4 * nzr + 4 * nnz
    if len(body) != need:
        raise ClBoolException(13, f"{path}: truncated")
    rpt = np.frombuffer(body, dtype="<u8", count=nzr + 1, offset=off).astype(np.uint64)
    off += 8 * (nzr + 1)
    rows = np.frombuffer(body, dtype="<u4", count=nzr, offset=off).astype(np.uint32)
    off += 4 * nzr
    cols = np.frombuffer(body, dtype="<u4", count=nnz, offset=off).astype(np.uint32)
    return nrows, ncols, rpt, rows, cols


def save_device(controls: Controls, path: str, m: matrix_dcsr) -> None:
    if m.nnz() == 0:
        save(path, m.nrows(), m.ncols(), np.zeros(1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint32))
        return
    h = matrix_dcsr_from_gpu(controls, m)
    save(path, m.nrows(), m.ncols(), h.rpt, h.rows, h.cols)


def load_device(controls: Controls, path: str) -> matrix_dcsr:
    nrows, ncols, rpt, rows, cols = load(path)
    if cols.size == 0:
        return matrix_dcsr.zeros(nrows, ncols)
    return matrix_dcsr_from_cpu(controls, matrix_dcsr_cpu(rpt, rows, cols), nrows, ncols)
