"""Boolean SpGEMM with A's rows split over the GPUs of one node (no
counterpart in the reference, a single-device library whose Controls hold
one device: src/core/controls.hpp:12-28).

C = A*B shards by independent row blocks: the stored rows of A are cut into
contiguous blocks of about equal products (the workload pass,
count_workload, src/dcsr/dcsr_matrix_multiplication.cpp:388-404), rank r
multiplies block r against its own copy of B in its own HBM, and the ranks
exchange only sizes.  One process per GPU over a torch.distributed process
group (NCCL between GPUs, gloo for host-only tests):

  * ``broadcast_dcsr``: a matrix from one rank into every rank's device
    memory (its sizes first, then its three arrays, NCCL broadcasts over
    NVLink);
  * ``partition``: the row blocks, from the products of A's rows;
  * ``global_offsets``: every rank's first C row and first C column
    position from the all-gathered (nzr, nnz) of the blocks;
  * ``multiply_block``: one rank's block, no collective (so one GPU can also
    compute every block in turn);
  * ``matrix_multiplication_sharded``: the three steps together.

C stays sharded: rank r holds rows [row_offset, row_offset + nzr) of C's
stored rows, whose columns start at nnz_offset in C; ``assemble`` joins host
copies of the blocks into the whole C.  Every load of every kernel reads the
rank's own memory: B and A arrive by NCCL broadcasts, never as peer-memory
operands.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._capi import clb_dcsr, lib
from .core import Controls, DeviceBuffer, check, matrix_dcsr
from .ops import matrix_multiplication_hash, workload


def partition(work: np.ndarray, world: int) -> list[tuple[int, int]]:
    """Contiguous blocks [lo, hi) of A's stored rows, one per rank, each
    with about 1/world of the products (the cut lands after the row whose
    running sum first reaches q/world of the total)."""
    work = np.asarray(work, dtype=np.int64)
    n = int(work.size)
    if world <= 1:
        return [(0, n)]
    cum = np.cumsum(work, dtype=np.float64)
    tot = float(cum[-1]) if n else 0.0
    cuts = [0]
    for q in range(1, world):
        c = int(np.searchsorted(cum, tot * q / world, side="left")) + 1 if n else 0
        cuts.append(min(max(c, cuts[-1]), n))
    cuts.append(n)
    return [(cuts[k], cuts[k + 1]) for k in range(world)]


def global_offsets(counts) -> tuple[list[tuple[int, int]], int, int]:
    """([(row_offset, nnz_offset) per rank], total nzr, total nnz) from the
    per-rank (nzr, nnz) of the blocks, in rank order."""
    offs, r, j = [], 0, 0
    for nzr, nnz in counts:
        offs.append((r, j))
        r += int(nzr)
        j += int(nnz)
    return offs, r, j


def row_block(controls: Controls, a: matrix_dcsr, lo: int, hi: int) -> matrix_dcsr:
    """Stored rows [lo, hi) of A (device copy, row ids kept)."""
    out = clb_dcsr()
    sa = a.c_struct()
    check(lib.clb_dcsr_row_block(controls.handle, C.byref(sa), int(lo), int(hi), C.byref(out)), "row_block")
    return matrix_dcsr.adopt(controls, out)


@dataclass
class ShardedProduct:
    """One rank's share of C = A*B."""
    block: matrix_dcsr          # C's rows of this rank's A rows (device)
    rows: tuple[int, int]       # the block of A's stored rows
    row_offset: int             # its first stored row within C
    nnz_offset: int             # its first column position within C
    nzr: int                    # C's stored rows, all ranks
    nnz: int                    # C's entries, all ranks
    products: int               # products of this rank's rows


def multiply_block(controls: Controls, a: matrix_dcsr, b: matrix_dcsr, rank: int, world: int, sizer=None,
                   tune=None, work: np.ndarray | None = None):
    """(block of C, (lo, hi), products) for `rank` of `world`, computed on
    controls' device without any collective."""
    if work is None:
        buf, _ = workload(controls, a, b)
        work = buf.to_host(a.nzr()).astype(np.int64) if a.nzr() else np.zeros(0, np.int64)
    lo, hi = partition(work, world)[rank]
    blk = row_block(controls, a, lo, hi)
    if sizer is not None:
        from .sizing import matrix_multiplication_learned
        c = matrix_multiplication_learned(controls, None, blk, b, sizer, tune=tune)
    elif tune is not None:
        from .batched import matrix_multiplication_tuned
        c = matrix_multiplication_tuned(controls, None, blk, b, tune)
    else:
        c = matrix_multiplication_hash(controls, None, blk, b)
    return c, (lo, hi), int(work[lo:hi].sum())


def _device_tensor(buf: DeviceBuffer, n: int, dtype, device: int):
    """A torch view of a device buffer on `device` (no copy), for the NCCL calls."""
    import torch

    class _Cai:
        def __init__(self, ptr, n, dt):
            self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": np.dtype(dt).str,
                                             "data": (int(ptr), False), "version": 3}
    signed = {np.dtype(np.uint32): np.int32, np.dtype(np.uint64): np.int64}[np.dtype(dtype)]
    return torch.as_tensor(_Cai(buf.ptr, n, signed), device=f"cuda:{device}")


def broadcast_dcsr(controls: Controls, m: matrix_dcsr | None, src: int = 0, group=None) -> matrix_dcsr:
    """`m` (given on rank `src`) in every rank's own device memory: one
    broadcast of the sizes, then one per array.  Other ranks pass None.
    The broadcasts run on torch's current stream of the controls' device,
    after the controls' stream has finished its work."""
    import torch
    with torch.cuda.device(controls.device):
        return _broadcast_dcsr(controls, m, src, group)


def _broadcast_dcsr(controls, m, src, group):
    import torch
    import torch.distributed as dist
    dev = torch.device(f"cuda:{controls.device}")
    me = dist.get_rank(group)
    head = torch.zeros(4, dtype=torch.int64, device=dev)
    if me == src:
        head[:] = torch.tensor([m.nrows(), m.ncols(), m.nnz(), m.nzr() if m.nnz() else 0], dtype=torch.int64)
        controls.sync()
    dist.broadcast(head, src, group=group)
    nrows, ncols, nnz, nzr = (int(x) for x in head.tolist())
    if nnz == 0:
        return m if me == src else matrix_dcsr.zeros(nrows, ncols)
    if me == src:
        rpt, rows, cols = m.rpt_gpu(), m.rows_gpu(), m.cols_gpu()
    else:
        rpt = DeviceBuffer.empty(controls, nzr + 1, np.uint64)
        rows = DeviceBuffer.empty(controls, nzr, np.uint32)
        cols = DeviceBuffer.empty(controls, nnz, np.uint32)
        controls.sync()
    for buf, n, dt in ((rpt, nzr + 1, np.uint64), (rows, nzr, np.uint32), (cols, nnz, np.uint32)):
        dist.broadcast(_device_tensor(buf, n, dt, controls.device), src, group=group)
    torch.cuda.synchronize(dev)
    if me == src:
        return m
    return matrix_dcsr(rpt, rows, cols, nrows, ncols, nnz, nzr)


def allgather_counts(nzr: int, nnz: int, group=None, device: str | None = None) -> list[tuple[int, int]]:
    """Every rank's (nzr, nnz), in rank order (one all-gather of 16 bytes per rank)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    t = torch.tensor([int(nzr), int(nnz)], dtype=torch.int64, device=device or "cpu")
    out = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(out, t, group=group)
    return [(int(x[0]), int(x[1])) for x in out]


def matrix_multiplication_sharded(controls: Controls, a: matrix_dcsr | None, b: matrix_dcsr | None, group=None,
                                  src: int = 0, sizer=None, tune=None) -> ShardedProduct:
    """C = A*B over the ranks of `group` (one GPU each, controls on that
    GPU): A and B given on rank `src` are broadcast into every rank's HBM
    (pass them as None elsewhere), each rank multiplies its block of A's
    rows (learned form with `sizer`, tuned form with `tune`, else the exact
    two-pass form), and the block sizes are all-gathered into global
    offsets.  Returns this rank's ShardedProduct."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    A = broadcast_dcsr(controls, a, src, group)
    B = broadcast_dcsr(controls, b, src, group)
    c, rows, products = multiply_block(controls, A, B, rank, world, sizer=sizer, tune=tune)
    backend = dist.get_backend(group)
    counts = allgather_counts(c.nzr() if c.nnz() else 0, c.nnz(), group,
                              device=None if backend == "gloo" else f"cuda:{controls.device}")
    offs, nzr, nnz = global_offsets(counts)
    return ShardedProduct(c, rows, offs[rank][0], offs[rank][1], nzr, nnz, products)


def assemble(parts) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """The whole C (rpt u64, rows u32, cols u32) from host copies of every
    rank's block in rank order: [(rpt, rows, cols), ...] with each block's
    rpt starting at 0."""
    rpts, rows, cols, base = [], [], [], 0
    for rpt, r, c in parts:
        rpt = np.asarray(rpt, np.uint64)
        if len(c) == 0:
            continue
        rpts.append(rpt[:-1] + np.uint64(base))
        rows.append(np.asarray(r, np.uint32))
        cols.append(np.asarray(c, np.uint32))
        base += len(c)
    if not cols:
        return np.zeros(1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint32)
    return (np.concatenate(rpts + [np.array([base], np.uint64)]), np.concatenate(rows), np.concatenate(cols))
