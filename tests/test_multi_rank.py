"""Row-sharded A*B across ranks (clbool_b200.sharded): world_size-2 process
groups on the gloo backend (CPU, no GPU needed) for the host protocol, and
the sharded entry point on one GPU.

The protocol: every rank takes a contiguous block of A's stored rows
balanced by products (sharded.partition), multiplies it against the whole
B, all-gathers its block's (nzr, nnz) (sharded.allgather_counts) and turns
the gathered sizes into its first C row and column position
(sharded.global_offsets).  On CPU the blocks are multiplied by the oracle;
the test checks that the blocks partition the rows, that their products are
balanced, that every rank derives the same offsets, and that the blocks
placed at those offsets (sharded.assemble) are exactly the full product."""
import os
import socket

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    from clbool_b200 import gen, sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, c = gen.rmat(12, seed=3)
        n = 1 << 12
        A = O.coo_to_dcsr(O.Coo(n, n, r, c))
        work = O.workload(A, A).astype(np.int64)
        blocks = sharded.partition(work, world)
        lo, hi = blocks[rank]
        rpt = np.asarray(A.rpt, np.uint64)
        sub = O.Dcsr(n, n, (rpt[lo:hi + 1] - rpt[lo]).astype(np.uint64), np.asarray(A.rows)[lo:hi],
                     np.asarray(A.cols)[int(rpt[lo]):int(rpt[hi])])
        C = O.spgemm(sub, A) if hi > lo else O.Dcsr(n, n, np.zeros(1, np.uint64), np.zeros(0, np.uint32),
                                                     np.zeros(0, np.uint32))
        counts = sharded.allgather_counts(len(C.rows) if len(C.cols) else 0, len(C.cols))
        offs, nzr, nnz = sharded.global_offsets(counts)
        part = {"blocks": blocks, "products": int(work[lo:hi].sum()), "offsets": offs, "nzr": nzr, "nnz": nnz,
                "rows": np.asarray(C.rows).tolist(), "rpt": np.asarray(C.rpt, np.int64).tolist(),
                "cols": np.asarray(C.cols).tolist()}
        parts = [None] * world
        dist.all_gather_object(parts, part)
        if rank == 0:
            q.put(parts)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_row_shards_reassemble_the_product():
    import torch.multiprocessing as mp

    from clbool_b200 import gen, sharded
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    parts = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    r, c = gen.rmat(12, seed=3)
    n = 1 << 12
    A = O.coo_to_dcsr(O.Coo(n, n, r, c))
    want = O.spgemm(A, A)
    work = O.workload(A, A).astype(np.int64)
    blocks = parts[0]["blocks"]
    # the blocks partition A's stored rows, in order, with balanced products
    assert blocks[0][0] == 0 and blocks[-1][1] == len(A.rows)
    assert all(blocks[k][1] == blocks[k + 1][0] for k in range(world - 1))
    prods = [p["products"] for p in parts]
    assert sum(prods) == int(work.sum())
    assert max(prods) <= int(work.sum()) / world + int(work.max())
    # every rank derived the same offsets, and the blocks placed there are C
    assert all(p["offsets"] == parts[0]["offsets"] and p["nnz"] == len(want.cols) for p in parts)
    for k, p in enumerate(parts):
        assert p["offsets"][k][1] == int(want.rpt[p["offsets"][k][0]]) if p["cols"] else True
    rpt, rows, cols = sharded.assemble([(p["rpt"], p["rows"], p["cols"]) for p in parts])
    assert np.array_equal(rows, want.rows)
    assert np.array_equal(rpt, np.asarray(want.rpt, np.uint64))
    assert np.array_equal(cols, want.cols)


def test_partition_and_offsets_edge_cases():
    from clbool_b200 import sharded
    assert sharded.partition(np.zeros(0, np.int64), 4) == [(0, 0)] * 4
    assert sharded.partition(np.array([5, 0, 0]), 1) == [(0, 3)]
    b = sharded.partition(np.array([100, 1, 1, 1]), 3)  # one heavy row: later ranks may get nothing
    assert b[0][0] == 0 and b[-1][1] == 4 and all(lo <= hi for lo, hi in b)
    assert all(b[k][1] == b[k + 1][0] for k in range(2))
    offs, nzr, nnz = sharded.global_offsets([(3, 10), (0, 0), (2, 5)])
    assert offs == [(0, 0), (3, 10), (3, 10)] and (nzr, nnz) == (5, 15)


@pytest.mark.gpu
def test_blocks_on_one_gpu_reassemble_the_product(controls):
    """Every rank's block of a 4-way split computed in turn on one GPU
    (sharded.multiply_block, no collective), exact and learned forms."""
    from clbool_b200 import gen, sharded, sizing
    from util import to_device
    r, c = gen.rmat(13, seed=4)
    n = 1 << 13
    a = O.coo_to_dcsr(O.Coo(n, n, r, c))
    want = O.spgemm(a, a)
    A = to_device(controls, a)
    for sizer in (None, sizing.RowSizer.load(controls)):
        parts = []
        for rank in range(4):
            blk, rows, _ = sharded.multiply_block(controls, A, A, rank, 4, sizer=sizer)
            if blk.nnz():
                h = __import__("clbool_b200").matrix_dcsr_from_gpu(controls, blk)
                parts.append((h.rpt, h.rows, h.cols))
        rpt, rows, cols = sharded.assemble(parts)
        assert np.array_equal(rows, want.rows) and np.array_equal(cols, want.cols)
        assert np.array_equal(rpt, np.asarray(want.rpt, np.uint64))


@pytest.mark.gpu
def test_sharded_entry_point_single_rank(controls):
    """matrix_multiplication_sharded over a one-rank NCCL group: the
    broadcasts, the block and the all-gathered offsets."""
    import torch
    import torch.distributed as dist

    import clbool_b200 as cb
    from clbool_b200 import gen, sharded
    from util import to_device
    r, c = gen.rmat(12, seed=6)
    n = 1 << 12
    a = O.coo_to_dcsr(O.Coo(n, n, r, c))
    want = O.spgemm(a, a)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1)
    try:
        A = to_device(controls, a)
        part = sharded.matrix_multiplication_sharded(controls, A, A)
        assert (part.row_offset, part.nnz_offset, part.nnz) == (0, 0, len(want.cols))
        assert part.rows == (0, len(a.rows))
        h = cb.matrix_dcsr_from_gpu(controls, part.block)
        assert np.array_equal(h.cols, want.cols) and np.array_equal(h.rows, want.rows)
        B = sharded.broadcast_dcsr(controls, A, src=0)
        assert B is A
    finally:
        dist.destroy_process_group()
