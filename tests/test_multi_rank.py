"""Row sharding of A*B across ranks, as bench.py runs it under torchrun:
world_size-2 process groups on the gloo backend (CPU, no GPU needed).

Every rank takes a contiguous block of A's stored rows balanced by products
(bench.shard_rows) and multiplies it against the whole B; no collective
touches the data.  The test checks on the oracle that the blocks partition
the rows, that their products are balanced, and that the row blocks of C
gathered from the ranks are exactly the full product."""
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

    import bench
    from clbool_b200 import gen
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, c = gen.rmat(12, seed=3)
        n = 1 << 12
        A = O.coo_to_dcsr(O.Coo(n, n, r, c))
        work = O.workload(A, A).astype(np.int64)
        lo, hi = bench.shard_rows(work, world, rank)
        rpt = np.asarray(A.rpt, np.uint64)
        sub = O.Dcsr(n, n, (rpt[lo:hi + 1] - rpt[lo]).astype(np.uint64), np.asarray(A.rows)[lo:hi],
                     np.asarray(A.cols)[int(rpt[lo]):int(rpt[hi])])
        C = O.spgemm(sub, A) if hi > lo else None
        part = {"lo": lo, "hi": hi, "products": int(work[lo:hi].sum()),
                "rows": None if C is None else np.asarray(C.rows).tolist(),
                "rpt": None if C is None else np.asarray(C.rpt, np.int64).tolist(),
                "cols": None if C is None else np.asarray(C.cols).tolist()}
        parts = [None] * world
        dist.all_gather_object(parts, part)
        if rank == 0:
            q.put(parts)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_row_shards_reassemble_the_product():
    import torch.multiprocessing as mp
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    parts = q.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    from clbool_b200 import gen
    r, c = gen.rmat(12, seed=3)
    n = 1 << 12
    A = O.coo_to_dcsr(O.Coo(n, n, r, c))
    want = O.spgemm(A, A)
    # the blocks partition A's stored rows, in order
    assert parts[0]["lo"] == 0 and parts[-1]["hi"] == len(A.rows)
    assert all(parts[k]["hi"] == parts[k + 1]["lo"] for k in range(world - 1))
    # balanced by products (within one row's products of the ideal split)
    work = O.workload(A, A).astype(np.int64)
    ideal = work.sum() / world
    assert all(abs(p["products"] - ideal) <= work.max() for p in parts)
    # C's row blocks from the ranks are the full product
    rows = np.concatenate([np.asarray(p["rows"], np.uint32) for p in parts if p["rows"] is not None])
    cols = np.concatenate([np.asarray(p["cols"], np.uint32) for p in parts if p["cols"] is not None])
    assert np.array_equal(rows, want.rows) and np.array_equal(cols, want.cols)
    lens = np.concatenate([np.diff(np.asarray(p["rpt"], np.int64)) for p in parts if p["rpt"] is not None])
    assert np.array_equal(lens, np.diff(np.asarray(want.rpt, np.int64)))


def test_shard_rows_edge_cases():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.shard_rows(np.zeros(0, np.int64), 4, 2) == (0, 0)
    w = np.array([5, 0, 0, 7, 1], np.int64)
    assert bench.shard_rows(w, 1, 0) == (0, 5)
    blocks = [bench.shard_rows(w, 3, r) for r in range(3)]
    assert blocks[0][0] == 0 and blocks[-1][1] == 5
    assert all(blocks[k][1] == blocks[k + 1][0] for k in range(2))
