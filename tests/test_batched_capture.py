"""The host-sync-free batched product (clb_dcsr_spgemm_batched_capture) and
its replay from a CUDA graph, bit-exact against the oracle.

The product has no counterpart in the reference (which multiplies one pair
per call, src/dcsr/dcsr.hpp:27-36); each pair's result must equal the
oracle's product of that pair.  The graph test records the call once, then
changes the pairs' column indices in place (same row structure, so the same
sizes) and replays: the replay must give the new products."""
import ctypes

import numpy as np
import pytest

import oracle as O
from util import pairs_dcsr, to_device


def _random_dcsr(nrows, ncols, row_len, seed, nz_rows=None):
    rng = np.random.default_rng(seed)
    rows = np.sort(rng.choice(nrows, nz_rows or nrows, replace=False)).astype(np.uint32)
    lens = np.minimum(rng.integers(1, row_len + 1, rows.size), ncols)
    cols = np.concatenate([np.sort(rng.choice(ncols, int(l), replace=False)) for l in lens]).astype(np.uint32)
    rpt = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    return O.Dcsr(nrows, ncols, rpt, rows, cols)


def _reshuffle(m, seed):
    """Same rows and row lengths, new sorted distinct columns."""
    rng = np.random.default_rng(seed)
    lens = np.diff(m.rpt.astype(np.int64))
    parts = [np.sort(rng.choice(m.ncols, int(l), replace=False)) for l in lens]
    cols = np.concatenate(parts).astype(np.uint32) if parts else np.zeros(0, np.uint32)
    return O.Dcsr(m.nrows, m.ncols, m.rpt.copy(), m.rows.copy(), cols)


def _host_pairs(seed=0):
    from clbool_b200 import gen
    r, c = gen.rmat(10, seed=3)
    rm = O.coo_to_dcsr(O.Coo(1 << 10, 1 << 10, r, c))
    heavy_b = _random_dcsr(3000, 3000, 300, seed + 1)                 # rows over 4096 products: bitmap
    empty = O.Dcsr(50, 40, np.zeros(1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    return [
        (pairs_dcsr(300, 8), pairs_dcsr(300, 8)),
        (rm, rm),
        (_random_dcsr(200, 500, 12, seed + 2, nz_rows=150), _random_dcsr(500, 70000, 40, seed + 3)),
        (empty, _random_dcsr(40, 60, 5, seed + 4)),
        (_random_dcsr(400, 3000, 60, seed + 5, nz_rows=300), heavy_b),
        (_random_dcsr(64, 64, 3, seed + 6, nz_rows=10), _random_dcsr(64, 2, 2, seed + 7)),
    ]


def _check(got, host_pairs, what):
    for k, ((rpt, rows, cols), (a, b)) in enumerate(zip(got, host_pairs)):
        want = O.spgemm(a, b)
        if len(want.cols) == 0:
            assert len(cols) == 0 and len(rows) == 0 and list(rpt) == [0], f"{what} pair {k}: not empty"
            continue
        assert np.array_equal(cols, want.cols), f"{what} pair {k}: cols"
        assert np.array_equal(rows, want.rows), f"{what} pair {k}: rows"
        assert np.array_equal(rpt, np.asarray(want.rpt, np.uint64)), f"{what} pair {k}: rpt"


@pytest.mark.gpu
def test_capture_form_matches_oracle(controls):
    from clbool_b200 import batched
    hp = _host_pairs()
    pairs = [(to_device(controls, a), to_device(controls, b)) for a, b in hp]
    cb = batched.CapturedBatch(controls, pairs)
    for _ in range(2):  # the second call reuses the same buffers
        cb.enqueue()
        _check(cb.result(), hp, "direct")


@pytest.mark.gpu
def test_graph_replay_follows_new_contents(controls):
    import clbool_b200 as cbm
    from clbool_b200 import batched
    hp1 = _host_pairs(seed=10)
    hp2 = [(_reshuffle(a, 100 + k), _reshuffle(b, 200 + k)) for k, (a, b) in enumerate(hp1)]
    pairs = [(to_device(controls, a), to_device(controls, b)) for a, b in hp1]
    _, need2 = batched.batched_plan(controls, [(to_device(controls, a), to_device(controls, b)) for a, b in hp2])
    _, need1 = batched.batched_plan(controls, pairs)
    cap = max(need1, need2)
    batch = batched.CapturedBatch(controls, pairs, slot_capacity=cap, cols_capacity=cap)
    graph = batched.Graph(controls, batch.enqueue)
    graph.launch()
    _check(batch.result(), hp1, "graph, first contents")
    # new column indices into the same device arrays, then replay
    for (da, db), (ha, hb) in zip(pairs, hp2):
        for dev, host in ((da, ha), (db, hb)):
            if len(host.cols):
                assert cbm.lib.clb_memcpy_h2d(controls.handle, ctypes.c_void_p(dev.cols_gpu().ptr),
                                              host.cols.ctypes.data_as(ctypes.c_void_p), host.cols.nbytes) == 0
    controls.sync()
    for _ in range(2):
        graph.launch()
        _check(batch.result(), hp2, "graph replay, new contents")
    graph.close()


@pytest.mark.gpu
def test_capture_capacities_are_enforced(controls):
    from clbool_b200 import ClBoolException, batched
    hp = _host_pairs(seed=20)
    pairs = [(to_device(controls, a), to_device(controls, b)) for a, b in hp]
    _, need = batched.batched_plan(controls, pairs)
    small_slots = batched.CapturedBatch(controls, pairs, slot_capacity=need // 2, cols_capacity=need)
    small_slots.enqueue()
    with pytest.raises(ClBoolException, match="slot capacity"):
        small_slots.result()
    small_cols = batched.CapturedBatch(controls, pairs, slot_capacity=need, cols_capacity=need // 3)
    small_cols.enqueue()
    with pytest.raises(ClBoolException, match="column capacity"):
        small_cols.result()
    # the same buffers with enough room again: complete and exact
    ok = batched.CapturedBatch(controls, pairs)
    ok.enqueue()
    _check(ok.result(), hp, "after overflow")


def test_capture_rejects_bad_arguments():
    """Host-side checks run before any device work (no GPU needed)."""
    import clbool_b200 as cbm
    r = cbm.lib.clb_dcsr_spgemm_batched_capture(None, 1, None, None, None, 0, None, None, None, 0, None, None)
    assert r == 12  # CLBOOL_INVALID_ARGUMENT
