"""Every secondary workload checked against the oracle at the size it is
measured at:

  * 256 independent products, n log-uniform in [2^10, 2^18], power-law
    rows (exponent 2.1, mean 6, at most 4096), seeded per pair: the batched
    call and the host-sync-free form replayed from a CUDA graph, each with
    upper-bound and with learned slots, pair by pair against the oracle's
    product (coo_utils::matrix_multiplication_cpu, coo_utils.cpp:470-514,
    restated);
  * R-MAT scale 21 A*A (seed 21) by the learned single pass in row blocks:
    each block bit-identical to the exact two-pass form on the device, and
    768 seeded rows (640 by products, 128 uniform) against the oracle;
  * the closure C <- C v sum_i C L_i over three uniform label matrices of
    n = 2^18, average degree 3: iterations 1 and 2 (2.4e8 products) in full
    by both iteration methods, iteration 3 (2.1e9 products) on 768 seeded
    rows;
  * the DCSR Kronecker product of two R-MAT scale-11 graphs (6.6e8
    entries, dcsr::kronecker_product, src/dcsr/dcsr_kronecker_product.cpp:5-64)
    in full.
Inputs are the benchmark's own (same generators and seeds)."""
import numpy as np
import pytest

import oracle as O
from util import assert_dcsr_equal, assert_rows_match, from_device, same_on_device, sub_rows, to_device, weighted_pick

pytestmark = pytest.mark.gpu


# ------------------------------------------------------- 256-pair batch --
@pytest.fixture(scope="module")
def batch256():
    """The benchmark's batch: n_k = exp(U(log 2^10, log 2^18)) from seed 17,
    pair k's operands from seeds 1000 + 2k + 1 and 1000 + 2k + 2."""
    from clbool_b200 import gen
    rng = np.random.default_rng(17)
    ns = np.exp(rng.uniform(np.log(1 << 10), np.log(1 << 18), size=256)).astype(int)
    pairs = []
    for k, n in enumerate(ns):
        n = int(n)
        mats = []
        for s in (2 * k + 1, 2 * k + 2):
            r, c = gen.power_law_rows(n, n, 2.1, 6.0, 4096, seed=1000 + s)
            mats.append(O.coo_to_dcsr(O.Coo(n, n, r, c)))
        pairs.append(tuple(mats))
    want = [O.spgemm(a, b) for a, b in pairs]
    return pairs, want


def test_batch256_batched_call(controls, batch256):
    import clbool_b200 as cb
    pairs, want = batch256
    dev = [(to_device(controls, a), to_device(controls, b)) for a, b in pairs]
    st = {}
    outs = cb.dcsr.matrix_multiplication_batched(controls, dev, stats=st)
    assert st["nnz"] == sum(len(w.cols) for w in want)
    for k, (c, w) in enumerate(zip(outs, want)):
        assert_dcsr_equal(from_device(controls, c), w, f"pair {k}")


def test_batch256_graph_replay(controls, batch256):
    from clbool_b200 import batched
    pairs, want = batch256
    dev = [(to_device(controls, a), to_device(controls, b)) for a, b in pairs]
    cap = batched.CapturedBatch(controls, dev)
    graph = batched.Graph(controls, cap.enqueue)
    try:
        for _ in range(2):
            graph.launch()
            got = cap.result()
            for k, ((rpt, rows, cols), w) in enumerate(zip(got, want)):
                assert np.array_equal(cols, w.cols), f"pair {k}: cols"
                if len(w.cols):
                    assert np.array_equal(rows, w.rows) and np.array_equal(rpt, np.asarray(w.rpt, np.uint64)), k
    finally:
        graph.close()


def test_batch256_learned_forms(controls, batch256):
    """The learned-sized batch: the batched call and the graph-replayed
    capture form with learned slots."""
    import clbool_b200 as cb
    from clbool_b200 import batched, sizing
    pairs, want = batch256
    dev = [(to_device(controls, a), to_device(controls, b)) for a, b in pairs]
    sizer = sizing.RowSizer.load(controls)
    outs = cb.dcsr.matrix_multiplication_batched_learned(controls, dev, sizer)
    for k, (c, w) in enumerate(zip(outs, want)):
        assert_dcsr_equal(from_device(controls, c), w, f"learned batched, pair {k}")
    del outs
    cap = batched.CapturedBatch(controls, dev, sizer=sizer)
    graph = batched.Graph(controls, cap.enqueue)
    try:
        graph.launch()
        got = cap.result()
        assert not cap.fell_back
        for k, ((rpt, rows, cols), w) in enumerate(zip(got, want)):
            assert np.array_equal(cols, w.cols), f"learned capture, pair {k}: cols"
            if len(w.cols):
                assert np.array_equal(rows, w.rows) and np.array_equal(rpt, np.asarray(w.rpt, np.uint64)), k
    finally:
        graph.close()


# ----------------------------------------------- R-MAT scale 21, learned --
def _blocks(work, count):
    """Contiguous blocks of stored rows with about equal products."""
    cum = np.cumsum(work, dtype=np.float64)
    cuts = [0] + [int(np.searchsorted(cum, cum[-1] * q / count, side="left")) + 1 for q in range(1, count)]
    cuts.append(work.size)
    return [(lo, hi) for lo, hi in zip(cuts[:-1], cuts[1:]) if hi > lo]


def test_rmat21_learned_row_blocks(controls):
    import clbool_b200 as cb
    from clbool_b200 import gen, sizing
    r, c = gen.rmat(21, seed=21)
    n = 1 << 21
    a = O.coo_to_dcsr(O.Coo(n, n, r, c))
    del r, c
    work = O.workload(a, a).astype(np.int64)
    pick = weighted_pick(work, 640, seed=21, uniform=128)
    want = O.spgemm(sub_rows(a, pick), a)
    A_full = to_device(controls, a)
    sizer = sizing.RowSizer.load(controls)
    total = {"products": 0, "fallback_rows": 0}
    for lo, hi in _blocks(work, 8):
        blk = sub_rows(a, np.arange(lo, hi))
        A = to_device(controls, blk)
        st = {}
        Cl = sizing.matrix_multiplication_learned(controls, None, A, A_full, sizer, stats=st)
        Ct = cb.dcsr.matrix_multiplication_hash(controls, None, A, A_full)
        controls.sync()
        same_on_device(Cl, Ct, f"block [{lo}, {hi}): learned vs two-pass")
        del Ct
        sel = (pick >= lo) & (pick < hi)
        if sel.any():
            rows_sel = np.asarray(a.rows)[pick[sel]]
            k = np.flatnonzero(np.isin(want.rows, rows_sel))
            assert_rows_match(controls, Cl, sub_rows(want, k), f"block [{lo}, {hi})")
        total["products"] += st["products"]
        total["fallback_rows"] += st["fallback_rows"]
        del Cl, A
    assert total["products"] == int(work.sum())
    assert total["fallback_rows"] <= 16, total


# ------------------------------------------------- closure, n = 2^18 ----
@pytest.fixture(scope="module")
def labels18():
    from clbool_b200 import gen
    n = 1 << 18
    labels = []
    for seed in (1, 2, 3):
        r, c = gen.poisson_rows(n, n, 3.0, seed=seed)
        labels.append(O.coo_to_dcsr(O.Coo(n, n, r, c)))
    ident = O.Dcsr(n, n, np.arange(n + 1, dtype=np.uint64), np.arange(n, dtype=np.uint32),
                   np.arange(n, dtype=np.uint32))
    M = O.union([ident] + labels)  # C v sum_i C L_i = C (I v L_1 v L_2 v L_3)
    C = O.union(labels)
    iters = [C]
    for _ in range(2):
        iters.append(O.spgemm(iters[-1], M))
    return labels, M, iters


@pytest.mark.parametrize("method,learned", [("fused", False), ("batched", False), ("fused", True),
                                            ("batched", True)])
def test_closure_n2e18_two_iterations(controls, labels18, method, learned):
    from clbool_b200 import cfpq, sizing
    labels, _, iters = labels18
    L = [to_device(controls, m) for m in labels]
    sizer = sizing.RowSizer.load(controls) if learned else None
    C, hist = cfpq.closure(controls, L, max_iters=2, method=method, sizer=sizer)
    assert [h["nnz"] for h in hist] == [len(m.cols) for m in iters]
    assert_dcsr_equal(from_device(controls, C), iters[2], f"{method}: C_2")


def test_closure_n2e18_third_iteration_sampled(controls, labels18):
    from clbool_b200 import cfpq, sizing
    labels, M, iters = labels18
    C2 = iters[2]
    work = O.workload(C2, M).astype(np.int64)
    assert int(work.sum()) > 2_000_000_000
    pick = weighted_pick(work, 640, seed=3, uniform=128)
    want = O.spgemm(sub_rows(C2, pick), M)
    L = [to_device(controls, m) for m in labels]
    for sizer in (None, sizing.RowSizer.load(controls)):
        C3, hist = cfpq.closure(controls, L, start=to_device(controls, C2), max_iters=1, sizer=sizer)
        assert hist[-1]["products"] == int(work.sum())
        assert_rows_match(controls, C3, want, f"C_3 (learned: {sizer is not None})")
        del C3


# ------------------------------------------- Kronecker, R-MAT 11 x 11 ---
def test_kronecker_rmat11_full(controls):
    import clbool_b200 as cb
    from clbool_b200 import gen
    n = 1 << 11
    ms = []
    for seed in (1, 2):
        r, c = gen.rmat(11, seed=seed)
        ms.append(O.coo_to_dcsr(O.Coo(n, n, r, c)))
    want = O.kronecker(ms[0], ms[1])
    assert len(want.cols) > 600_000_000
    K = cb.dcsr.kronecker_product(controls, None, to_device(controls, ms[0]), to_device(controls, ms[1]))
    assert_dcsr_equal(from_device(controls, K), want, "A (x) B")
