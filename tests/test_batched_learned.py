"""The learned-sized batched product and its host-sync-free, graph-replayable
form, bit-exact against the oracle.

No counterpart in the reference, which multiplies one pair per call
(src/dcsr/dcsr.hpp:27-36); every pair's product must equal the oracle's
restatement of coo_utils::matrix_multiplication_cpu (coo_utils.cpp:470-514)
whatever the predictor says: with the packaged predictor, with a predictor
pushed to one-entry slots (every bitmap row spills or is recomputed by the
exact two-pass form), and in the capture form with an arena too small for
the spills (the batch is then recomputed by the exact batched form)."""
import ctypes

import numpy as np
import pytest

import oracle as O
from util import assert_dcsr_equal, from_device, pairs_dcsr, to_device

pytestmark = pytest.mark.gpu


def _host_pairs():
    """Mixed pairs: power-law rows, an R-MAT graph by itself (bitmap rows),
    a heavy right operand, a rectangular pair and an empty left operand."""
    from clbool_b200 import gen
    rng = np.random.default_rng(3)
    pairs = []
    for k, n in enumerate((1500, 4000, 9000)):
        ra, ca = gen.power_law_rows(n, n, 2.1, 6.0, 4096, seed=50 + 2 * k)
        rb, cb_ = gen.power_law_rows(n, n, 2.1, 6.0, 4096, seed=51 + 2 * k)
        pairs.append((O.coo_to_dcsr(O.Coo(n, n, ra, ca)), O.coo_to_dcsr(O.Coo(n, n, rb, cb_))))
    r, c = gen.rmat(12, seed=5)
    rm = O.coo_to_dcsr(O.Coo(1 << 12, 1 << 12, r, c))
    pairs.append((rm, rm))
    hr = np.repeat(np.arange(2000, dtype=np.uint32), 300)
    hc = rng.integers(0, 60000, hr.size).astype(np.uint32)
    heavy = O.coo_to_dcsr(O.Coo(2000, 60000, *O.unique_pairs(*O.sort_pairs(hr, hc))))
    pairs.append((pairs_dcsr(2000, 20), heavy))
    empty = O.Dcsr(30, 40, np.zeros(1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    pairs.append((empty, pairs_dcsr(40, 3)))
    return pairs


@pytest.fixture(scope="module")
def host_pairs():
    pairs = _host_pairs()
    return pairs, [O.spgemm(a, b) for a, b in pairs]


@pytest.mark.parametrize("margin_log2,slack", [(0.25, 8.0), (-30.0, 0.0)])
def test_learned_batched_matches_oracle(controls, host_pairs, margin_log2, slack):
    import clbool_b200 as cb
    from clbool_b200 import sizing
    pairs, want = host_pairs
    dev = [(to_device(controls, a), to_device(controls, b)) for a, b in pairs]
    sizer = sizing.RowSizer.load(controls)
    st = {}
    outs = cb.dcsr.matrix_multiplication_batched_learned(controls, dev, sizer, margin_log2, slack, stats=st)
    for k, (c, w) in enumerate(zip(outs, want)):
        assert_dcsr_equal(from_device(controls, c), w, f"pair {k} (margin {margin_log2})")
    assert st["nnz"] == sum(len(w.cols) for w in want)
    if margin_log2 < 0:  # one-entry slots: the bitmap rows spilled or were recomputed
        assert st["spilled_rows"] + st["fallback_rows"] > 0, st


def test_learned_batched_features_are_per_pair(controls):
    """The row features of a stacked batch equal those of each pair alone:
    the learned batch gives every pair the capacities it gets alone, so its
    slot total is the sum of the pairs' own learned slot totals."""
    from clbool_b200 import batched, sizing
    pairs = _host_pairs()[:4]
    sizer = sizing.RowSizer.load(controls)
    dev = [(to_device(controls, a), to_device(controls, b)) for a, b in pairs]
    _, together = batched.batched_plan(controls, dev, sizer)
    alone = sum(batched.batched_plan(controls, [p], sizer)[1] for p in dev)
    assert together == alone


def _check(got, want, what):
    for k, ((rpt, rows, cols), w) in enumerate(zip(got, want)):
        assert np.array_equal(cols, w.cols), f"{what} pair {k}: cols"
        if len(w.cols):
            assert np.array_equal(rows, w.rows), f"{what} pair {k}: rows"
            assert np.array_equal(rpt, np.asarray(w.rpt, np.uint64)), f"{what} pair {k}: rpt"


def test_learned_capture_graph_replay(controls, host_pairs):
    from clbool_b200 import batched, sizing
    pairs, want = host_pairs
    dev = [(to_device(controls, a), to_device(controls, b)) for a, b in pairs]
    sizer = sizing.RowSizer.load(controls)
    _, upper = batched.batched_plan(controls, dev)
    # an arena as large as the upper-bound slots: every row that outgrows its
    # learned slot spills there, none is left for the exact recomputation
    cap = batched.CapturedBatch(controls, dev, sizer=sizer, arena_capacity=upper)
    assert cap.slot_capacity <= upper
    cap.enqueue()
    _check(cap.result(), want, "direct")
    assert not cap.fell_back
    graph = batched.Graph(controls, cap.enqueue)
    try:
        for _ in range(2):
            graph.launch()
            _check(cap.result(), want, "graph replay")
    finally:
        graph.close()


def test_learned_capture_falls_back_when_the_arena_is_full(controls, host_pairs):
    from clbool_b200 import batched, sizing
    pairs, want = host_pairs
    dev = [(to_device(controls, a), to_device(controls, b)) for a, b in pairs]
    sizer = sizing.RowSizer.load(controls)
    cap = batched.CapturedBatch(controls, dev, sizer=sizer, margin_log2=-30.0, slack=0.0, arena_capacity=64,
                                cols_capacity=sum(len(w.cols) for w in want))
    cap.enqueue()
    assert cap.flags_now() & 8
    _check(cap.result(), want, "exact recomputation")
    assert cap.fell_back


def test_learned_batched_rejects_null_sizer():
    """Host-side checks run before any device work."""
    import clbool_b200 as cbm
    assert cbm.lib.clb_dcsr_spgemm_batched_learned(None, 0, None, None, None, None, 0.0, 0.0, None, None) == 12
    assert cbm.lib.clb_dcsr_spgemm_batched_capture_learned(None, 1, None, None, None, 0.0, 0.0, None, 0, 0, None,
                                                           None, None, 0, None, None) == 12
