"""Tuned and batched SpGEMM on the GPU vs the oracle, bit-exact.

No counterpart in the reference, which multiplies one pair per call; every
pair's product must equal the oracle's restatement of
coo_utils::matrix_multiplication_cpu (coo_utils.cpp:470-514), under every
accumulator tuning."""
import numpy as np
import pytest

import oracle as O
from util import assert_dcsr_equal, from_device, pairs_dcsr, to_device

pytestmark = pytest.mark.gpu


def power_law_pair(seed: int, n: int):
    """One synthetic pair: n x n, power-law row lengths (exponent 2.1, mean 6,
    at most 4096), columns uniform without replacement."""
    from clbool_b200 import gen
    ra, ca = gen.power_law_rows(n, n, 2.1, 6.0, 4096, seed=2 * seed + 1)
    rb, cb_ = gen.power_law_rows(n, n, 2.1, 6.0, 4096, seed=2 * seed + 2)
    return O.coo_to_dcsr(O.Coo(n, n, ra, ca)), O.coo_to_dcsr(O.Coo(n, n, rb, cb_))


def batch(count: int, lo: int = 1 << 10, hi: int = 1 << 14, seed: int = 0):
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(lo), np.log(hi), size=count)).astype(int)
    return [power_law_pair(seed * 1000 + k, int(n)) for k, n in enumerate(ns)]


def run_batched(ctl, pairs, tune=None, stats=None):
    import clbool_b200 as cb
    dev = [(to_device(ctl, a), to_device(ctl, b)) for a, b in pairs]
    outs = cb.dcsr.matrix_multiplication_batched(ctl, dev, tune=tune, stats=stats)
    return [from_device(ctl, c) for c in outs]


def test_batch_of_power_law_pairs(controls):
    pairs = batch(24)
    st = {}
    got = run_batched(controls, pairs, stats=st)
    total = 0
    for k, ((a, b), c) in enumerate(zip(pairs, got)):
        want = O.spgemm(a, b)
        assert_dcsr_equal(c, want, f"pair {k}")
        total += len(want.cols)
    assert st["nnz"] == total
    assert st["products"] == sum(int(O.workload(a, b).sum()) for a, b in pairs)


@pytest.mark.parametrize("form,warp_max,bitmap_min,bitmap_threads,small_lanes", [
    ("two_pass", 256, 4096, 1024, 8), ("single_pass", 256, 4096, 1024, 8), ("two_pass", 64, 256, 256, 32),
    ("single_pass", 32, 256, 512, 16), ("two_pass", 128, 1024, 256, 16), ("single_pass", 64, 1024, 1024, 32),
    ("two_pass_kept", 256, 256, 1024, 8), ("two_pass_kept", 64, 1024, 256, 32)])
def test_every_tuning_gives_the_same_product(controls, form, warp_max, bitmap_min, bitmap_threads, small_lanes):
    import clbool_b200 as cb
    pairs = batch(6, seed=3) + [(pairs_dcsr(1500, 40), pairs_dcsr(1500, 40))]
    t = cb.dcsr.tuning(form, warp_max, bitmap_min, bitmap_threads, small_lanes)
    got = run_batched(controls, pairs, tune=t)
    for k, ((a, b), c) in enumerate(zip(pairs, got)):
        assert_dcsr_equal(c, O.spgemm(a, b), f"pair {k} {t.as_dict()}")


def test_tuned_single_product_wide_columns(controls):
    """Tunings on one product whose columns span more than one bitmap chunk."""
    import clbool_b200 as cb
    n = (1 << 21) + 77
    rng = np.random.default_rng(9)
    ra = np.repeat(np.arange(300, dtype=np.uint32), 12)
    ca = rng.integers(0, 2000, ra.size).astype(np.uint32)
    a = O.coo_to_dcsr(O.Coo(300, 2000, *O.unique_pairs(*O.sort_pairs(ra, ca))))
    rb = np.repeat(np.arange(2000, dtype=np.uint32), 400)
    cbb = rng.integers(0, n, rb.size).astype(np.uint32)
    b = O.coo_to_dcsr(O.Coo(2000, n, *O.unique_pairs(*O.sort_pairs(rb, cbb))))
    want = O.spgemm(a, b)
    for t in (cb.dcsr.tuning("two_pass", 256, 256, 256), cb.dcsr.tuning("single_pass", 64, 1024, 512)):
        c = cb.dcsr.matrix_multiplication_tuned(controls, None, to_device(controls, a), to_device(controls, b), t)
        assert_dcsr_equal(from_device(controls, c), want, str(t.as_dict()))


def test_batch_edge_cases(controls):
    z = O.coo_to_dcsr(O.Coo(50, 60, np.zeros(0, np.uint32), np.zeros(0, np.uint32)))
    z2 = O.coo_to_dcsr(O.Coo(60, 70, np.zeros(0, np.uint32), np.zeros(0, np.uint32)))
    rng = np.random.default_rng(4)
    a = O.coo_to_dcsr(O.Coo(800, 300, *O.unique_pairs(*O.sort_pairs(
        rng.integers(0, 800, 6000).astype(np.uint32), rng.integers(0, 300, 6000).astype(np.uint32)))))
    b = O.coo_to_dcsr(O.Coo(300, 5000, *O.unique_pairs(*O.sort_pairs(
        np.random.default_rng(1).integers(0, 300, 3000).astype(np.uint32),
        np.random.default_rng(2).integers(0, 5000, 3000).astype(np.uint32)))))
    a2 = pairs_dcsr(60, 5)
    pairs = [(z, z2), (a, b), (a2, pairs_dcsr(60, 8)), (z, z2), (pairs_dcsr(50, 3, ncols=60), z2), (a, b)]
    got = run_batched(controls, pairs)
    for k, ((x, y), c) in enumerate(zip(pairs, got)):
        want = O.spgemm(x, y)
        assert c.nrows == x.nrows and c.ncols == y.ncols
        assert_dcsr_equal(c, want, f"pair {k}")
    assert run_batched(controls, []) == []


def test_batch_rejects_mismatched_pair(controls):
    import clbool_b200 as cb
    a, b = pairs_dcsr(100, 3), pairs_dcsr(120, 3)
    with pytest.raises(cb.ClBoolException) as e:
        run_batched(controls, [(a, a), (a, b)])
    assert e.value.status_name == "CLBOOL_INVALID_ARGUMENT"
    with pytest.raises(cb.ClBoolException) as e:
        cb.dcsr.matrix_multiplication_batched(controls, [(to_device(controls, a), to_device(controls, a))],
                                              tune=cb.dcsr.tuning("two_pass", 100))
    assert e.value.status_name == "CLBOOL_INVALID_VALUE"


def test_autotune_picks_a_tuning(controls):
    import clbool_b200 as cb
    pairs = batch(8, seed=5)
    dev = [(to_device(controls, a), to_device(controls, b)) for a, b in pairs]
    best, tried = cb.dcsr.autotune(controls, dev)
    assert len(tried) == 48  # forms 0, 1 and 2 (pairs within one bitmap chunk)
    assert {t["form"] for t, _ in tried} == {"two_pass", "single_pass", "two_pass_kept"}
    assert all(ms > 0 for _, ms in tried)
    fastest = min(tried, key=lambda t: t[1])
    assert fastest[0] == best.as_dict()
    got = [from_device(controls, c) for c in cb.dcsr.matrix_multiplication_batched(controls, dev, tune=best)]
    for k, ((a, b), c) in enumerate(zip(pairs, got)):
        assert_dcsr_equal(c, O.spgemm(a, b), f"pair {k}")
