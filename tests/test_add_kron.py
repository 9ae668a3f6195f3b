"""coo::matrix_addition, csr::matrix_addition, dcsr::kronecker_product and
dcsr::transpose on the GPU vs the oracle and the golden digests recorded from
the reference's CPU functions (test/test_operations.cpp:14-277)."""
import numpy as np
import pytest

import oracle as O
from util import assert_dcsr_equal, coo_digest, csr_digest, dcsr_digest, from_device, golden, pairs_dcsr, to_device

pytestmark = pytest.mark.gpu
G = golden()


def _coo_dev(ctl, rows, cols, n):
    import clbool_b200 as cb
    return cb.matrix_coo.from_host(ctl, rows, cols, n, n)


def _csr_dev(ctl, rows, cols, n):
    import clbool_b200 as cb
    return cb.csr_from_cpu(ctl, cb.csr_cpu_from_pairs(rows, cols, n, n))


def test_addition_coo_golden(controls):
    import clbool_b200 as cb
    for case in G["addition_coo"]:
        s, ka, kb = case["size"], case["k_a"], case["k_b"]
        ar, ac = O.generate_coo_pairs(s * ka, s)
        br, bc = O.generate_coo_pairs(s * kb, s)
        c = cb.matrix_coo()
        cb.coo.matrix_addition(controls, c, _coo_dev(controls, ar, ac, s), _coo_dev(controls, br, bc, s))
        h = cb.matrix_coo_from_gpu(controls, c)
        assert coo_digest(h.rows, h.cols) == case["sum"], case


def test_addition_coo_small_grid(controls):
    """addition_coo_small: sizes 0..2000 step 15 x k_a, k_b in 0..9 (subsampled)."""
    import clbool_b200 as cb
    for s in range(0, 2000, 15 * 9):
        for ka in range(0, 10, 3):
            for kb in range(0, 10, 4):
                a = O.Coo(s, s, *O.generate_coo_pairs(s * ka, s))
                b = O.Coo(s, s, *O.generate_coo_pairs(s * kb, s))
                c = cb.coo.matrix_addition(controls, None, _coo_dev(controls, a.rows, a.cols, s),
                                           _coo_dev(controls, b.rows, b.cols, s))
                want = O.coo_add(a, b)
                h = cb.matrix_coo_from_gpu(controls, c)
                assert np.array_equal(h.rows, want.rows) and np.array_equal(h.cols, want.cols), (s, ka, kb)


def test_addition_csr_golden(controls):
    import clbool_b200 as cb
    for case in G["addition_csr"]:
        s, ka, kb = case["size"], case["k_a"], case["k_b"]
        ar, ac = O.generate_coo_pairs(s * ka, s)
        br, bc = O.generate_coo_pairs(s * kb, s)
        c = cb.matrix_csr()
        cb.csr.matrix_addition(controls, c, _csr_dev(controls, ar, ac, s), _csr_dev(controls, br, bc, s))
        h = cb.matrix_csr_from_gpu(controls, c)
        if case["sum"]["nnz"] == 0:
            assert c.nnz() == 0
            continue
        assert csr_digest(O.Csr(s, s, h.rpt, h.cols)) == case["sum"], case


def test_addition_csr_skewed(controls):
    """Long rows beside short ones (tiles inside one row and tiles spanning
    thousands of rows), empty rows, and a row that only one side has."""
    import clbool_b200 as cb
    from clbool_b200 import gen
    r, c = gen.rmat(14, seed=5)
    n = 1 << 14
    a = O.Coo(n, n, r, c)
    aa = O.spgemm(O.coo_to_dcsr(a), O.coo_to_dcsr(a))
    csr_c = O.dcsr_to_csr(aa)
    csr_a = O.coo_to_csr(a)
    A = cb.csr_from_cpu(controls, cb.matrix_csr_cpu(csr_c.rpt, csr_c.cols, n, n))
    B = cb.csr_from_cpu(controls, cb.matrix_csr_cpu(csr_a.rpt, csr_a.cols, n, n))
    out = cb.csr.matrix_addition(controls, None, A, B)
    h = cb.matrix_csr_from_gpu(controls, out)
    want = O.csr_add(csr_c, csr_a)
    assert np.array_equal(h.rpt, want.rpt) and np.array_equal(h.cols, want.cols)


def test_addition_csr_insertion(controls):
    """One operand far sparser than the other (the insertion path): entries
    before, between (several at one gap) and after the long row's entries,
    duplicates, rows only one side has, a row where the sparse side is the
    longer one, rows of 60000 entries (split over a CTA), both operand
    orders."""
    import clbool_b200 as cb
    rng = np.random.default_rng(8)
    n, ncols = 3000, 100000
    big_r, big_c, small_r, small_c = [], [], [], []
    for r in range(n):
        if r % 7 == 3:
            continue  # empty on the long side
        wide = r >= n - 6  # rows longer than one warp's share: copied in pieces by a CTA
        cols = np.sort(rng.choice(np.arange(10, ncols - 10), 60000 if wide else 300, replace=False))
        big_r.append(np.full(cols.size, r)); big_c.append(cols)
        if r % 5 == 0 or wide:
            k = int(rng.integers(1, 6))
            picks = [0, ncols - 1, int(cols[0]) + 1 if cols[1] > cols[0] + 2 else 1]
            picks += list(rng.choice(cols, k))                       # duplicates
            picks += [int(cols[40]) + 1, int(cols[40]) + 2] if cols[41] > cols[40] + 3 else []
            sc = np.unique(np.array(picks))
            small_r.append(np.full(sc.size, r)); small_c.append(sc)
    for r in (3, 10, 17):  # rows the long side does not have
        sc = np.sort(rng.choice(ncols, 4, replace=False))
        small_r.append(np.full(sc.size, r)); small_c.append(sc)
    sc = np.arange(0, 700, 1)  # the sparse side is longer in this row (r = 24 has 300 on the other)
    small_r.append(np.full(sc.size, 24)); small_c.append(sc)
    br, bc = np.concatenate(big_r).astype(np.uint32), np.concatenate(big_c).astype(np.uint32)
    sr, sc_ = np.concatenate(small_r).astype(np.uint32), np.concatenate(small_c).astype(np.uint32)
    o = np.lexsort((sc_, sr)); sr, sc_ = sr[o], sc_[o]
    keep = np.concatenate([[True], (sr[1:] != sr[:-1]) | (sc_[1:] != sc_[:-1])]); sr, sc_ = sr[keep], sc_[keep]
    big = O.coo_to_csr(O.Coo(n, ncols, br, bc))
    small = O.coo_to_csr(O.Coo(n, ncols, sr, sc_))
    assert len(small.cols) * 16 < len(big.cols)
    for x, y in ((big, small), (small, big)):
        X = cb.csr_from_cpu(controls, cb.matrix_csr_cpu(x.rpt, x.cols, n, ncols))
        Y = cb.csr_from_cpu(controls, cb.matrix_csr_cpu(y.rpt, y.cols, n, ncols))
        h = cb.matrix_csr_from_gpu(controls, cb.csr.matrix_addition(controls, None, X, Y))
        want = O.csr_add(x, y)
        assert np.array_equal(h.rpt, want.rpt) and np.array_equal(h.cols, want.cols)


def test_addition_empty_and_shape(controls):
    import clbool_b200 as cb
    a = _coo_dev(controls, *O.generate_coo_pairs(500, 100), 100)
    e = cb.matrix_coo.zeros(100, 100)
    c = cb.coo.matrix_addition(controls, None, a, e)
    assert c.nnz() == a.nnz() and c.rows_gpu() is not a.rows_gpu()  # a copy
    assert cb.coo.matrix_addition(controls, None, e, e).nnz() == 0
    with pytest.raises(cb.ClBoolException) as ex:
        cb.coo.matrix_addition(controls, None, a, cb.matrix_coo.zeros(100, 101))
    assert ex.value.status_name == "CLBOOL_INVALID_ARGUMENT"


def test_kronecker_golden(controls):
    import clbool_b200 as cb
    for case in G["kronecker_dcsr"]:
        r, c = O.generate_coo_pairs(case["nnz"], case["size"])
        a = O.coo_to_dcsr(O.Coo(case["size"], case["size"], r, c))
        k = cb.dcsr.kronecker_product(controls, None, to_device(controls, a), to_device(controls, a))
        got = O.dcsr_to_coo(from_device(controls, k))
        assert coo_digest(got.rows, got.cols) == case["kron"]


@pytest.mark.parametrize("na,nb", [(300, 40), (1000, 3000), (1, 5000)])
def test_kronecker_vs_oracle(controls, na, nb):
    import clbool_b200 as cb
    a = O.coo_to_dcsr(O.Coo(60, 70, *O.generate_coo_pairs(na, 60)))
    b = O.coo_to_dcsr(O.Coo(500, 400, *O.generate_coo_pairs(nb, 400)))
    a = a._replace(ncols=70)
    b = b._replace(nrows=500)
    k = cb.dcsr.kronecker_product(controls, None, to_device(controls, a), to_device(controls, b))
    assert dcsr_digest(from_device(controls, k)) == dcsr_digest(O.kronecker(a, b))


def test_kronecker_row_length_sweep(controls):
    """Every B row length from 1 to 260 against A rows of 1-5, 7, 31-33 and
    127-129 entries: C's rows start at every 16-byte alignment, and the
    column kernel's head, whole-group and tail entries, its step carry and
    its short-row division all occur."""
    import clbool_b200 as cb
    rng = np.random.default_rng(29)
    la = np.array([1, 2, 3, 4, 5, 7, 31, 32, 33, 127, 128, 129])
    ra = np.repeat(np.arange(la.size, dtype=np.uint32), la)
    ca = np.concatenate([np.sort(rng.choice(200, k, replace=False)) for k in la]).astype(np.uint32)
    a = O.coo_to_dcsr(O.Coo(la.size, 200, ra, ca))
    lb = np.arange(1, 261)
    rb = np.repeat(np.arange(lb.size, dtype=np.uint32), lb)
    cbb = np.concatenate([np.sort(rng.choice(300, k, replace=False)) for k in lb]).astype(np.uint32)
    b = O.coo_to_dcsr(O.Coo(lb.size, 300, rb, cbb))
    want = O.kronecker(a, b)
    assert len(want.cols) == int(la.sum()) * int(lb.sum())
    k = cb.dcsr.kronecker_product(controls, None, to_device(controls, a), to_device(controls, b))
    assert_dcsr_equal(from_device(controls, k), want, "row length sweep")


@pytest.mark.parametrize("size,k", [(0, 0), (5, 3), (95, 19), (900, 25), (9400, 60)])
def test_transpose(controls, size, k):
    """transpose_* suites (test_operations.cpp:14-37)."""
    import clbool_b200 as cb
    a = pairs_dcsr(size, k)
    t = cb.dcsr.transpose(controls, None, to_device(controls, a))
    assert dcsr_digest(from_device(controls, t)) == dcsr_digest(O.transpose(a))


# ------------------------------------------------------------ closure (CFPQ) --
def _labels(n, deg, count, seed):
    from clbool_b200 import gen
    out = []
    for k in range(count):
        r, c = gen.poisson_rows(n, n, float(deg), seed=seed + k)
        out.append(O.coo_to_dcsr(O.Coo(n, n, r, c)))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("method,learned", [("fused", False), ("batched", False), ("fused", True),
                                            ("batched", True)])
def test_closure_fixpoint_matches_oracle(controls, method, learned):
    """Three uniform label matrices (n = 2^9, average degree 0.6 so the
    closure stays sparse): every iteration's nnz and the fixpoint equal the
    oracle's, by both iteration methods, with and without learned sizing."""
    from clbool_b200 import cfpq, sizing
    labels = _labels(1 << 9, 0.6, 3, seed=11)
    want, want_hist = O.closure(labels)
    sizer = sizing.RowSizer.load(controls) if learned else None
    C, hist = cfpq.closure(controls, [to_device(controls, L) for L in labels], method=method, sizer=sizer)
    assert [h["nnz"] for h in hist] == want_hist
    assert hist[-1]["stop"] == "fixpoint"
    assert_dcsr_equal(from_device(controls, C), want, "closure")


@pytest.mark.gpu
def test_closure_bounds(controls):
    """Degree 3 per label: the closure grows fast; the iteration cap and the
    products guard stop it, and the iterations done match the oracle's."""
    from clbool_b200 import cfpq
    labels = _labels(1 << 10, 3, 3, seed=21)
    C, hist = cfpq.closure(controls, [to_device(controls, L) for L in labels], max_iters=2, method="batched")
    assert hist[-1]["stop"] == "max_iters" and len(hist) == 3
    want, want_hist = O.closure(labels, max_iters=2)
    assert [h["nnz"] for h in hist] == want_hist
    assert_dcsr_equal(from_device(controls, C), want, "closure, 2 iterations")
    C2, hist2 = cfpq.closure(controls, [to_device(controls, L) for L in labels], max_products=1)
    assert hist2[-1]["stop"] == "max_products" and len(hist2) == 1


def _csr_of(m: O.Dcsr) -> O.Csr:
    return O.dcsr_to_csr(m)


def test_addition_csr_batched(controls):
    """Many independent additions in one call (no counterpart in the
    reference, which adds one pair per call): pairs of different shapes,
    power-law and R-MAT operands, a much sparser side (the stack takes the
    insertion path when most of it is), empty operands on either side, a pair
    of two empty operands; each sum equal to the oracle's."""
    import clbool_b200 as cb
    from clbool_b200 import gen
    pairs = []
    for k, n in enumerate((700, 3000, 12000)):
        ra, ca = gen.power_law_rows(n, n + 5, 2.1, 6.0, 512, seed=300 + 2 * k)
        rb, cb_ = gen.power_law_rows(n, n + 5, 2.1, 6.0, 512, seed=301 + 2 * k)
        pairs.append((O.coo_to_csr(O.Coo(n, n + 5, ra, ca)), O.coo_to_csr(O.Coo(n, n + 5, rb, cb_))))
    r, c = gen.rmat(12, seed=9)
    g = O.coo_to_dcsr(O.Coo(1 << 12, 1 << 12, r, c))
    pairs.append((_csr_of(O.spgemm(g, g)), _csr_of(g)))
    e = O.Csr(40, 50, np.zeros(41, np.uint64), np.zeros(0, np.uint32))
    ra, ca = O.generate_coo_pairs(40 * 3, 40)
    f = O.coo_to_csr(O.Coo(40, 50, ra, ca))
    pairs += [(e, f), (f, e), (e, e)]

    def dev(m):
        return cb.csr_from_cpu(controls, cb.matrix_csr_cpu(m.rpt, m.cols, m.nrows, m.ncols))

    for order in (pairs, pairs[::-1]):
        got = cb.csr.matrix_addition_batched(controls, [(dev(a), dev(b)) for a, b in order])
        for k, ((a, b), s_) in enumerate(zip(order, got)):
            want = O.csr_add(a, b)
            assert s_.nrows() == a.nrows and s_.ncols() == a.ncols and s_.nnz() == len(want.cols), k
            if len(want.cols):
                h = cb.matrix_csr_from_gpu(controls, s_)
                assert np.array_equal(h.rpt, want.rpt) and np.array_equal(h.cols, want.cols), k
    assert cb.csr.matrix_addition_batched(controls, []) == []
    with pytest.raises(cb.ClBoolException) as ex:
        cb.csr.matrix_addition_batched(controls, [(dev(pairs[0][0]), dev(pairs[0][1])), (dev(f), dev(pairs[0][0]))])
    assert ex.value.status_name == "CLBOOL_INVALID_ARGUMENT"


def test_union_matches_oracle(controls):
    """The one-pass union of k matrices of one shape (no counterpart in the
    reference): power-law and R-MAT pieces, an empty operand, a single
    operand, rows that only one operand stores, duplicates across all of
    them; equal to the oracle's union, under both accumulator forms."""
    import clbool_b200 as cb
    from clbool_b200 import gen
    n = 3000
    mats = []
    for k in range(5):
        r, c = gen.power_law_rows(n, n + 11, 2.1, 12.0, 2048, seed=600 + k)
        mats.append(O.coo_to_dcsr(O.Coo(n, n + 11, r, c)))
    r, c = gen.rmat(11, seed=3)
    g = O.coo_to_dcsr(O.Coo(n, n + 11, r, c))
    mats += [g, g, O.coo_to_dcsr(O.Coo(n, n + 11, np.zeros(0, np.uint32), np.zeros(0, np.uint32)))]
    dev = [to_device(controls, m) for m in mats]
    for sel in (list(range(len(mats))), [0], [5, 6], [7, 2], [7]):
        want = O.union([mats[i] for i in sel])
        for t in (None, cb.dcsr.tuning("two_pass")):
            got = cb.dcsr.matrix_union(controls, [dev[i] for i in sel], t)
            assert_dcsr_equal(from_device(controls, got), want, f"union {sel}")
    with pytest.raises(cb.ClBoolException) as ex:
        cb.dcsr.matrix_union(controls, [dev[0], to_device(controls, pairs_dcsr(100, 3))])
    assert ex.value.status_name == "CLBOOL_INVALID_ARGUMENT"


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["fused", "batched"])
def test_closure_with_the_kept_two_pass_tuning(controls, method):
    """The tuning the autotuner now often returns (the two-pass form keeping
    its bitmaps, bitmap rows from 256 products), through both iteration
    methods (the batched one also hands it to the one-pass union)."""
    import clbool_b200 as cb
    from clbool_b200 import cfpq
    labels = _labels(1 << 10, 3, 3, seed=23)
    want, want_hist = O.closure(labels, max_iters=2)
    t = cb.dcsr.tuning("two_pass_kept", bitmap_min=256, bitmap_threads=256)
    C, hist = cfpq.closure(controls, [to_device(controls, L) for L in labels], max_iters=2, method=method, tune=t)
    assert [h["nnz"] for h in hist] == want_hist
    assert_dcsr_equal(from_device(controls, C), want, f"closure {method}, kept two-pass tuning")
