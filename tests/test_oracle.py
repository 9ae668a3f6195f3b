"""The oracle, pinned: against the golden vectors recorded from the
reference's own CPU functions, and (when oracle/_ref is built) against those
functions directly on the reference's own test grids."""
import numpy as np
import pytest

import oracle as O
from util import coo_digest, csr_digest, dcsr_digest, golden, pairs_dcsr, sha

G = golden()
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference CPU library not built")


def test_readme_example():
    g = G["readme"]
    a = O.coo_to_dcsr(O.Coo(5, 5, np.array(g["a"]["rows"], np.uint32), np.array(g["a"]["cols"], np.uint32)))
    b = O.coo_to_dcsr(O.Coo(5, 5, np.array(g["b"]["rows"], np.uint32), np.array(g["b"]["cols"], np.uint32)))
    c = O.spgemm(a, b)
    assert c.rpt.tolist() == g["mxm"]["rpt"] == [0, 2, 5, 6]
    assert c.rows.tolist() == g["mxm"]["rows"]
    assert c.cols.tolist() == g["mxm"]["cols"]
    s = O.coo_add(O.dcsr_to_coo(a), O.dcsr_to_coo(b))
    assert s.rows.tolist() == g["add"]["rows"] and s.cols.tolist() == g["add"]["cols"]
    k = O.dcsr_to_coo(O.kronecker(a, b))
    assert k.rows.tolist() == g["kron"]["rows"] and k.cols.tolist() == g["kron"]["cols"]


def test_coo_constructor_kat():
    g = G["coo_constructor"]
    r, c = O.unique_pairs(g["rows"], g["cols"])
    assert len(r) == g["nnz_after"] == 9
    assert r.tolist() == g["out_rows"] and c.tolist() == g["out_cols"]


def test_csr_from_pairs_kat():
    g = G["csr_from_pairs"]
    c = O.coo_to_csr(O.Coo(g["m"], g["n"], np.array(g["rows"], np.uint32), np.array(g["cols"], np.uint32)))
    assert c.rpt.tolist() == g["rpt"] == [0, 3, 3, 6, 9, 9]
    assert c.cols.tolist() == g["out_cols"]


@pytest.mark.parametrize("case", G["multiplication_hash"], ids=lambda c: f"s{c['size']}k{c['k']}")
def test_multiplication_hash_grid(case):
    a = pairs_dcsr(case["size"], case["k"])
    assert dcsr_digest(a) == case["a"]
    assert dcsr_digest(O.spgemm(a, a)) == case["c"]


def test_multiplication_merge_grid():
    for case in G["multiplication_merge"]:
        a = pairs_dcsr(case["size"], case["k"])
        assert dcsr_digest(a) == case["a"], case
        assert dcsr_digest(O.spgemm(a, a)) == case["c"], case


def test_addition_grids():
    for case in G["addition_coo"]:
        s, ka, kb = case["size"], case["k_a"], case["k_b"]
        a = O.Coo(s, s, *O.generate_coo_pairs(s * ka, s))
        b = O.Coo(s, s, *O.generate_coo_pairs(s * kb, s))
        r = O.coo_add(a, b)
        assert coo_digest(r.rows, r.cols) == case["sum"], case
    for case in G["addition_csr"]:
        s, ka, kb = case["size"], case["k_a"], case["k_b"]
        a = O.coo_to_csr(O.Coo(s, s, *O.generate_coo_pairs(s * ka, s)))
        b = O.coo_to_csr(O.Coo(s, s, *O.generate_coo_pairs(s * kb, s)))
        assert csr_digest(O.csr_add(a, b)) == case["sum"], case


def test_kronecker_grid():
    for case in G["kronecker_dcsr"]:
        r, c = O.generate_coo_pairs(case["nnz"], case["size"])
        a = O.coo_to_dcsr(O.Coo(case["size"], case["size"], r, c))
        k = O.dcsr_to_coo(O.kronecker(a, a))
        assert coo_digest(k.rows, k.cols) == case["kron"]


def test_prefix_sum_and_sort_vectors():
    for case in G["prefix_sum"]:
        v = O.fill_random_buffer(case["n"], 3)
        assert sha(v, np.uint32) == case["input"]
        x, total = O.prefix_sum_u32(v)
        assert sha(x, np.uint32) == case["scan"] and total == case["total"]
    for case in G["bitonic_sort"]:
        r, c = O.fill_random_matrix(case["n"])
        assert sha(r, np.uint32) == case["input_rows"] and sha(c, np.uint32) == case["input_cols"]
        rs, cs = O.sort_pairs(r, c)
        assert sha(rs, np.uint32) == case["rows"] and sha(cs, np.uint32) == case["cols"]


@needs_ref
def test_esc_large_fixtures():
    R = O.Ref()
    for case in G["esc_large_fixtures"]:
        a, b = R.random_matrices(case["which"], case["max_size"], case["seed"])
        assert dcsr_digest(a) == case["a"] and dcsr_digest(b) == case["b"]
        assert dcsr_digest(O.spgemm(a, b)) == case["c"]


@needs_ref
@pytest.mark.parametrize("size,k", [(0, 0), (5, 3), (200, 7), (600, 19), (2000, 13)])
def test_against_reference_functions(size, k):
    R = O.Ref()
    r, c = O.generate_coo_pairs(size * k, size)
    rr, rc = R.generate_coo_pairs(size * k, size)
    assert np.array_equal(r, rr) and np.array_equal(c, rc)
    a = O.coo_to_dcsr(O.Coo(size, size, r, c))
    assert dcsr_digest(O.spgemm(a, a)) == dcsr_digest(R.spgemm(a, a))
    w = O.workload(a, a)
    assert np.array_equal(w.astype(np.uint32), R.workload(a, a))
    b = O.Coo(size, size, *O.generate_coo_pairs(size * (k + 2), size))
    s1, s2 = O.coo_add(O.Coo(size, size, r, c), b), R.coo_add(O.Coo(size, size, r, c), b)
    assert np.array_equal(s1.rows, s2.rows) and np.array_equal(s1.cols, s2.cols)
    assert np.array_equal(O.fill_random_buffer(size * k + 1, 3), R.fill_random_buffer(size * k + 1, 3))


def test_conversions_roundtrip():
    a = pairs_dcsr(3000, 9)
    coo = O.dcsr_to_coo(a)
    assert dcsr_digest(O.coo_to_dcsr(coo)) == dcsr_digest(a)
    csr = O.dcsr_to_csr(a)
    assert dcsr_digest(O.csr_to_dcsr(csr)) == dcsr_digest(a)
    t = O.transpose(O.transpose(a))
    assert dcsr_digest(t) == dcsr_digest(a)


def test_rowwise_nnz_matches_product():
    a = pairs_dcsr(1500, 20)
    c = O.spgemm(a, a)
    nnz = O.spgemm_row_nnz(a, a)
    assert int(nnz.sum()) == len(c.cols)
    assert np.array_equal(nnz[nnz > 0], np.diff(c.rpt))


def test_submatrix_reduce_golden():
    """README example (test_operations.cpp:309-310) and seeded ranges of the
    reference's submatrix / reduce tests, recorded from the reference."""
    g = G["readme"]
    a = O.coo_to_dcsr(O.Coo(5, 5, np.array(g["a"]["rows"], np.uint32), np.array(g["a"]["cols"], np.uint32)))
    r = O.reduce(a)
    assert r.rpt.tolist() == g["reduce"]["rpt"] and r.rows.tolist() == g["reduce"]["rows"]
    assert r.cols.tolist() == g["reduce"]["cols"]
    s = O.submatrix(a, 0, 2, 3, 2)
    assert s.rpt.tolist() == g["submatrix_0_2_3_2"]["rpt"] and s.rows.tolist() == g["submatrix_0_2_3_2"]["rows"]
    assert s.cols.tolist() == g["submatrix_0_2_3_2"]["cols"]
    for case in G["submatrix_reduce"]:
        a = pairs_dcsr(case["size"], case["k"])
        assert dcsr_digest(O.submatrix(a, case["i"], case["j"], case["nrows"], case["ncols"])) == case["submatrix"]
        assert dcsr_digest(O.reduce(a)) == case["reduce"]
