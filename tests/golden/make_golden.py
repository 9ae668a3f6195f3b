"""Generate tests/golden/golden.json from the reference's own CPU functions.

Run in a checkout where the reference sources are available and
``oracle/_ref/libclbool_ref.so`` has been built (``make -C oracle REF=<reference tree>``):

    python tests/golden/make_golden.py

Every case is produced by the reference's code (``coo_utils::*_cpu``,
``csr_cpu_from_pairs``) through ``oracle.Ref``; nothing here uses the
restated oracle or the CUDA library.  Inputs are regenerated in the tests
from the recorded generator parameters (the reference's FastRandom
generators are deterministic); large outputs are recorded as SHA-256 digests
of their arrays (rpt as little-endian uint64, rows/cols as uint32), small
ones inline.

Cases follow the reference's own test grids (test/test_operations.cpp,
test/test_procedures.cpp, test/check_test_utils.cpp) and known-answer tests.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")


def sha(a, dtype) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


def dcsr_digest(m: O.Dcsr) -> dict:
    nnz = len(m.cols)
    rpt = np.asarray(m.rpt, np.uint64) if nnz else np.zeros(0, np.uint64)
    return {"nnz": nnz, "nzr": len(m.rows) if nnz else 0, "rpt": sha(rpt, np.uint64),
            "rows": sha(m.rows if nnz else [], np.uint32), "cols": sha(m.cols, np.uint32)}


def coo_digest(rows, cols) -> dict:
    return {"nnz": len(rows), "rows": sha(rows, np.uint32), "cols": sha(cols, np.uint32)}


def csr_digest(c: O.Csr) -> dict:
    return {"nnz": len(c.cols), "rpt": sha(c.rpt, np.uint64), "cols": sha(c.cols, np.uint32)}


def main():
    R = O.Ref()
    g: dict = {"generator": "oracle/_ref (reference CPU functions)", "cases": {}}
    cases = g["cases"]

    # README / test_operations.cpp:279-319 example matrices (5x5).
    a_rows, a_cols = [0, 0, 0, 2, 2, 4], [0, 1, 4, 2, 3, 2]
    b_rows, b_cols = [1, 1, 2, 3, 3, 3, 5], [0, 4, 2, 2, 3, 4, 2]
    A = R.pairs_to_dcsr(a_rows, a_cols, 5, 5)
    B = R.pairs_to_dcsr(b_rows, b_cols, 5, 5)
    C = R.spgemm(A, B)
    S = R.coo_add(O.Coo(5, 5, np.array(a_rows, np.uint32), np.array(a_cols, np.uint32)),
                  O.Coo(5, 5, np.array(b_rows, np.uint32), np.array(b_cols, np.uint32)))
    K = R.kronecker_pairs(O.Coo(5, 5, np.array(a_rows, np.uint32), np.array(a_cols, np.uint32)),
                          O.Coo(5, 5, np.array(b_rows, np.uint32), np.array(b_cols, np.uint32)), 5, 5)
    cases["readme"] = {
        "a": {"rows": a_rows, "cols": a_cols}, "b": {"rows": b_rows, "cols": b_cols}, "n": 5,
        "mxm": {"rpt": C.rpt.tolist(), "rows": C.rows.tolist(), "cols": C.cols.tolist()},
        "add": {"rows": S.rows.tolist(), "cols": S.cols.tolist()},
        "kron": {"rows": K.rows.tolist(), "cols": K.cols.tolist()},
    }

    # coo_constructor known answer (test_procedures.cpp:20-31): 11 -> 9.
    rows = [0, 0, 1, 1, 3, 4, 4, 5, 5, 5, 6]
    cols = [1, 2, 0, 3, 5, 2, 2, 0, 3, 3, 5]
    ur, uc = O.unique_pairs(rows, cols)
    assert len(ur) == 9
    cases["coo_constructor"] = {"rows": rows, "cols": cols, "n": 7, "nnz_after": 9,
                                "out_rows": ur.tolist(), "out_cols": uc.tolist()}

    # csr_cpu_from_pairs known answer (check_test_utils.cpp:21-39).
    pr = [0, 0, 0, 2, 2, 2, 3, 3, 3]
    pc = [0, 1, 3, 1, 3, 5, 1, 4, 5]
    cs = R.csr_from_pairs(pr, pc, 5, 7)
    cases["csr_from_pairs"] = {"rows": pr, "cols": pc, "m": 5, "n": 7, "rpt": cs.rpt.tolist(),
                               "out_cols": cs.cols.tolist()}

    # multiplication_hash grid (test_operations.cpp:127-134): C = A*A.
    grid = []
    for k in (50, 55):
        for size in range(3000, 4000, 200):
            r, c = R.generate_coo_pairs(size * k, size)
            A = R.pairs_to_dcsr(r, c, size, size)
            grid.append({"size": size, "k": k, "a": dcsr_digest(A), "c": dcsr_digest(R.spgemm(A, A))})
    cases["multiplication_hash"] = grid

    # multiplication_merge grid (test_operations.cpp:114-121).
    grid = []
    for k in range(0, 20):
        for size in range(0, 1000, 200):
            r, c = R.generate_coo_pairs(size * k, size)
            A = R.pairs_to_dcsr(r, c, size, size)
            grid.append({"size": size, "k": k, "a": dcsr_digest(A), "c": dcsr_digest(R.spgemm(A, A))})
    cases["multiplication_merge"] = grid

    # ESC / large-row fixtures (coo_utils.cpp:13-132; seeds of the reference's
    # kernel tests src/test/esc_kernels_test.cpp:18, large_rows_test.cpp:17).
    fx = []
    for which, seeds in (("esc", range(234523, 234543)), ("large", [342787282, 234523])):
        for seed in seeds:
            A, B = R.random_matrices(which, 1000, seed)
            if len(A.rows) != len(A.rpt) - 1 or len(B.rows) != len(B.rpt) - 1:
                continue  # the generator skipped a short row; arrays inconsistent
            fx.append({"which": which, "max_size": 1000, "seed": seed, "a": dcsr_digest(A), "b": dcsr_digest(B),
                       "c": dcsr_digest(R.spgemm(A, B))})
    cases["esc_large_fixtures"] = fx

    # addition_coo grids (test_operations.cpp:142-176), subsampled.
    grid = []
    for size in (0, 15, 300, 1005, 1995, 3000, 7500):
        for ka, kb in ((0, 0), (0, 5), (3, 0), (3, 9), (9, 9), (20, 25), (45, 60)):
            ar, ac = R.generate_coo_pairs(size * ka, size)
            br, bc = R.generate_coo_pairs(size * kb, size)
            s = R.coo_add(O.Coo(size, size, ar, ac), O.Coo(size, size, br, bc))
            grid.append({"size": size, "k_a": ka, "k_b": kb, "sum": coo_digest(s.rows, s.cols)})
    cases["addition_coo"] = grid

    # addition_csr grids (test_operations.cpp:182-217), subsampled; the
    # reference checks csr::matrix_addition against csr_cpu_from_pairs of the
    # COO sum (test/src/operations.cpp:420-452).
    grid = []
    for size in (0, 15, 600, 1000, 3800, 7000, 9990):
        for ka, kb in ((0, 0), (0, 7), (5, 0), (9, 9), (20, 35), (35, 20)):
            ar, ac = R.generate_coo_pairs(size * ka, size)
            br, bc = R.generate_coo_pairs(size * kb, size)
            s = R.coo_add(O.Coo(size, size, ar, ac), O.Coo(size, size, br, bc))
            grid.append({"size": size, "k_a": ka, "k_b": kb,
                         "sum": csr_digest(R.csr_from_pairs(s.rows, s.cols, size, size))})
    cases["addition_csr"] = grid

    # kronecker_dcsr (test_operations.cpp:258-277): A (x) A of
    # generate_coo_pairs(1000k, 10000), here for k = 0, 1 (output up to 1e6).
    grid = []
    for k in (0, 1):
        nnz = 1000 * k
        r, c = R.generate_coo_pairs(nnz, 10000)
        kp = R.kronecker_pairs(O.Coo(10000, 10000, r, c), O.Coo(10000, 10000, r, c), 10000, 10000)
        grid.append({"nnz": nnz, "size": 10000, "kron": coo_digest(kp.rows, kp.cols)})
    cases["kronecker_dcsr"] = grid

    # prefix sums (test_procedures.cpp:9-14): fill_random_buffer(n, 3).
    grid = []
    for n in (1, 10000, 250000, 1190000):
        v = R.fill_random_buffer(n, 3)
        ex = np.concatenate([[0], np.cumsum(v.astype(np.uint64))[:-1]]).astype(np.uint32)
        grid.append({"n": n, "input": sha(v, np.uint32), "scan": sha(ex, np.uint32), "total": int(v.sum())})
    cases["prefix_sum"] = grid

    # bitonic sort (test_procedures.cpp:2-7): fill_random_matrix(n) sorted.
    grid = []
    for n in (15, 1500, 4980):
        r, c = R.fill_random_matrix(n)
        key = np.sort((r.astype(np.uint64) << np.uint64(32)) | c)
        grid.append({"n": n, "input_rows": sha(r, np.uint32), "input_cols": sha(c, np.uint32),
                     "rows": sha((key >> np.uint64(32)).astype(np.uint32), np.uint32),
                     "cols": sha((key & np.uint64(0xFFFFFFFF)).astype(np.uint32), np.uint32)})
    cases["bitonic_sort"] = grid

    # reduce / submatrix: the README example (test_operations.cpp:309-310) and
    # the reference's submatrix / reduce test shapes (test_operations.cpp:52-106,
    # operations.cpp:84-166) with seeded ranges (the reference draws them from
    # std::random_device).
    Ar = R.pairs_to_dcsr(a_rows, a_cols, 5, 5)
    rr = R.reduce(Ar)
    rs = R.submatrix(Ar, 0, 2, 3, 2)
    cases["readme"]["reduce"] = {"rpt": rr.rpt.tolist(), "rows": rr.rows.tolist(), "cols": rr.cols.tolist()}
    cases["readme"]["submatrix_0_2_3_2"] = {"rpt": rs.rpt.tolist(), "rows": rs.rows.tolist(),
                                            "cols": rs.cols.tolist()}
    rng = np.random.default_rng(2024)
    grid = []
    for size, k in ((5, 3), (400, 7), (995, 19), (1800, 30), (5000, 45)):
        r, c = R.generate_coo_pairs(size * k, size)
        a = R.pairs_to_dcsr(r, c, size, size)
        i1, i2, i3, i4 = (int(x) for x in rng.integers(0, size + 1, 4))
        i, nr, j, nc = min(i1, i2), abs(i1 - i2), min(i3, i4), abs(i3 - i4)
        sub = R.submatrix(a, i, j, nr, nc)
        red = R.reduce(a)
        grid.append({"size": size, "k": k, "i": i, "j": j, "nrows": nr, "ncols": nc,
                     "submatrix": dcsr_digest(sub), "reduce": dcsr_digest(red)})
    cases["submatrix_reduce"] = grid

    with open(OUT, "w") as f:
        json.dump(g, f, indent=1, sort_keys=True)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
