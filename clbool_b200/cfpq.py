"""Fixpoint driver of the boolean closure used by CFPQ/RPQ-style callers
(no counterpart in the reference library; its users build such loops on top
of dcsr::matrix_multiplication and the additions).

    C_0 = start (default: L_1 v L_2 v ... v L_k)
    C_{t+1} = C_t v (C_t L_1) v ... v (C_t L_k)        until nnz(C) is stable

Two equivalent iteration methods:
  "batched": the k products C_t L_i as ONE batched call
             (dcsr.matrix_multiplication_batched, or the learned-sized
             dcsr.matrix_multiplication_batched_learned when a sizer is
             given), then the union C_t v P_1 v ... v P_k in one pass
             (batched.matrix_union);
  "fused":   C_{t+1} = C_t M with M = I v L_1 v ... v L_k built once (the
             boolean semiring distributes: C v C L_1 v ... = C (I v L_1 v ...)),
             i.e. one product per iteration (learned-sized when a sizer is
             given) and no union pass.
On random graphs the closure tends to the
dense n x n matrix, so the loop is bounded: it stops at a fixpoint, after
`max_iters` iterations, or before an iteration whose products would exceed
`max_products` (a memory guard: the batch needs room for about that many
candidate columns), and reports nnz and timing per iteration.
"""
from __future__ import annotations

import time

import numpy as np

from .batched import (matrix_multiplication_batched, matrix_multiplication_batched_learned,
                      matrix_multiplication_tuned, matrix_union)
from .core import Controls, matrix_dcsr, matrix_dcsr_cpu
from .ops import matrix_dcsr_from_cpu, workload


def union(controls: Controls, mats: list[matrix_dcsr], tune=None) -> matrix_dcsr:
    """Boolean sum of DCSR matrices of one shape in one pass
    (batched.matrix_union: the SpGEMM accumulators merge every output row's
    rows of the operands)."""
    return matrix_union(controls, mats, tune)


def identity(controls: Controls, n: int) -> matrix_dcsr:
    ids = np.arange(n, dtype=np.uint32)
    return matrix_dcsr_from_cpu(controls, matrix_dcsr_cpu(np.arange(n + 1, dtype=np.uint64), ids, ids), n)


def closure(controls: Controls, labels: list[matrix_dcsr], start: matrix_dcsr | None = None, max_iters: int = 64,
            max_products: int | None = None, tune=None, method: str = "fused", sizer=None):
    """(C, history): the bounded fixpoint and one dict per iteration
    (iteration, nnz, products, ms, stop reason on the last).  `sizer`
    (sizing.RowSizer, optional): the products run in the learned-sized
    single pass; the result does not depend on it."""
    if not labels:
        raise ValueError("closure needs at least one label matrix")
    if method not in ("fused", "batched"):
        raise ValueError("method must be 'fused' or 'batched'")
    C = union(controls, labels) if start is None else start
    M = union(controls, [identity(controls, labels[0].nrows())] + list(labels)) if method == "fused" else None
    history = [{"iteration": 0, "nnz": C.nnz(), "products": 0, "ms": 0.0}]
    reason = "max_iters"
    for it in range(1, max_iters + 1):
        products = (workload(controls, C, M)[1] if M is not None else
                    sum(workload(controls, C, L)[1] for L in labels))
        if max_products is not None and products > max_products:
            reason = "max_products"
            break
        t0 = time.perf_counter()
        if M is not None:
            if sizer is not None:
                from .sizing import matrix_multiplication_learned
                Cn = matrix_multiplication_learned(controls, None, C, M, sizer, tune=tune)
            else:
                Cn = matrix_multiplication_tuned(controls, None, C, M, tune)
        else:
            if sizer is not None:
                prods = matrix_multiplication_batched_learned(controls, [(C, L) for L in labels], sizer, tune=tune)
            else:
                prods = matrix_multiplication_batched(controls, [(C, L) for L in labels], tune=tune)
            Cn = union(controls, [C] + prods, tune)
        controls.sync()
        ms = (time.perf_counter() - t0) * 1e3
        history.append({"iteration": it, "nnz": Cn.nnz(), "products": int(products), "ms": ms})
        stable = Cn.nnz() == C.nnz()
        C = Cn
        if stable:
            reason = "fixpoint"
            break
    history[-1]["stop"] = reason
    return C, history
