"""Train the row-size predictor and write its checkpoint.

    python -m clbool_b200.train_sizer [--family rmat|mixed] [--scales 14 15 16 17 18 19]
                                      [--eval-scale 21] [--out PATH]

Training data: the six row features of a product and the exact nnz of every
C row, both from the library's kernels (row_features, and row_nnz -- the
symbolic pass alone).
  * family "rmat" (clbool_b200/sizer_rmat.npz): A*A for every R-MAT scale s
    (edge factor 16, a,b,c = 0.57,0.19,0.19, seed s);
  * family "mixed" (clbool_b200/sizer_mixed.npz): the same R-MAT products
    plus products of other shapes -- independent pairs with power-law rows
    (exponent 2.1, mean 6, at most 4096; n log-uniform in [2^12, 2^18]),
    uniform rows (Poisson(8), n from 2^12 to 2^16), and the steps C_t M of a
    boolean closure over uniform label matrices (n = 2^14 and 2^16, degree
    3) -- whose rows collide far less than R-MAT's; rows of at most 1024
    products, which never get a learned slot, are subsampled to a tenth.
Training: Adam in the library's CUDA kernels.  Evaluation on a larger
R-MAT scale (symbolic pass only, since C itself does not fit next to its
slots) and, for the mixed family, on held-out power-law pairs and a closure
step: the mean absolute error in log2, the share of rows whose exact size
exceeds the capacity the learned SpGEMM would give them (the fallback rate),
and the slots allocated relative to the exact nnz and to the upper bound.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import gen
from .core import DeviceBuffer, create_controls, matrix_dcsr_cpu
from .ops import matrix_dcsr_from_cpu
from .sizing import (DEFAULT_CHECKPOINT, DEFAULT_MARGIN_LOG2, DEFAULT_SLACK, FEATURE_SCALE, MIXED_CHECKPOINT,
                     NUM_FEATURES, RowSizer, row_features, row_nnz, targets_from_row_nnz)


def rmat_dcsr(ctl, scale: int):
    r, c = gen.rmat(scale, seed=scale)
    rpt, rows, cols = gen.to_dcsr(r, c)
    n = 1 << scale
    return matrix_dcsr_from_cpu(ctl, matrix_dcsr_cpu(rpt, rows, cols), n, n)


def harvest_pair(ctl, a, b):
    """(features f32[n, 6], row nnz u32[n], products u32[n], ncols) of A*B."""
    n = a.nzr()
    feat, work = row_features(ctl, a, b)
    nnz = row_nnz(ctl, a, b)
    return feat.to_host(n * NUM_FEATURES).reshape(n, NUM_FEATURES), nnz.to_host(n), work.to_host(n), b.ncols()


def harvest(ctl, scale: int):
    """(features, row nnz, products, ncols) of A*A, A = R-MAT(scale)."""
    a = rmat_dcsr(ctl, scale)
    return harvest_pair(ctl, a, a)


def _dev(ctl, rc, n):
    rpt, rows, cols = gen.to_dcsr(*rc)
    return matrix_dcsr_from_cpu(ctl, matrix_dcsr_cpu(rpt, rows, cols), n, n)


def other_families(ctl, seed_base: int, count_pl: int = 40):
    """Products of other shapes than R-MAT A*A (see the module docstring)."""
    from . import cfpq
    rng = np.random.default_rng(seed_base)
    out = []
    for k, n in enumerate(np.exp(rng.uniform(np.log(1 << 12), np.log(1 << 18), size=count_pl)).astype(int)):
        n = int(n)
        a = _dev(ctl, gen.power_law_rows(n, n, 2.1, 6.0, 4096, seed=seed_base + 2 * k), n)
        b = _dev(ctl, gen.power_law_rows(n, n, 2.1, 6.0, 4096, seed=seed_base + 2 * k + 1), n)
        out.append(harvest_pair(ctl, a, b))
    for k, n in enumerate((1 << 12, 1 << 14, 1 << 16)):
        a = _dev(ctl, gen.poisson_rows(n, n, 8.0, seed=seed_base + 500 + 2 * k), n)
        b = _dev(ctl, gen.poisson_rows(n, n, 8.0, seed=seed_base + 501 + 2 * k), n)
        out.append(harvest_pair(ctl, a, b))
    for k, n in enumerate((1 << 14, 1 << 16)):
        labels = [_dev(ctl, gen.poisson_rows(n, n, 3.0, seed=seed_base + 700 + 3 * k + j), n) for j in range(3)]
        M = cfpq.union(ctl, [cfpq.identity(ctl, n)] + labels)
        C = cfpq.union(ctl, labels)
        for _ in range(3 if n <= (1 << 14) else 2):
            out.append(harvest_pair(ctl, C, M))
            C = cfpq.closure(ctl, labels, start=C, max_iters=1)[0]
    return out


def subsample_light(f, nnz, work, rng, keep: float = 0.1, light: int = 1024):
    """Rows of at most `light` products kept with probability `keep`."""
    m = (work > light) | (rng.random(work.size) < keep)
    return f[m], nnz[m], work[m]


def capacities(pred: np.ndarray, work: np.ndarray, ncols: int, margin_log2: float, slack: float) -> np.ndarray:
    """Host restatement of the capacity rule of the learned SpGEMM (for reporting)."""
    ub = np.minimum(work.astype(np.int64), ncols)
    c = np.exp2(np.minimum(pred.astype(np.float64) / FEATURE_SCALE + margin_log2, 40.0)) - 1.0 + slack
    k = np.where(c <= 1.0, 1, np.ceil(np.minimum(c, 4.0e9))).astype(np.int64)
    return np.where(ub == 0, 0, np.minimum(k, ub))


def evaluate(ctl, sizer: RowSizer, scale: int, margin_log2: float, slack: float) -> dict:
    f, nnz, work, ncols = harvest(ctl, scale)
    n = len(nnz)
    pred = sizer.predict(DeviceBuffer.from_host(ctl, f, np.float32), n).to_host(n)
    cap = capacities(pred, work, ncols, margin_log2, slack)
    t = targets_from_row_nnz(nnz)
    ub = np.minimum(work.astype(np.int64), ncols)
    return {"scale": scale, "rows": int(n), "nnz": int(nnz.astype(np.int64).sum()),
            "mae_log2": float(np.abs(pred - t).mean() / FEATURE_SCALE),
            "fallback_rate": float((nnz > cap).mean()),
            "slots_over_nnz": float(cap.sum() / max(1, nnz.astype(np.int64).sum())),
            "slots_over_upper_bound": float(cap.sum() / max(1, ub.sum())),
            "margin_log2": margin_log2, "slack": slack}


def evaluate_rows(sizer: RowSizer, ctl, parts, margin_log2: float, slack: float, label: str) -> dict:
    """The evaluation figures over harvested products (features, nnz, work, ncols)."""
    f = np.concatenate([p[0] for p in parts]).astype(np.float32)
    nnz = np.concatenate([p[1] for p in parts])
    work = np.concatenate([p[2] for p in parts])
    ncols = np.concatenate([np.full(len(p[1]), p[3], np.int64) for p in parts])
    n = len(nnz)
    pred = sizer.predict(DeviceBuffer.from_host(ctl, f, np.float32), n).to_host(n)
    cap = capacities(pred, work, ncols, margin_log2, slack)
    t = targets_from_row_nnz(nnz)
    ub = np.minimum(work.astype(np.int64), ncols)
    heavy = work > 4096  # the rows that get a learned slot
    return {"set": label, "rows": int(n), "learned_rows": int(heavy.sum()),
            "mae_log2_learned_rows": float(np.abs(pred - t)[heavy].mean() / FEATURE_SCALE) if heavy.any() else 0.0,
            "fallback_rate_learned_rows": float((nnz > cap)[heavy].mean()) if heavy.any() else 0.0,
            "slots_over_nnz_learned_rows": float(cap[heavy].sum() / max(1, nnz[heavy].astype(np.int64).sum())),
            "slots_over_upper_bound_learned_rows": float(cap[heavy].sum() / max(1, ub[heavy].sum()))}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--family", choices=["rmat", "mixed"], default="rmat")
    ap.add_argument("--scales", type=int, nargs="+", default=[14, 15, 16, 17, 18, 19])
    ap.add_argument("--eval-scale", type=int, default=21)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    if args.out is None:
        args.out = DEFAULT_CHECKPOINT if args.family == "rmat" else MIXED_CHECKPOINT

    ctl = create_controls(0, 0)
    t0 = time.time()
    feats, targets = [], []
    for s in args.scales:
        f, nnz, _, _ = harvest(ctl, s)
        feats.append(f)
        targets.append(targets_from_row_nnz(nnz))
        print(f"scale {s}: {len(nnz)} rows", flush=True)
    if args.family == "mixed":
        rng = np.random.default_rng(args.seed)
        for f, nnz, work, _ in other_families(ctl, seed_base=90000):
            f, nnz, _ = subsample_light(f, nnz, work, rng)
            feats.append(f)
            targets.append(targets_from_row_nnz(nnz))
        print(f"other families: {sum(len(t) for t in targets)} rows in all", flush=True)
    f = np.concatenate(feats).astype(np.float32)
    t = np.concatenate(targets)
    fd = DeviceBuffer.from_host(ctl, f, np.float32)
    td = DeviceBuffer.from_host(ctl, t, np.float32)
    sizer = RowSizer(ctl, seed=args.seed)
    loss0, _ = sizer.gradients(fd, td, len(t))
    t1 = time.time()
    sizer.train(fd, td, len(t), epochs=args.epochs, batch=args.batch, lr=args.lr, seed=args.seed)
    train_s = time.time() - t1
    loss1, _ = sizer.gradients(fd, td, len(t))
    ev = evaluate(ctl, sizer, args.eval_scale, DEFAULT_MARGIN_LOG2, DEFAULT_SLACK)
    meta = {"family": args.family, "train_scales": args.scales, "train_rows": int(len(t)), "epochs": args.epochs,
            "batch": args.batch, "lr": args.lr, "seed": args.seed, "loss_initial": loss0, "loss_final": loss1,
            "train_seconds": round(train_s, 3), "eval": ev}
    # held-out products of the other shapes (seeds the training never used)
    held = other_families(ctl, seed_base=777000, count_pl=24)
    meta["eval_other"] = [evaluate_rows(sizer, ctl, held[:24], DEFAULT_MARGIN_LOG2, DEFAULT_SLACK, "power-law pairs"),
                          evaluate_rows(sizer, ctl, held[24:27], DEFAULT_MARGIN_LOG2, DEFAULT_SLACK, "Poisson(8) pairs"),
                          evaluate_rows(sizer, ctl, held[27:], DEFAULT_MARGIN_LOG2, DEFAULT_SLACK, "closure steps")]
    meta["total_seconds"] = round(time.time() - t0, 1)
    sizer.save(args.out, meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
