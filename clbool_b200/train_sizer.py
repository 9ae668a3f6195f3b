"""Train the row-size predictor on R-MAT products and write its checkpoint.

    python -m clbool_b200.train_sizer [--scales 14 15 16 17 18 19] [--eval-scale 21]
                                      [--out clbool_b200/sizer_rmat.npz]

Training data: for every R-MAT scale s (edge factor 16, a,b,c = 0.57,0.19,0.19,
seed s) the six row features of A*A and the exact nnz of every C row, both
from the library's kernels (row_features, and row_nnz -- the symbolic pass
alone).  Training: Adam in the library's CUDA kernels.  Evaluation on a larger
scale (symbolic pass only, since C itself does not fit next to its slots):
the mean absolute error in log2, the share of rows whose exact size exceeds
the capacity the learned SpGEMM would give them (the fallback rate), and the
slots allocated relative to the exact nnz and to the upper bound.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import gen
from .core import DeviceBuffer, create_controls, matrix_dcsr_cpu
from .ops import matrix_dcsr_from_cpu
from .sizing import (DEFAULT_CHECKPOINT, DEFAULT_MARGIN_LOG2, DEFAULT_SLACK, FEATURE_SCALE, NUM_FEATURES, RowSizer,
                     row_features, row_nnz, targets_from_row_nnz)


def rmat_dcsr(ctl, scale: int):
    r, c = gen.rmat(scale, seed=scale)
    rpt, rows, cols = gen.to_dcsr(r, c)
    n = 1 << scale
    return matrix_dcsr_from_cpu(ctl, matrix_dcsr_cpu(rpt, rows, cols), n, n)


def harvest(ctl, scale: int):
    """(features f32[n, 6], row nnz u32[n], products u32[n]) of A*A, A = R-MAT(scale)."""
    a = rmat_dcsr(ctl, scale)
    n = a.nzr()
    feat, work = row_features(ctl, a, a)
    nnz = row_nnz(ctl, a, a)
    return feat.to_host(n * NUM_FEATURES).reshape(n, NUM_FEATURES), nnz.to_host(n), work.to_host(n), a.ncols()


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


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--scales", type=int, nargs="+", default=[14, 15, 16, 17, 18, 19])
    ap.add_argument("--eval-scale", type=int, default=21)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=DEFAULT_CHECKPOINT)
    args = ap.parse_args(argv)

    ctl = create_controls(0, 0)
    t0 = time.time()
    feats, targets = [], []
    for s in args.scales:
        f, nnz, _, _ = harvest(ctl, s)
        feats.append(f)
        targets.append(targets_from_row_nnz(nnz))
        print(f"scale {s}: {len(nnz)} rows", flush=True)
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
    meta = {"train_scales": args.scales, "train_rows": int(len(t)), "epochs": args.epochs, "batch": args.batch,
            "lr": args.lr, "seed": args.seed, "loss_initial": loss0, "loss_final": loss1,
            "train_seconds": round(train_s, 3), "eval": ev, "total_seconds": round(time.time() - t0, 1)}
    sizer.save(args.out, meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
