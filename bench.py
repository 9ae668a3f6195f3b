"""Benchmark: boolean SpGEMM intermediate products/s on R-MAT scale-20 A*A.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--scale 20] [--form two_pass|learned]

One step = one product C = A*A of the synthetic R-MAT scale-20 graph by
itself (2^20 vertices, edge factor 16, a/b/c/d = .57/.19/.19/.05,
duplicates removed, self-loops kept) by the learned-sized single pass
(default; the exact two-pass dcsr::matrix_multiplication_hash is timed beside
it), producing C on the GPU.  `value` is products/s with A resident in HBM;
`e2e` is the same metric through the public API with host buffers (pinned
H2D of A, D2H of all of C inside the timed region).  With N > 1 ranks
(torchrun) rank 0 generates A and broadcasts it into every rank's HBM with
NCCL (clbool_b200.sharded), and every rank computes the C rows of its share
of A's rows (balanced by products) against its own copy; no collective
touches the timed data path.

`--impl reference` times the reference's own CPU implementation
(coo_utils::matrix_multiplication_cpu, compiled from the reference sources
into oracle/_ref) on a bounded sample of A's rows with all host threads, and
reports the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "bool SpGEMM products/s: learned-sized vs two-pass, same GPU, bit-exact"
UNIT = "products/s"
HBM_FALLBACK_GBS = 6650.0


# ------------------------------------------------------------------ helpers --
def peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def load_gen():
    """clbool_b200/gen.py (numpy only) loaded by file path, so that the
    reference arm generates its inputs without importing the package (whose
    import loads the CUDA library)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("clbool_b200_gen", os.path.join(ROOT, "clbool_b200", "gen.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def rmat_a(scale: int):
    gen = load_gen()
    r, c = gen.rmat(scale, seed=1)
    rpt, rows, cols = gen.to_dcsr(r, c)
    return 1 << scale, rpt, rows, cols


def rmat_config(scale: int, nnz_a: int, products: int, world: int, row_fraction: float = 1.0) -> dict:
    """The workload's identity, the same in both arms."""
    return {"workload": f"rmat_s{scale}_AxA" + (f"_rows{row_fraction:g}" if row_fraction < 1.0 else ""),
            "scale": scale, "edge_factor": 16, "abcd": [0.57, 0.19, 0.19, 0.05], "seed": 1,
            "nnz_A": nnz_a, "products": products, "parallelism": f"rows{world}"}


def bin_of(p: np.ndarray, bound: np.ndarray) -> np.ndarray:
    """The accumulator bin of every row under the default tuning (mirrors
    bin_of in spgemm_kernels.cuh)."""
    b = np.full(p.shape, 11, np.int32)
    b[p > (1 << 17)] = 10
    b[p > (1 << 20)] = 9
    for lim, k in ((4096, 8), (2048, 7), (1024, 6), (512, 5)):
        b[(p <= 4096) & (bound <= lim)] = k
    for lim, k in ((256, 4), (128, 3), (64, 2), (32, 1), (16, 13), (8, 12)):
        b[p <= lim] = k
    b[p == 0] = 0
    return b


KERNEL_BIN = {"bitmap": (9, 10, 11), "hash8k": 8, "hash4k": 7, "hash2k": 6, "hash1k": 5, "cta_esc4096": 8,
              "cta_esc2048": 7, "cta_esc1024": 6, "cta_esc512": 5, "esc256": 4, "esc128": 3, "esc16": 13, "esc8": 12,
              "esc64": 2, "esc32": 1}


def algorithmic_bytes(kernel: str, a_len: np.ndarray, work: np.ndarray, c_len: np.ndarray, ncols: int,
                      bound: np.ndarray | None = None) -> int:
    """Bytes the accumulator launch `kernel` must move for its rows, by the
    per-row model: A row pointer pair + row id (12 B), per A entry its column
    and B's row pointer pair (12 B), every product's B column (4 B), and for
    the numeric pass C's columns (4 B each) plus C's row pointer and id (12 B);
    the symbolic pass writes one 4-byte count per row instead."""
    symbolic = kernel.endswith("_symbolic")
    base = kernel.rsplit("_", 1)[0] if symbolic or kernel.endswith("_numeric") else kernel
    if base not in KERNEL_BIN:
        return 0
    bins = bin_of(work, np.minimum(work, ncols) if bound is None else bound)
    m = np.isin(bins, np.atleast_1d(KERNEL_BIN[base]))
    rows = int(m.sum())
    reads = 12 * rows + 12 * int(a_len[m].sum()) + 4 * int(work[m].sum())
    if not symbolic:
        return reads + 4 * int(c_len[m].sum()) + 12 * rows
    return reads + 4 * rows


# --------------------------------------------------------------- our arm --
def make_mxm(form: str, ctl, cb, sizer_path: str, tune=None):
    """The public call one step makes: (A, B, stats) -> C."""
    if form == "learned":
        from clbool_b200 import sizing
        sizer = sizing.RowSizer.load(ctl, sizer_path)
        return lambda A, B, stats=None: sizing.matrix_multiplication_learned(ctl, None, A, B, sizer, stats=stats,
                                                                             tune=tune)
    if form == "esc":
        return lambda A, B, stats=None: cb.dcsr.matrix_multiplication(ctl, None, A, B, stats=stats)
    if form == "two_pass_kept":
        kept = cb.dcsr.tuning("two_pass_kept")
        return lambda A, B, stats=None: cb.dcsr.matrix_multiplication_tuned(ctl, None, A, B, kept, stats=stats)
    return lambda A, B, stats=None: cb.dcsr.matrix_multiplication_hash(ctl, None, A, B, stats=stats)


def timed_steps(ctl, mxm, A, B, steps: int, l2_flush, barrier, srows, dev, want_c_len: bool):
    """K steps, each bracketed by a CUDA event pair on the library's stream
    (the whole call, host-side gaps included); the library's per-launch
    profile records (also CUDA events on that stream) attribute the time to
    kernels.  L2 is flushed between steps, outside the events."""
    import torch
    stream = torch.cuda.ExternalStream(ctl.stream, device=f"cuda:{dev}")
    ev_ms, kern_ms, prof_tot, launches, st, c_len = [], [], {}, 0, {}, None
    with ClockSampler(dev) as clk:
        barrier()
        ctl.sync()
        t0 = time.perf_counter()
        for k in range(steps):
            l2_flush()
            ctl.profile(True)
            st = {}
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            c = mxm(A, B, st)
            e1.record(stream)
            e1.synchronize()
            prof = ctl.profile_read()
            ctl.profile(False)
            launches += st["kernel_launches"]
            ev_ms.append(e0.elapsed_time(e1))
            kern_ms.append(sum(v[1] for v in prof.values()))
            for name, (cnt, ms) in prof.items():
                a, b = prof_tot.get(name, (0, 0.0))
                prof_tot[name] = (a + cnt, b + ms)
            if want_c_len and k == steps - 1 and c.nnz():
                crpt = c.rpt_gpu().to_host(c.nzr() + 1).astype(np.int64)
                crow = c.rows_gpu().to_host(c.nzr())
                c_len = np.zeros(srows.size, np.int64)
                c_len[np.searchsorted(srows, crow)] = np.diff(crpt)
            del c
        ctl.sync()
        barrier()
        wall = time.perf_counter() - t0
    return {"ev_ms": ev_ms, "kern_ms": kern_ms, "prof": prof_tot, "launches": launches, "stats": st,
            "c_len": c_len, "wall": wall, "clocks": clk.summary()}


def reduce_over_ranks(dist, dev, my_ms: float, my_products: int, my_nnz: int):
    if dist is None:
        return my_ms, float(my_products), float(my_nnz)
    import torch
    t = torch.tensor([my_ms, float(my_products), float(my_nnz)], dtype=torch.float64, device=f"cuda:{dev}")
    mx = t.clone()
    dist.all_reduce(mx[:1], op=dist.ReduceOp.MAX)
    dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
    return float(mx[0]), float(t[1]), float(t[2])


def learned_bounds(ctl, cb, A, B, sizer_path: str, work: np.ndarray, ncols: int) -> np.ndarray:
    """The capacities the learned form gives A's rows (host restatement of its
    capacity rule), to attribute rows to accumulator bins."""
    from clbool_b200 import sizing
    from clbool_b200.train_sizer import capacities
    sizer = sizing.RowSizer.load(ctl, sizer_path)
    feat, _ = sizing.row_features(ctl, A, B)
    pred = sizer.predict(feat, A.nzr()).to_host(A.nzr())
    return capacities(pred, work, ncols, sizing.DEFAULT_MARGIN_LOG2, sizing.DEFAULT_SLACK)


def run_ours(args, rank: int, world: int, dist) -> dict | None:
    import clbool_b200 as cb
    from clbool_b200 import sharded
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    ctl = cb.create_controls(0, dev)
    n = 1 << args.scale
    # rank 0 generates A; every other rank receives it by an NCCL broadcast
    # into its own HBM (A is both operands: B = A)
    A0 = None
    if rank == 0:
        _, rpt, rows, cols = rmat_a(args.scale)
        A0 = cb.matrix_dcsr_from_cpu(ctl, cb.matrix_dcsr_cpu(rpt, rows, cols), n)
    A_full = sharded.broadcast_dcsr(ctl, A0, 0) if world > 1 else A0
    if rank != 0:
        h = cb.matrix_dcsr_from_gpu(ctl, A_full)  # host copy: row sampling and the end-to-end leg
        rpt, rows, cols = h.rpt.astype(np.uint64), h.rows, h.cols
    nnz_a = cols.size
    work_buf, total_products = cb.dcsr.workload(ctl, A_full, A_full)
    work = work_buf.to_host(rows.size).astype(np.int64)
    # left operand: A itself, or (for profiling) a seeded sample of its rows
    lrpt, lrows, lcols = rpt, rows, cols
    if args.row_fraction < 1.0:
        pick = _row_sample(rows.size, args.row_fraction, seed=3)
        lrpt, lrows, lcols = _sub_dcsr(rpt, rows, cols, pick)
        work = work[pick]
    lo, hi = sharded.partition(work, world)[rank]
    srpt = (lrpt[lo:hi + 1] - lrpt[lo]).astype(np.uint64)
    srows, scols = lrows[lo:hi], lcols[int(lrpt[lo]):int(lrpt[hi])]
    A = cb.matrix_dcsr_from_cpu(ctl, cb.matrix_dcsr_cpu(srpt, srows, scols), n) if hi > lo else \
        cb.matrix_dcsr.zeros(n, n)
    my_products = int(work[lo:hi].sum())
    a_len = np.diff(srpt.astype(np.int64))
    mywork = work[lo:hi]

    flush = cb.DeviceBuffer.empty(ctl, 256 << 20, np.uint8)

    def l2_flush():
        cb.lib.clb_fill_u32(ctl.handle, __import__("ctypes").c_void_p(flush.ptr), (256 << 20) // 4, 0)

    def barrier():
        if dist is not None:
            dist.barrier()

    mxm = make_mxm(args.form, ctl, cb, args.sizer)
    for _ in range(args.warmup):
        c = mxm(A, A_full)
        del c
    ctl.sync()
    run = timed_steps(ctl, mxm, A, A_full, args.steps, l2_flush, barrier, srows, dev, True)
    st = run["stats"]
    total_ms, products_all, nnz_all = reduce_over_ranks(dist, dev, sum(run["ev_ms"]), my_products, st.get("nnz", 0))
    ms_per_step = total_ms / args.steps
    value = products_all / (ms_per_step / 1e3)

    # the same workload through the exact two-pass form, for the comparison
    compare = None
    if args.form != "two_pass" and not args.no_compare:
        mxm2 = make_mxm("two_pass", ctl, cb, args.sizer)
        for _ in range(max(1, args.warmup // 2)):
            c = mxm2(A, A_full)
            del c
        ctl.sync()
        run2 = timed_steps(ctl, mxm2, A, A_full, args.steps, l2_flush, barrier, srows, dev, False)
        t2, _, _ = reduce_over_ranks(dist, dev, sum(run2["ev_ms"]), my_products, 0)
        v2 = products_all / (t2 / args.steps / 1e3)
        compare = {"form": "two_pass", "value": v2, "ms_per_step": t2 / args.steps,
                   f"{args.form}_over_two_pass": value / v2,
                   "kernels_ms_per_step": {k: round(v[1] / args.steps, 3) for k, v in
                                           sorted(run2["prof"].items(), key=lambda kv: -kv[1][1])}}
        if args.form != "two_pass_kept":
            # the exact two-pass form keeping its symbolic pass's bitmaps
            mxm3 = make_mxm("two_pass_kept", ctl, cb, args.sizer)
            for _ in range(max(1, args.warmup // 2)):
                c = mxm3(A, A_full)
                del c
            ctl.sync()
            run3 = timed_steps(ctl, mxm3, A, A_full, args.steps, l2_flush, barrier, srows, dev, False)
            t3, _, _ = reduce_over_ranks(dist, dev, sum(run3["ev_ms"]), my_products, 0)
            v3 = products_all / (t3 / args.steps / 1e3)
            compare["two_pass_kept"] = {
                "value": v3, "ms_per_step": t3 / args.steps, f"{args.form}_over_two_pass_kept": value / v3,
                "kernels_ms_per_step": {k: round(v[1] / args.steps, 3) for k, v in
                                        sorted(run3["prof"].items(), key=lambda kv: -kv[1][1])}}

    # roofline of the dominant kernel (largest device time in the timed steps)
    peak, peak_kind = peaks()
    prof_tot = run["prof"]
    top_name, (top_launches, top_ms) = max(prof_tot.items(), key=lambda kv: kv[1][1])
    bound = None
    if args.form == "learned":
        bound = learned_bounds(ctl, cb, A, A_full, args.sizer, mywork, n)
    elif args.form == "esc":
        bound = mywork
    c_len = run["c_len"]
    alg = algorithmic_bytes(top_name, a_len, mywork, c_len if c_len is not None else np.zeros_like(mywork), n, bound)
    if top_name == "bitmap_numeric" and "bitmap_expand" in prof_tot:
        # the bitmap rows that kept their bitmap in their slot are emitted by
        # bitmap_expand (one launch per call as well): the pair does the rows' work
        top_ms += prof_tot["bitmap_expand"][1]
        top_name = "bitmap_numeric+bitmap_expand"
    per_launch_ms = top_ms / max(top_launches, 1)
    achieved = alg / (per_launch_ms / 1e3) / 1e9 if alg else None
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get(f"{top_name}@rmat_s{args.scale}")
        except Exception:
            traffic = None

    # end to end through the public API with host buffers
    e2e = run_e2e(args, ctl, cb, n, srpt, srows, scols, A_full, my_products, dist, dev, mxm)

    if rank != 0:
        return None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic", "impl": "ours",
        "config": rmat_config(args.scale, int(nnz_a), int(products_all), world=world,
                              row_fraction=args.row_fraction),
        "form": args.form, "nnz_C": int(nnz_all),
        "l2": "256 MiB device memset between steps, outside the step events; C (>30 GB) also exceeds L2",
        "roofline": {"bound": "hbm", "kernel": top_name, "achieved": achieved, "peak": peak,
                     "peak_source": peak_kind, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "alg_bytes_per_launch": alg, "launch_ms": per_launch_ms},
        "kernels_ms_per_step": {k: round(v[1] / args.steps, 3) for k, v in sorted(prof_tot.items(),
                                                                                 key=lambda kv: -kv[1][1])},
        "kernel_ms_per_step_sum": sum(run["kern_ms"]) / args.steps,
        "e2e": e2e, "gpu_launches": run["launches"], "clocks": run["clocks"], "wall_s": run["wall"],
    }
    if args.form in ("learned", "esc"):
        line["form_stats"] = {k: st.get(k) for k in ("capacity", "fallback_rows", "spilled_rows", "nzr", "nnz")}
    if compare is not None:
        line["compare"] = compare
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(n, rpt, rows, cols, work)
    return line


E2E_BLOCKS = 8  # row blocks of the end-to-end call (copy of one overlaps the next's product)


def run_e2e(args, ctl, cb, n, srpt, srows, scols, A_full, products, dist, dev, mxm) -> dict:
    """products/s through the public API: pinned host A -> device, then
    C = A*B delivered into pinned host arrays by clb_dcsr_spgemm_to_host (row
    blocks: each block's copy overlaps the next block's product), per step."""
    import ctypes
    from clbool_b200 import batched, sizing
    lib = cb.lib

    def pinned(nbytes):
        p = ctypes.c_void_p()
        cb.core.check(lib.clb_host_alloc(max(nbytes, 1), ctypes.byref(p)), "host_alloc")
        return p

    h_rpt, h_rows, h_cols = pinned(srpt.nbytes), pinned(srows.nbytes), pinned(scols.nbytes)
    ctypes.memmove(h_rpt, srpt.ctypes.data, srpt.nbytes)
    ctypes.memmove(h_rows, srows.ctypes.data, srows.nbytes)
    ctypes.memmove(h_cols, scols.ctypes.data, scols.nbytes)
    # size of C, to stage the read-back in pinned memory
    c0 = mxm(cb.matrix_dcsr_from_cpu(ctl, cb.matrix_dcsr_cpu(srpt, srows, scols), n), A_full)
    c_nzr, c_nnz = c0.nzr(), c0.nnz()
    c_bytes = (8 * (c_nzr + 1) + 4 * c_nzr + 4 * c_nnz) if c_nnz else 0
    h_c = pinned(c_bytes)
    del c0
    sizer = sizing.RowSizer.load(ctl, args.sizer) if args.form == "learned" else None
    tune = ({"esc": batched.tuning(form="single_pass"), "two_pass_kept": batched.tuning(form="two_pass_kept")}
            .get(args.form))
    steps = max(1, min(args.steps, 3))
    times = []
    for _ in range(steps):
        if dist is not None:
            dist.barrier()
        ctl.sync()
        t0 = time.perf_counter()
        d_rpt = cb.DeviceBuffer.empty(ctl, srpt.size, np.uint64)
        d_rows = cb.DeviceBuffer.empty(ctl, max(srows.size, 1), np.uint32)
        d_cols = cb.DeviceBuffer.empty(ctl, max(scols.size, 1), np.uint32)
        lib.clb_memcpy_h2d(ctl.handle, ctypes.c_void_p(d_rpt.ptr), h_rpt, srpt.nbytes)
        lib.clb_memcpy_h2d(ctl.handle, ctypes.c_void_p(d_rows.ptr), h_rows, srows.nbytes)
        lib.clb_memcpy_h2d(ctl.handle, ctypes.c_void_p(d_cols.ptr), h_cols, scols.nbytes)
        A = cb.matrix_dcsr(d_rpt, d_rows, d_cols, n, n, scols.size, srows.size)
        if c_nnz:
            base = h_c.value
            got = sizing.matrix_multiplication_to_host(ctl, A, A_full, base, base + 8 * (c_nzr + 1),
                                                       base + 8 * (c_nzr + 1) + 4 * c_nzr, c_nzr, c_nnz,
                                                       sizer=sizer, blocks=E2E_BLOCKS, tune=tune)
            assert got == (c_nzr, c_nnz), got
        del A, d_rpt, d_rows, d_cols
        ctl.sync()
        dt = time.perf_counter() - t0
        if dist is not None:
            import torch
            t = torch.tensor([dt], dtype=torch.float64, device=f"cuda:{dev}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t[0])
        times.append(dt)
    lib.clb_host_free(h_rpt)
    lib.clb_host_free(h_rows)
    lib.clb_host_free(h_cols)
    lib.clb_host_free(h_c)
    tot_products = products
    if dist is not None:
        import torch
        t = torch.tensor([float(products)], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t)
        tot_products = float(t[0])
    sec = statistics.median(times)
    return {"value": tot_products / sec, "unit": UNIT, "h2d_bytes_per_step": int(srpt.nbytes + srows.nbytes + scols.nbytes),
            "d2h_bytes_per_step": int(c_bytes), "s_per_step": sec, "steps": steps,
            "call": "clb_dcsr_spgemm_to_host", "row_blocks": E2E_BLOCKS}


# ------------------------------------------------------------ CPU baselines --
def _row_sample(rows_n: int, frac: float, seed: int = 7) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(rows_n, size=max(1, int(rows_n * frac)), replace=False))


def _sub_dcsr(rpt, rows, cols, pick):
    lens = (rpt[pick + 1] - rpt[pick]).astype(np.int64)
    srpt = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    idx = np.concatenate([np.arange(int(rpt[i]), int(rpt[i + 1])) for i in pick]) if pick.size else np.zeros(0, np.int64)
    return srpt, rows[pick], cols[idx]


def cpu_baseline(n, rpt, rows, cols, work) -> dict:
    """The oracle's multithreaded CPU product on a seeded sample of A's rows."""
    import oracle as O
    threads = O.set_threads(os.cpu_count() or 1)
    pick = _row_sample(rows.size, 0.10)
    srpt, srows, scols = _sub_dcsr(rpt, rows, cols, pick)
    A = O.Dcsr(n, n, srpt, srows, scols)
    B = O.Dcsr(n, n, rpt, rows, cols)
    t0 = time.perf_counter()
    C = O.spgemm(A, B)
    dt = time.perf_counter() - t0
    p = int(work[pick].sum())
    del C
    return {"value": p / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"10% of A's stored rows (seed 7): {pick.size} rows, {p} products, {dt:.2f} s"}


def c1_cpu(ra, ca, rb, cb_, n: int, products: int, gpu_product, gpu_sum, reps: int = 5) -> dict:
    """CPU legs of the 4096^2 Poisson pair, the one configuration where the
    reference's own CPU functions are tractable in full: its
    coo_utils::matrix_multiplication_cpu (coo_utils.cpp:470-514) and
    matrix_addition_cpu (coo_utils.cpp:315-324) on the whole pair, single
    threaded as written, each result compared with the GPU's; plus the
    oracle's multithreaded product (the port baseline)."""
    import oracle as O
    A = O.coo_to_dcsr(O.Coo(n, n, ra, ca))
    B = O.coo_to_dcsr(O.Coo(n, n, rb, cb_))

    def med(fn):
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            r = fn()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts), r

    threads = O.set_threads(os.cpu_count() or 1)
    t, _ = med(lambda: O.spgemm(A, B))
    res = {"cpu_baseline": {"value": products / t, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": f"whole 4096^2 pair, median of {reps} calls ({t * 1e6:.0f} us)"}}
    if O.ref_available():
        R = O.Ref()
        tm, Cr = med(lambda: R.spgemm(A, B))
        ta, Sr = med(lambda: R.coo_add(O.Coo(n, n, ra, ca), O.Coo(n, n, rb, cb_)))
        rpt, rows, cols = gpu_product
        res["reference"] = {
            "kind": "reference", "cores": 1, "calls": reps,
            "spgemm": {"function": "coo_utils::matrix_multiplication_cpu", "us": tm * 1e6,
                       "products_per_s": products / tm,
                       "bit_exact_vs_gpu": bool(np.array_equal(np.asarray(Cr.rpt, np.uint64), rpt) and
                                                np.array_equal(Cr.rows, rows) and np.array_equal(Cr.cols, cols))},
            "coo_add": {"function": "coo_utils::matrix_addition_cpu", "us": ta * 1e6,
                        "entries_per_s": Sr.rows.size / ta,
                        "bit_exact_vs_gpu": bool(np.array_equal(Sr.rows, gpu_sum[0]) and
                                                 np.array_equal(Sr.cols, gpu_sum[1]))}}
    return res


def run_reference(args) -> dict:
    """The reference's own CPU product (matrix_multiplication_cpu) on bounded
    samples of A's rows, one sample per host thread."""
    import concurrent.futures as cf
    import oracle as O
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "reference CPU library (oracle/_ref) was not built"}
    R = O.Ref()
    n, rpt, rows, cols = rmat_a(args.scale)
    B = O.Dcsr(n, n, rpt, rows, cols)
    prod = O.workload(B, B).astype(np.int64)
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(11)
    # The reference's product looks every A entry's column up by a linear
    # std::find over B's stored rows (coo_utils.cpp:487), so its cost is
    # ~ entries * nzr(B); size each thread's sample for a few seconds.
    per_thread_rows = max(1, int(args.ref_rows))
    samples = [np.sort(rng.choice(rows.size, size=per_thread_rows, replace=False)) for _ in range(threads)]

    def one(pick):
        srpt, srows, scols = _sub_dcsr(rpt, rows, cols, pick)
        R.spgemm(O.Dcsr(n, n, srpt, srows, scols), B)
        return int(prod[pick].sum())

    def step():
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            p = sum(ex.map(one, samples))
        return p, time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    ps, ts = 0, 0.0
    for _ in range(args.steps):
        p, t = step()
        ps += p
        ts += t
    value = ps / ts
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ts / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic", "impl": "reference",
            "config": rmat_config(args.scale, int(cols.size), int(prod.sum()), world=args.gpus),
            "form": "coo_utils::matrix_multiplication_cpu",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{threads} threads x {per_thread_rows} random stored rows of A per step "
                                       f"(coo_utils::matrix_multiplication_cpu)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ------------------------------------------------------ secondary workloads --
def _event_ms(stream, fn, reps: int):
    """Per-call device time (CUDA events on the library's stream), median."""
    import torch
    out = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        out.append(e0.elapsed_time(e1))
    return statistics.median(out)


def run_batch(args) -> dict:
    """256 independent pairs (n log-uniform in [2^10, 2^18], power-law rows:
    exponent 2.1, mean 6, at most 4096; seed per pair): one batched call
    (default and autotuned tuning) against one call per pair."""
    import torch

    import clbool_b200 as cb
    from clbool_b200 import gen
    ctl = cb.create_controls(0, 0)
    stream = torch.cuda.ExternalStream(ctl.stream, device="cuda:0")
    rng = np.random.default_rng(17)
    ns = np.exp(rng.uniform(np.log(1 << 10), np.log(1 << 18), size=args.pairs)).astype(int)
    pairs = []
    for k, n in enumerate(ns):
        n = int(n)
        mats = []
        for s in (2 * k + 1, 2 * k + 2):
            r, c = gen.power_law_rows(n, n, 2.1, 6.0, 4096, seed=1000 + s)
            rpt, rows, cols = gen.to_dcsr(r, c)
            mats.append(cb.matrix_dcsr_from_cpu(ctl, cb.matrix_dcsr_cpu(rpt, rows, cols), n))
        pairs.append(tuple(mats))
    products = sum(cb.dcsr.workload(ctl, a, b)[1] for a, b in pairs)
    default = cb.dcsr.tuning()
    best, tried = cb.dcsr.autotune(ctl, pairs)
    st = {}

    def batched(t):
        def f():
            outs = cb.dcsr.matrix_multiplication_batched(ctl, pairs, tune=t, stats=st)
            del outs
        return f

    def sequential():
        for a, b in pairs:
            c = cb.dcsr.matrix_multiplication_hash(ctl, None, a, b)
            del c

    from clbool_b200 import sizing
    sizer_path = args.sizer_mixed if os.path.exists(args.sizer_mixed) else args.sizer
    sizer = sizing.RowSizer.load(ctl, sizer_path)
    st_l = {}

    def learned():
        outs = cb.dcsr.matrix_multiplication_batched_learned(ctl, pairs, sizer, tune=best, stats=st_l)
        del outs

    # the exact two-pass form under the autotuned accumulator settings
    two_pass_best = cb.dcsr.tuning("two_pass", best.warp_max, best.bitmap_min, best.bitmap_threads, best.small_lanes)

    for _ in range(args.warmup):
        batched(best)()
        learned()
        sequential()
    ms_best = _event_ms(stream, batched(best), args.steps)
    ms_default = _event_ms(stream, batched(default), args.steps)
    ms_learned = _event_ms(stream, learned, args.steps)
    ms_two_pass_best = _event_ms(stream, batched(two_pass_best), args.steps)
    ms_seq = _event_ms(stream, sequential, max(1, args.steps // 2))
    batched(best)()
    # the host-sync-free batched form recorded once into a CUDA graph, replayed
    from clbool_b200 import batched as bt
    cap = bt.CapturedBatch(ctl, pairs, tune=best)
    graph = bt.Graph(ctl, cap.enqueue)
    for _ in range(max(3, args.warmup)):
        graph.launch()
    got = cap.result()
    ref = cb.dcsr.matrix_multiplication_batched(ctl, pairs, tune=best)
    exact = True
    for (rpt, rws, cls), c in zip(got, ref):
        h = cb.matrix_dcsr_from_gpu(ctl, c) if c.nnz() else None
        if h is None:
            exact &= len(cls) == 0
        else:
            exact &= bool(np.array_equal(rpt, h.rpt) and np.array_equal(rws, h.rows) and np.array_equal(cls, h.cols))
    del ref
    ms_graph = _event_ms(stream, graph.launch, args.steps)
    graph.close()
    # the learned-sized capture form, recorded once and replayed
    capl = bt.CapturedBatch(ctl, pairs, tune=best, sizer=sizer)
    graphl = bt.Graph(ctl, capl.enqueue)
    for _ in range(max(3, args.warmup)):
        graphl.launch()
    gotl = capl.result()
    exact_l = not capl.fell_back and all(
        np.array_equal(x[2], y[2]) and np.array_equal(x[1], y[1]) and np.array_equal(x[0], y[0])
        for x, y in zip(gotl, got))
    ms_graph_l = _event_ms(stream, graphl.launch, args.steps)
    graphl.close()
    return {"metric": METRIC, "workload": f"batch{args.pairs}_powerlaw", "value": products / (ms_best / 1e3),
            "unit": UNIT, "ms_per_step": ms_best, "steps": args.steps, "warmup": args.warmup, "n_gpus": 1,
            "higher_is_better": True, "dtype": "u32", "data": "synthetic",
            "config": {"workload": f"batch{args.pairs}_powerlaw", "pairs": args.pairs, "n_min": int(ns.min()),
                       "n_max": int(ns.max()), "products": int(products), "nnz_C": int(st.get("nnz", 0)),
                       "row_lengths": "power law 2.1, mean 6, max 4096"},
            "autotuned": best.as_dict(), "default_ms": ms_default, "sequential_ms": ms_seq,
            "batched_over_sequential": ms_seq / ms_best,
            "learned_batched": {"ms": ms_learned, "products_per_s": products / (ms_learned / 1e3),
                                "over_two_pass_batched_default": ms_default / ms_learned,
                                "two_pass_batched_same_tuning_ms": ms_two_pass_best,
                                "over_two_pass_batched_same_tuning": ms_two_pass_best / ms_learned,
                                "tuning": best.as_dict(),
                                "capacity": st_l.get("capacity"), "spilled_rows": st_l.get("spilled_rows"),
                                "fallback_rows": st_l.get("fallback_rows"),
                                "graph_replay_ms": ms_graph_l, "graph_slot_capacity": capl.slot_capacity,
                                "graph_bit_exact_vs_upper_bound_graph": exact_l,
                                "sizer": os.path.basename(sizer_path)},
            "graph_replay": {"ms": ms_graph, "products_per_s": products / (ms_graph / 1e3),
                             "bit_exact_vs_batched": exact, "slot_capacity": cap.slot_capacity},
            "kernel_launches_per_batch": st.get("kernel_launches"),
            "candidates_ms": sorted(((t, round(m, 3)) for t, m in tried), key=lambda x: x[1])}


def run_rmat_add(args) -> dict:
    """The headline workload's second operation: CSR addition C + A with
    C = A*A at R-MAT scale 20 (entries/s of C + A; 64 seeded rows of the sum
    checked against the union of the operands' rows)."""
    import ctypes

    import torch

    import clbool_b200 as cb
    from clbool_b200 import sizing
    ctl = cb.create_controls(0, 0)
    stream = torch.cuda.ExternalStream(ctl.stream, device="cuda:0")
    n, rpt, rows, cols = rmat_a(args.scale)
    A = cb.matrix_dcsr_from_cpu(ctl, cb.matrix_dcsr_cpu(rpt, rows, cols), n)
    sizer = sizing.RowSizer.load(ctl, args.sizer)
    C = sizing.matrix_multiplication_learned(ctl, None, A, A, sizer)
    Cc, Ac = cb.dcsr_to_csr(ctl, C), cb.dcsr_to_csr(ctl, A)
    del C
    S = cb.csr.matrix_addition(ctl, None, Cc, Ac)
    nnz_c, nnz_s = Cc.nnz(), S.nnz()

    def row(m, r, rp):
        lo, hi = int(rp[r]), int(rp[r + 1])
        seg = np.empty(hi - lo, np.uint32)
        if hi > lo:
            cb.lib.clb_memcpy_d2h(ctl.handle, seg.ctypes.data_as(ctypes.c_void_p),
                                  ctypes.c_void_p(m.cols_gpu().ptr + 4 * lo), 4 * (hi - lo))
        return seg
    crp, srp = Cc.rpt_gpu().to_host(n + 1), S.rpt_gpu().to_host(n + 1)
    arp = np.zeros(n + 1, np.int64)
    arp[rows.astype(np.int64) + 1] = np.diff(rpt.astype(np.int64))
    arp = np.cumsum(arp)
    exact = True
    for r in np.random.default_rng(5).choice(n, 64, replace=False):
        want = np.union1d(row(Cc, r, crp), cols[arp[r]:arp[r + 1]])
        exact &= bool(np.array_equal(row(S, r, srp), want))
    del S

    def step():
        out = cb.csr.matrix_addition(ctl, None, Cc, Ac)
        del out
    for _ in range(max(1, args.warmup - 1)):
        step()
    ms = _event_ms(stream, step, max(3, args.steps))
    alg = 4 * (cols.size + nnz_c + nnz_s) + 8 * (n + 1) * 3
    peak, kind = peaks()
    achieved = alg / (ms / 1e3) / 1e9
    return {"metric": "bool CSR addition entries/s (C + A)", "workload": f"rmat_s{args.scale}_csr_add",
            "value": nnz_s / (ms / 1e3), "unit": "entries/s", "ms_per_step": ms, "n_gpus": 1, "data": "synthetic",
            "higher_is_better": True, "dtype": "u32",
            "config": {"workload": f"rmat_s{args.scale}_C_plus_A", "nnz_A": int(cols.size), "nnz_C": int(nnz_c),
                       "nnz_sum": int(nnz_s), "rows_checked": 64, "rows_match_union": exact},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "peak_source": kind, "unit": "GB/s",
                         "frac": achieved / peak, "alg_bytes": alg}}


def run_small(args) -> dict:
    """4096 x 4096, Poisson(8) rows (columns uniform without replacement, seeds
    1 and 2): latency of one A*B (each form) and of one COO A+B."""
    import torch

    import clbool_b200 as cb
    from clbool_b200 import gen
    ctl = cb.create_controls(0, 0)
    stream = torch.cuda.ExternalStream(ctl.stream, device="cuda:0")
    n = 4096
    mats = []
    for seed in (1, 2):
        r, c = gen.poisson_rows(n, n, 8.0, seed=seed)
        mats.append((r, c))
    (ra, ca), (rb, cb_) = mats
    A = cb.matrix_dcsr_from_cpu(ctl, cb.matrix_dcsr_cpu(*gen.to_dcsr(ra, ca)), n)
    B = cb.matrix_dcsr_from_cpu(ctl, cb.matrix_dcsr_cpu(*gen.to_dcsr(rb, cb_)), n)
    Ac = cb.matrix_coo.from_host(ctl, ra, ca, n, n)
    Bc = cb.matrix_coo.from_host(ctl, rb, cb_, n, n)
    products = cb.dcsr.workload(ctl, A, B)[1]
    best, _ = cb.dcsr.autotune(ctl, [(A, B)])
    out = {}
    calls = {
        "hash_two_pass": lambda st: cb.dcsr.matrix_multiplication_hash(ctl, None, A, B, stats=st),
        "esc_single_pass": lambda st: cb.dcsr.matrix_multiplication(ctl, None, A, B, stats=st),
        "autotuned": lambda st: cb.dcsr.matrix_multiplication_tuned(ctl, None, A, B, best, stats=st),
        "coo_add": lambda st: cb.coo.matrix_addition(ctl, None, Ac, Bc),
    }
    for name, f in calls.items():
        st = {}
        for _ in range(max(3, args.warmup)):
            f(st)
        ms = _event_ms(stream, lambda: f(st), max(20, args.steps))
        out[name] = {"us": ms * 1e3, "launches": st.get("kernel_launches")}
        if name != "coo_add":
            out[name]["products_per_s"] = products / (ms / 1e3)
    out["autotuned"]["tuning"] = best.as_dict()
    # the host-sync-free form recorded once into a CUDA graph and replayed
    from clbool_b200 import batched
    cap = batched.CapturedBatch(ctl, [(A, B)], tune=best)
    graph = batched.Graph(ctl, cap.enqueue)
    for _ in range(max(3, args.warmup)):
        graph.launch()
    got = cap.result()[0]
    want = cb.matrix_dcsr_from_gpu(ctl, cb.dcsr.matrix_multiplication_hash(ctl, None, A, B))
    exact = bool(np.array_equal(got[0], want.rpt) and np.array_equal(got[1], want.rows)
                 and np.array_equal(got[2], want.cols))
    ms = _event_ms(stream, graph.launch, max(20, args.steps))
    out["graph_replay"] = {"us": ms * 1e3, "products_per_s": products / (ms / 1e3), "bit_exact_vs_two_pass": exact}
    ms = _event_ms(stream, cap.enqueue, max(20, args.steps))
    out["capture_form_direct"] = {"us": ms * 1e3, "products_per_s": products / (ms / 1e3)}
    graph.close()
    coo_sum = cb.coo.matrix_addition(ctl, None, Ac, Bc)
    got_sum = (coo_sum.rows_gpu().to_host(coo_sum.nnz()), coo_sum.cols_gpu().to_host(coo_sum.nnz()))
    cpu = c1_cpu(ra, ca, rb, cb_, n, int(products), (want.rpt, want.rows, want.cols), got_sum)
    return {"metric": METRIC, "workload": "poisson4096", "unit": UNIT, "n_gpus": 1, "data": "synthetic",
            "config": {"workload": "poisson4096_AxB", "n": n, "lambda": 8, "products": int(products),
                       "nnz_A": int(ra.size), "nnz_B": int(rb.size)}, "calls": out,
            "cpu_baseline": cpu["cpu_baseline"], "reference_cpu": cpu.get("reference")}


def run_cfpq(args) -> dict:
    """Bounded closure C <- C v sum_i C L_i over 3 uniform label matrices
    (n = 2^18, average degree 3 each, seeds 1-3), each iteration's three
    products in one batched call; stops at a fixpoint, 64 iterations, or
    before an iteration of more than 4e9 products."""
    import torch

    import clbool_b200 as cb
    from clbool_b200 import cfpq, gen
    ctl = cb.create_controls(0, 0)
    n = 1 << 18
    labels = []
    for seed in (1, 2, 3):
        r, c = gen.poisson_rows(n, n, 3.0, seed=seed)
        labels.append(cb.matrix_dcsr_from_cpu(ctl, cb.matrix_dcsr_cpu(*gen.to_dcsr(r, c)), n))
    out = {}
    # accumulator tuning: autotuned on the second iteration's product C_2 M
    C2, _ = cfpq.closure(ctl, labels, max_iters=2)
    M = cfpq.union(ctl, [cfpq.identity(ctl, n)] + labels)
    best, _ = cb.dcsr.autotune(ctl, [(C2, M)])
    best_b, _ = cb.dcsr.autotune(ctl, [(C2, L) for L in labels])  # the batched iteration's three products
    del C2
    from clbool_b200 import sizing
    sizer_path = args.sizer_mixed if os.path.exists(args.sizer_mixed) else args.sizer
    sizer = sizing.RowSizer.load(ctl, sizer_path)
    out["sizer"] = os.path.basename(sizer_path)
    for method, tune, sz in (("fused", None, None), ("fused_autotuned", best, None), ("fused_learned", None, sizer),
                             ("fused_learned_autotuned", best, sizer), ("batched", None, None),
                             ("batched_autotuned", best_b, None), ("batched_learned", None, sizer),
                             ("batched_learned_autotuned", best_b, sizer)):
        m = "batched" if method.startswith("batched") else "fused"
        # warm-up: the whole bounded closure, so that the timed run's largest
        # product (the last iteration's) is not the first of its size in the
        # process (the first one grows the stream-ordered memory pool, which
        # took from 0.05 to 1.5 s here)
        del_c, _ = cfpq.closure(ctl, labels, max_iters=64, max_products=int(4e9), method=m, tune=tune, sizer=sz)
        del del_c
        torch.cuda.synchronize()
        C, hist = cfpq.closure(ctl, labels, max_iters=64, max_products=int(4e9), method=m, tune=tune, sizer=sz)
        out[method] = {"iterations": hist, "final_nnz": C.nnz(), "stop": hist[-1].get("stop"),
                       "products": sum(h["products"] for h in hist), "ms": sum(h["ms"] for h in hist)}
        if tune is not None:
            out[method]["tuning"] = tune.as_dict()
        del C
    f = out["fused_autotuned"]
    return {"metric": METRIC, "workload": "cfpq3_n2^18_deg3", "value": f["products"] / (f["ms"] / 1e3),
            "unit": UNIT, "n_gpus": 1, "data": "synthetic", "higher_is_better": True,
            "config": {"workload": "cfpq3_n2^18_deg3", "n": n, "labels": 3, "degree": 3, "max_products": 4e9,
                       "value_method": "fused (C <- C (I v L1 v L2 v L3)), autotuned on C_2 M"},
            "methods": out}


def run_kron(args) -> dict:
    """DCSR Kronecker product of two R-MAT scale-11 graphs (seeds 1, 2)."""
    import torch

    import clbool_b200 as cb
    from clbool_b200 import gen
    ctl = cb.create_controls(0, 0)
    stream = torch.cuda.ExternalStream(ctl.stream, device="cuda:0")
    mats = []
    for seed in (1, 2):
        r, c = gen.rmat(11, seed=seed)
        mats.append(cb.matrix_dcsr_from_cpu(ctl, cb.matrix_dcsr_cpu(*gen.to_dcsr(r, c)), 1 << 11))
    A, B = mats
    k = cb.dcsr.kronecker_product(ctl, None, A, B)
    nnz, nzr = k.nnz(), k.nzr()
    del k

    def f():
        out = cb.dcsr.kronecker_product(ctl, None, A, B)
        del out
    for _ in range(max(3, args.warmup)):
        f()
    ms = _event_ms(stream, f, max(5, args.steps))
    out_bytes = 4 * nnz + 8 * (nzr + 1) + 4 * nzr
    peak, src = peaks()
    return {"metric": "Kronecker output entries/s", "workload": "kron_rmat11_x_rmat11", "value": nnz / (ms / 1e3),
            "unit": "entries/s", "ms_per_step": ms, "n_gpus": 1, "data": "synthetic", "higher_is_better": True,
            "config": {"workload": "kron_rmat11_x_rmat11", "nnz_A": A.nnz(), "nnz_B": B.nnz(), "nnz_C": nnz,
                       "nzr_C": nzr},
            "roofline": {"bound": "hbm", "achieved": out_bytes / (ms / 1e3) / 1e9, "peak": peak, "peak_source": src,
                         "unit": "GB/s", "frac": out_bytes / (ms / 1e3) / 1e9 / peak,
                         "alg_bytes": out_bytes}}


def run_primitives(args) -> dict:
    """The primitives under the products, each on an input larger than L2
    (126 MB) and timed with CUDA events on the library's stream (median of
    `steps` calls, L2 flushed before each): COO addition of two R-MAT
    scale-20 graphs (seeds 1 and 2, 2 x 16M entries, merge path), the COO
    sort of the first graph's pairs shuffled (LSD radix), the prefix sum of
    2^28 uint32 entries, and the DCSR -> CSR -> DCSR conversions of the first
    graph.  Achieved GB/s are algorithmic bytes (each input read once, each
    output written once) over the call's time."""
    import ctypes

    import torch

    import clbool_b200 as cb
    from clbool_b200 import gen
    ctl = cb.create_controls(0, 0)
    stream = torch.cuda.ExternalStream(ctl.stream, device="cuda:0")
    n = 1 << 20
    (ra, ca), (rb, cbb) = gen.rmat(20, seed=1), gen.rmat(20, seed=2)
    Ac = cb.matrix_coo.from_host(ctl, ra, ca, n, n)
    Bc = cb.matrix_coo.from_host(ctl, rb, cbb, n, n)
    flush = cb.DeviceBuffer.empty(ctl, 256 << 20, np.uint8)
    peak, src = peaks()
    reps = max(3, args.steps)

    def timed(fn):
        out = []
        for _ in range(reps):
            cb.lib.clb_fill_u32(ctl.handle, ctypes.c_void_p(flush.ptr), (256 << 20) // 4, 0)
            out.append(_event_ms(stream, fn, 1))
        return statistics.median(out)

    res = {}
    S = cb.coo.matrix_addition(ctl, None, Ac, Bc)
    nnz_s = S.nnz()
    del S
    ms = timed(lambda: cb.coo.matrix_addition(ctl, None, Ac, Bc))
    alg = 8 * (ra.size + rb.size) + 8 * nnz_s
    res["coo_add_rmat20_x2"] = {"ms": ms, "entries_per_s": nnz_s / (ms / 1e3), "alg_bytes": alg,
                                "gbs": alg / (ms / 1e3) / 1e9, "nnz_a": int(ra.size), "nnz_b": int(rb.size),
                                "nnz_c": int(nnz_s)}
    perm = np.random.default_rng(9).permutation(ra.size)
    pr, pc = ra[perm], ca[perm]
    dr = cb.DeviceBuffer.from_host(ctl, pr, np.uint32)
    dc = cb.DeviceBuffer.from_host(ctl, pc, np.uint32)

    sort_ms = []
    for _ in range(reps):
        cb.lib.clb_memcpy_h2d(ctl.handle, ctypes.c_void_p(dr.ptr), pr.ctypes.data_as(ctypes.c_void_p), pr.nbytes)
        cb.lib.clb_memcpy_h2d(ctl.handle, ctypes.c_void_p(dc.ptr), pc.ctypes.data_as(ctypes.c_void_p), pc.nbytes)
        sort_ms.append(_event_ms(stream, lambda: cb.coo.sort_arrays(ctl, dr, dc, pr.size), 1))
    ok = bool(np.array_equal(dr.to_host(), ra) and np.array_equal(dc.to_host(), ca))
    ms = statistics.median(sort_ms)
    alg = 16 * pr.size
    res["coo_sort_rmat20_shuffled"] = {"ms": ms, "pairs_per_s": pr.size / (ms / 1e3), "alg_bytes": alg,
                                       "gbs": alg / (ms / 1e3) / 1e9, "pairs": int(pr.size), "sorted_ok": ok}
    m = 1 << 28
    buf = cb.DeviceBuffer.empty(ctl, m, np.uint32)
    cb.lib.clb_fill_u32(ctl.handle, ctypes.c_void_p(buf.ptr), m, 1)
    tot = ctypes.c_uint64()
    ms = timed(lambda: cb.lib.clb_prefix_sum_u32(ctl.handle, ctypes.c_void_p(buf.ptr), m, ctypes.byref(tot)))
    res["prefix_sum_u32_2e28"] = {"ms": ms, "entries_per_s": m / (ms / 1e3), "alg_bytes": 8 * m,
                                  "gbs": 8 * m / (ms / 1e3) / 1e9}
    del buf
    A = cb.coo_to_dcsr_shallow(ctl, Ac)
    ms = timed(lambda: cb.dcsr_to_csr(ctl, A))
    alg = 8 * (A.nzr() + 1) + 4 * A.nzr() + 8 * (n + 1)
    res["dcsr_to_csr_rmat20"] = {"ms": ms, "alg_bytes": alg, "gbs": alg / (ms / 1e3) / 1e9}
    Acsr = cb.dcsr_to_csr(ctl, A)
    ms = timed(lambda: cb.csr_to_dcsr(ctl, Acsr))
    res["csr_to_dcsr_rmat20"] = {"ms": ms, "alg_bytes": alg, "gbs": alg / (ms / 1e3) / 1e9}
    for v in res.values():
        if "gbs" in v:
            v["frac"] = v["gbs"] / peak
    return {"metric": "primitive throughput", "workload": "primitives_rmat20", "unit": "GB/s", "n_gpus": 1,
            "data": "synthetic", "peak_gbs": peak, "peak_source": src, "calls": res,
            "config": {"workload": "primitives_rmat20", "l2": "256 MiB memset before each timed call"}}


def run_rmat21(args) -> dict:
    """Learned-form A*A at R-MAT scale 21 (seed 21, the scale the predictor is
    evaluated on; never trained on): C (2.65e10 entries, 106 GB) does not fit
    beside its slots, so A's rows run in blocks balanced by products and each
    block's C is discarded after its nnz is read.  Reports products/s, the
    slots over nnz, spilled and fallback rows."""
    import torch

    import clbool_b200 as cb
    from clbool_b200 import gen, sizing
    ctl = cb.create_controls(0, 0)
    stream = torch.cuda.ExternalStream(ctl.stream, device="cuda:0")
    scale = 21
    n = 1 << scale
    r, c = gen.rmat(scale, seed=scale)
    rpt, rows, cols = gen.to_dcsr(r, c)
    del r, c
    A_full = cb.matrix_dcsr_from_cpu(ctl, cb.matrix_dcsr_cpu(rpt, rows, cols), n)
    work = cb.dcsr.workload(ctl, A_full, A_full)[0].to_host(rows.size).astype(np.int64)
    sizer = sizing.RowSizer.load(ctl, args.sizer)
    blocks = max(1, args.blocks)
    tot = {"products": 0, "nnz": 0, "capacity": 0, "spilled_rows": 0, "fallback_rows": 0, "ms": 0.0}
    from clbool_b200 import sharded
    for k, (lo, hi) in enumerate(sharded.partition(work, blocks)):
        if hi <= lo:
            continue
        srpt = (rpt[lo:hi + 1] - rpt[lo]).astype(np.uint64)
        A = cb.matrix_dcsr_from_cpu(ctl, cb.matrix_dcsr_cpu(srpt, rows[lo:hi], cols[int(rpt[lo]):int(rpt[hi])]), n)
        st = {}
        # one untimed call first: the memory pool grows to the block's footprint
        # and every kernel is loaded, as in the scale-20 warm-up steps
        c = sizing.matrix_multiplication_learned(ctl, None, A, A_full, sizer)
        del c
        ms = _event_ms(stream, lambda: sizing.matrix_multiplication_learned(ctl, None, A, A_full, sizer, stats=st), 1)
        for key in ("products", "nnz", "capacity", "spilled_rows", "fallback_rows"):
            tot[key] += int(st.get(key, 0))
        tot["ms"] += ms
        del A
    return {"metric": METRIC, "workload": "rmat_s21_AxA_learned_row_blocks", "value": tot["products"] / (tot["ms"] / 1e3),
            "unit": UNIT, "n_gpus": 1, "data": "synthetic", "higher_is_better": True,
            "config": {"workload": "rmat_s21_AxA_learned_row_blocks", "scale": scale, "seed": scale,
                       "row_blocks": blocks, "nnz_A": int(cols.size)},
            "ms": tot["ms"], "products": tot["products"], "nnz_C": tot["nnz"],
            "slots_over_nnz": tot["capacity"] / max(tot["nnz"], 1), "spilled_rows": tot["spilled_rows"],
            "fallback_rows": tot["fallback_rows"], "rows": int(rows.size)}


# --------------------------------------------------------------------- main --
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--form", default=None, choices=["two_pass", "two_pass_kept", "learned", "esc"],
                    help="default: learned when the packaged predictor checkpoint exists, else two_pass")
    ap.add_argument("--sizer", default=os.path.join(ROOT, "clbool_b200", "sizer_rmat.npz"),
                    help="predictor checkpoint of the learned form")
    ap.add_argument("--sizer-mixed", default=os.path.join(ROOT, "clbool_b200", "sizer_mixed.npz"),
                    help="predictor checkpoint of the batch and closure workloads (trained on R-MAT, power-law, "
                         "uniform and closure-step products); the R-MAT one when absent")
    ap.add_argument("--no-compare", action="store_true", help="skip timing the two-pass form beside it")
    ap.add_argument("--row-fraction", type=float, default=1.0,
                    help="left operand = this seeded fraction of A's stored rows (profiling captures)")
    ap.add_argument("--ref-rows", type=int, default=48)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="rmat",
                    choices=["rmat", "batch", "poisson4096", "cfpq", "kron", "rmat21", "rmat_add", "primitives"],
                    help="rmat: the headline A*A; batch / poisson4096: secondary workloads (own JSON line)")
    ap.add_argument("--pairs", type=int, default=256)
    ap.add_argument("--blocks", type=int, default=4, help="row blocks of the scale-21 run")
    args = ap.parse_args()
    if args.workload != "rmat":
        fn = {"batch": run_batch, "poisson4096": run_small, "cfpq": run_cfpq, "kron": run_kron,
              "rmat21": run_rmat21, "rmat_add": run_rmat_add, "primitives": run_primitives}[args.workload]
        print(json.dumps(fn(args)), flush=True)
        return
    if args.form is None:
        args.form = "learned" if os.path.exists(args.sizer) else "two_pass"

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist_mod
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = dist_mod
    try:
        line = run_ours(args, rank, world, dist)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
