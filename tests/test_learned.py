"""Learned row sizing: the predictor's kernels against the FP64 oracle, and the
learned single-pass SpGEMM bit-exact against the oracle's product.

The learned form has no counterpart in the reference; its result must equal
dcsr::matrix_multiplication_hash (src/dcsr/dcsr.hpp:32-36) on every input,
whatever the predictor says, because overflowing rows are recomputed."""
import numpy as np
import pytest

import oracle as O
from util import assert_dcsr_equal, from_device, pairs_dcsr, to_device

F = 6


def _rmat(scale, seed=None):
    from clbool_b200 import gen
    r, c = gen.rmat(scale, seed=scale if seed is None else seed)
    n = 1 << scale
    return O.coo_to_dcsr(O.Coo(n, n, r, c))


# --------------------------------------------------------------- CPU side --
def test_oracle_mlp_gradient_matches_autograd():
    """The oracle's hand-written FP64 backward equals torch autograd on the
    same BF16-rounded weights."""
    import torch
    rng = np.random.default_rng(3)
    npar = O.lib().orc_mlp_num_params()
    p = (rng.normal(size=npar) * 0.2).astype(np.float32)
    x = rng.random((257, F)).astype(np.float32)
    t = rng.random(257).astype(np.float32)
    loss, g, pred = O.mlp_grad(p, x, t)

    w = torch.tensor(p).to(torch.bfloat16).to(torch.float64).requires_grad_(True)
    H = 64
    o = 0
    W1 = w[o:o + H * F].view(H, F); o += H * F
    b1 = w[o:o + H]; o += H
    W2 = w[o:o + H * H].view(H, H); o += H * H
    b2 = w[o:o + H]; o += H
    w3 = w[o:o + H]; o += H
    b3 = w[o]
    X = torch.tensor(x, dtype=torch.float64)
    y = torch.relu(torch.relu(X @ W1.T + b1) @ W2.T + b2) @ w3 + b3
    L = ((y - torch.tensor(t, dtype=torch.float64)) ** 2).mean()
    L.backward()
    assert abs(L.item() - loss) < 1e-12 * max(1.0, abs(loss))
    np.testing.assert_allclose(pred, y.detach().numpy(), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(g, w.grad.numpy(), rtol=1e-9, atol=1e-12)


def test_oracle_row_features_small():
    # A row 0: cols {0, 2}; B row 0 has 3 entries, B row 2 has 1 -> P = 4
    a = O.coo_to_dcsr(O.Coo(4, 4, np.array([0, 0, 3], np.uint32), np.array([0, 2, 1], np.uint32)))
    b = O.coo_to_dcsr(O.Coo(4, 4, np.array([0, 0, 0, 2], np.uint32), np.array([0, 1, 3, 2], np.uint32)))
    f = O.row_features(a, b)
    assert f.shape == (2, F)
    np.testing.assert_allclose(f[0, :4] * 16, np.log2([3, 5, 4, 2]))
    np.testing.assert_allclose(f[1, :4] * 16, np.log2([2, 1, 1, 1]))  # B row 1 is empty
    np.testing.assert_allclose(f[:, 4], [0.0, 0.75])
    np.testing.assert_allclose(f[:, 5], np.log2(16 / 4) / 16)


# --------------------------------------------------------------- GPU side --
def _features(ctl, a, b):
    from clbool_b200 import sizing
    n = len(a.rows)
    feat, work = sizing.row_features(ctl, to_device(ctl, a), to_device(ctl, b))
    return feat, work, feat.to_host(n * F).reshape(n, F), work.to_host(n)


@pytest.mark.gpu
@pytest.mark.parametrize("scale", [10, 14])
def test_row_features_and_workload(controls, scale):
    a = _rmat(scale)
    _, _, f, w = _features(controls, a, a)
    np.testing.assert_allclose(f, O.row_features(a, a), rtol=0, atol=2e-6)
    assert np.array_equal(w, O.workload(a, a))


@pytest.mark.gpu
def test_row_features_hypersparse_rectangular(controls):
    a = pairs_dcsr(3000, 2, ncols=5000)
    b = O.coo_to_dcsr(O.Coo(5000, 700, *O.unique_pairs(*O.sort_pairs(
        np.random.default_rng(1).integers(0, 5000, 4000).astype(np.uint32),
        np.random.default_rng(2).integers(0, 700, 4000).astype(np.uint32)))))
    _, _, f, w = _features(controls, a, b)
    np.testing.assert_allclose(f, O.row_features(a, b), rtol=0, atol=2e-6)
    assert np.array_equal(w, O.workload(a, b))


@pytest.mark.gpu
@pytest.mark.parametrize("scale", [10, 15])
def test_row_nnz_exact(controls, scale):
    from clbool_b200 import sizing
    a = _rmat(scale)
    got = sizing.row_nnz(controls, to_device(controls, a), to_device(controls, a)).to_host(len(a.rows))
    assert np.array_equal(got, O.spgemm_row_nnz(a, a))


def _train_set(ctl, scale):
    from clbool_b200 import DeviceBuffer, sizing
    a = _rmat(scale)
    feat, _, f, _ = _features(ctl, a, a)
    t = sizing.targets_from_row_nnz(O.spgemm_row_nnz(a, a))
    return a, feat, f, DeviceBuffer.from_host(ctl, t, np.float32), t


@pytest.mark.gpu
def test_gradients_match_oracle(controls):
    """CUDA forward/backward (BF16 weights, FP32 accumulation) vs the FP64
    oracle on the same rounded weights: loss and gradient agree to FP32
    accumulation error."""
    from clbool_b200 import sizing
    _, feat, f, tdev, t = _train_set(controls, 12)
    n = len(t)
    s = sizing.RowSizer(controls, seed=7)
    for params in (s.get_params(), (np.random.default_rng(5).normal(size=sizing.num_params()) * 0.1).astype(np.float32)):
        s.set_params(params)
        loss, g = s.gradients(feat, tdev, n)
        rloss, rg, rpred = O.mlp_grad(params, f.astype(np.float32), t)
        assert abs(loss - rloss) <= 1e-4 * rloss + 1e-7
        rel = np.linalg.norm(g - rg) / np.linalg.norm(rg)
        assert rel < 1e-4, rel
        pred = s.predict(feat, n).to_host(n)
        np.testing.assert_allclose(pred, rpred, rtol=0, atol=5e-5)


@pytest.mark.gpu
def test_training_reduces_loss(controls):
    from clbool_b200 import sizing
    _, feat, f, tdev, t = _train_set(controls, 13)
    n = len(t)
    s = sizing.RowSizer(controls, seed=3)
    l0, _ = s.gradients(feat, tdev, n)
    s.train(feat, tdev, n, epochs=30, batch=1024, lr=2e-3, seed=1)
    l1, _ = s.gradients(feat, tdev, n)
    assert l1 < 0.1 * l0, (l0, l1)
    # the trained weights round-trip through the checkpoint API (the loss is
    # summed with FP32 atomics, so only its last bits may differ)
    p = s.get_params()
    s2 = sizing.RowSizer(controls, seed=99, params=p)
    assert np.array_equal(s2.get_params(), p)
    l2, _ = s2.gradients(feat, tdev, n)
    assert abs(l2 - l1) <= 1e-5 * l1


def _learned(ctl, a, b, sizer, margin=None, slack=None, tune=None):
    import clbool_b200 as cb
    from clbool_b200 import sizing
    kw = {"tune": tune}
    if margin is not None:
        kw["margin_log2"] = margin
    if slack is not None:
        kw["slack"] = slack
    st = {}
    c = sizing.matrix_multiplication_learned(ctl, None, to_device(ctl, a), to_device(ctl, b), sizer, stats=st, **kw)
    return from_device(ctl, c), st


@pytest.mark.gpu
@pytest.mark.parametrize("margin", [-1000.0, -2.0, 0.0, 1000.0])
def test_learned_bit_exact_any_predictor(controls, margin):
    """Untrained predictor, with capacities from one slot per row (margin
    -1000) to the exact upper bound (+1000): C is always the oracle's product."""
    from clbool_b200 import sizing
    s = sizing.RowSizer(controls, seed=11)
    for a, b, what in ((_rmat(12), None, "rmat12"), (pairs_dcsr(2000, 30), None, "pairs2000"),
                       (pairs_dcsr(1000, 40), pairs_dcsr(1000, 3), "pairs-rect")):
        b = a if b is None else b
        got, st = _learned(controls, a, b, s, margin=margin, slack=0.0)
        want = O.spgemm(a, b)
        assert_dcsr_equal(got, want, f"{what} margin {margin}")
        assert st["nnz"] == len(want.cols)
        ub = np.minimum(O.workload(a, b), b.ncols).astype(np.int64)
        assert st["capacity"] <= int(ub.sum())
        if margin >= 1000.0:
            assert st["fallback_rows"] == 0 and st["spilled_rows"] == 0
            assert st["capacity"] == int(ub.sum())
        if margin <= -1000.0:
            # rows up to 4096 products get their exact bound; the heavier ones
            # one slot, so exactly those with more than one output go to the
            # spill arena (all columns fit one bitmap chunk here)
            work = O.workload(a, b).astype(np.int64)
            heavy = work[work > 0] > 4096
            row_len = np.diff(want.rpt.astype(np.int64))
            assert st["fallback_rows"] == 0
            assert st["spilled_rows"] == int((heavy & (row_len > 1)).sum())


@pytest.mark.gpu
def test_learned_hypersparse_and_empty(controls):
    import clbool_b200 as cb
    from clbool_b200 import sizing
    s = sizing.RowSizer(controls, seed=2)
    z = O.coo_to_dcsr(O.Coo(100, 100, np.zeros(0, np.uint32), np.zeros(0, np.uint32)))
    a = pairs_dcsr(100, 3)
    for x, y in ((z, a), (a, z), (z, z)):
        got, st = _learned(controls, x, y, s)
        assert len(got.cols) == 0 and got.nrows == 100
    n = 1 << 20
    rng = np.random.default_rng(4)
    ra = np.sort(rng.choice(n, 300, replace=False)).astype(np.uint32)
    rows = np.repeat(ra, 5)
    cols = rng.integers(0, n, rows.size).astype(np.uint32)
    h = O.coo_to_dcsr(O.Coo(n, n, *O.unique_pairs(*O.sort_pairs(rows, cols))))
    got, _ = _learned(controls, h, h, s)
    assert_dcsr_equal(got, O.spgemm(h, h), "hypersparse")


@pytest.mark.gpu
def test_trained_predictor_gain(controls):
    """A predictor trained on R-MAT scales 11-13 and evaluated on scale 15:
    far fewer slots than the exact upper bound (the ESC form's capacity, i.e.
    no predictor), a minority of fallback rows, and still the oracle's
    product."""
    import clbool_b200 as cb
    from clbool_b200 import DeviceBuffer, sizing
    feats, targets = [], []
    for sc in (11, 12, 13):
        _, _, f, _, t = _train_set(controls, sc)
        feats.append(f)
        targets.append(t)
    f = np.concatenate(feats).astype(np.float32)
    t = np.concatenate(targets)
    s = sizing.RowSizer(controls, seed=5)
    s.train(DeviceBuffer.from_host(controls, f, np.float32), DeviceBuffer.from_host(controls, t, np.float32), len(t),
            epochs=40, batch=1024, lr=2e-3, seed=2)
    a = _rmat(15)
    got, st = _learned(controls, a, a, s)
    want = O.spgemm(a, a)
    assert_dcsr_equal(got, want, "rmat15 learned")
    ub = int(np.minimum(O.workload(a, a), a.ncols).astype(np.int64).sum())
    nzr = len(want.rows)
    assert st["capacity"] < 0.75 * ub, (st["capacity"], ub)
    assert st["capacity"] < 1.6 * len(want.cols), (st["capacity"], len(want.cols))
    # a small training set (scales 11-13, seconds of training): some rows
    # still fall back; the packaged predictor is tested separately
    assert st["fallback_rows"] + st["spilled_rows"] < 0.15 * nzr, st
    # without a predictor (ESC form: upper-bound capacity) the same product
    st_esc = {}
    c = cb.matrix_dcsr()
    cb.dcsr.matrix_multiplication(controls, c, to_device(controls, a), to_device(controls, a), stats=st_esc)
    assert st_esc["capacity"] == ub and st_esc["fallback_rows"] == 0


def test_packaged_checkpoint_metadata():
    """The packaged predictor: right size, trained on R-MAT scales 14-19 and
    evaluated on scale 21 with a small fallback rate."""
    meta_npz = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "..", "clbool_b200",
                                                  "sizer_rmat.npz"))
    import json
    meta = json.loads(str(meta_npz["meta"]))
    assert meta_npz["params"].size == O.lib().orc_mlp_num_params()
    assert meta["train_scales"] == [14, 15, 16, 17, 18, 19]
    assert meta["eval"]["scale"] == 21
    assert meta["eval"]["fallback_rate"] < 1e-3
    assert meta["eval"]["slots_over_upper_bound"] < 0.75


@pytest.mark.gpu
def test_packaged_checkpoint_rmat16(controls):
    from clbool_b200 import sizing
    s = sizing.RowSizer.load(controls)
    a = _rmat(16, seed=1)
    got, st = _learned(controls, a, a, s)
    want = O.spgemm(a, a)
    assert_dcsr_equal(got, want, "rmat16 packaged predictor")
    assert st["fallback_rows"] <= max(2, len(want.rows) // 1000)
    assert st["capacity"] < 1.5 * len(want.cols)


def _wide_pair(n, seed):
    rng = np.random.default_rng(seed)
    ra = np.repeat(np.arange(64, dtype=np.uint32), 40)
    ca = rng.integers(0, 3000, ra.size).astype(np.uint32)
    a = O.coo_to_dcsr(O.Coo(64, 3000, *O.unique_pairs(*O.sort_pairs(ra, ca))))
    rb = np.repeat(np.arange(3000, dtype=np.uint32), 200)
    cbb = rng.integers(0, n, rb.size).astype(np.uint32)
    b = O.coo_to_dcsr(O.Coo(3000, n, *O.unique_pairs(*O.sort_pairs(rb, cbb))))
    return a, b


@pytest.mark.gpu
@pytest.mark.parametrize("n", [(1 << 20) + 3, (1 << 21) + 5, (3 << 20) + 9])
@pytest.mark.parametrize("wide", ["cluster", "chunks"])
def test_learned_wide_rows(controls, n, wide):
    """Columns past one bitmap chunk but within four.  With a thread-block
    cluster per row the row's exact count is known after its one insertion
    pass, so rows over their slot spill in the same pass; walking the chunks
    one after another they can only be recomputed (fallback).  Either way C
    is the oracle's product."""
    from clbool_b200 import batched, sizing
    a, b = _wide_pair(n, 13)
    s = sizing.RowSizer(controls, seed=4)
    got, st = _learned(controls, a, b, s, margin=-1000.0, slack=0.0, tune=batched.tuning(wide_rows=wide))
    assert_dcsr_equal(got, O.spgemm(a, b), f"learned n={n} {wide}")
    if wide == "cluster":
        assert st["spilled_rows"] > 0 and st["fallback_rows"] == 0
    else:
        assert st["fallback_rows"] > 0 and st["spilled_rows"] == 0


@pytest.mark.gpu
def test_learned_fallback_on_wide_rows(controls):
    """Columns past four bitmap chunks (2^22 + 5): bitmap rows over their slot
    cannot spill (their count is only known after the last chunk), so they
    take the exact two-pass fallback; C is still the oracle's product."""
    from clbool_b200 import sizing
    n = (1 << 22) + 5
    rng = np.random.default_rng(12)
    ra = np.repeat(np.arange(64, dtype=np.uint32), 40)
    ca = rng.integers(0, 3000, ra.size).astype(np.uint32)
    a = O.coo_to_dcsr(O.Coo(64, 3000, *O.unique_pairs(*O.sort_pairs(ra, ca))))
    rb = np.repeat(np.arange(3000, dtype=np.uint32), 200)
    cbb = rng.integers(0, n, rb.size).astype(np.uint32)
    b = O.coo_to_dcsr(O.Coo(3000, n, *O.unique_pairs(*O.sort_pairs(rb, cbb))))
    s = sizing.RowSizer(controls, seed=4)
    got, st = _learned(controls, a, b, s, margin=-1000.0, slack=0.0)
    assert_dcsr_equal(got, O.spgemm(a, b), "wide learned")
    assert st["fallback_rows"] > 0 and st["spilled_rows"] == 0
