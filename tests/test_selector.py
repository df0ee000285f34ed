"""Learned variant selector: features, the FP64 oracle of the network, the
CUDA forward / loss-gradient / Adam kernels checked against it, training,
the trained model's gain over the untuned default, and the batch using it."""
import sys
from pathlib import Path

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi, selector
from helpers import fp_bound_ok, hi_ref, oracle_spmv

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import mlp_oracle as mo  # noqa: E402

K = capi.NVARIANTS


def features_np(n, ncols, rp, ci, k):
    """NumPy restatement of the 16 features (the C++ pass is the product)."""
    rp = rp.astype(np.int64)
    ci = ci.astype(np.int64)
    lens = np.diff(rp).astype(np.float64)
    nnz = int(rp[-1])
    mean = nnz / max(n, 1)
    rows = np.repeat(np.arange(n), np.diff(rp))
    d = np.abs(ci - rows).astype(np.float64)
    same = np.ones(nnz, dtype=bool)
    same[rp[:-1][lens > 0]] = False  # first nonzero of each row
    gaps = np.abs(np.diff(ci, prepend=0))[same]

    def blocks(b):
        return np.unique((rows // b) * ((ncols + b - 1) // b) + ci // b).size

    f = [np.log2(n + 1), np.log2(nnz + 1), np.log2(k), k % 4 == 0, k % 2 == 0, np.log2(mean + 1),
         np.sqrt(((lens - mean) ** 2).sum() / n) / mean if mean else 0, np.log2(lens.max() + 1),
         lens[lens > 4096].sum() / max(nnz, 1), np.mean(lens < 4), d.sum() / max(nnz, 1) / ncols,
         np.mean(d <= 64), nnz / (16 * blocks(4)), nnz / (64 * blocks(8)), np.log2(ncols * k * 4.0),
         np.log2((gaps.mean() if gaps.size else 0) + 1)]
    return np.array(f, dtype=np.float64)


@pytest.mark.parametrize("fam", sp.synth.SELECTOR_FAMILIES)
def test_features_match_restatement(fam):
    rng = np.random.default_rng(4)
    n, rp, ci = sp.synth.selector_matrix(rng, fam, 3000, 12.0)
    if fam == "zipf":  # one row past the long-row threshold
        extra = np.arange(5000, dtype=np.uint32) % n
        ci = np.concatenate([np.sort(np.unique(extra)), ci[rp[1]:]]).astype(np.uint32)
        rp = rp.astype(np.int64)
        rp[1:] += np.unique(extra).size - (rp[1] - rp[0])
        rp = rp.astype(np.uint32)
    for k in (1, 6, 32):
        got = capi.features(n, n, rp, ci, k)
        want = features_np(n, n, rp, ci, k)
        np.testing.assert_allclose(got, want, rtol=2e-5, atol=1e-6)


def test_oracle_gradient_is_the_derivative():
    """Pins the FP64 oracle: its gradient against central differences."""
    rng = np.random.default_rng(0)
    _, NP = mo.layout(K)
    w = rng.normal(0, 0.2, NP)
    x = rng.normal(0, 1, (40, 16))
    t = np.where(rng.random((40, K)) < 0.6, rng.uniform(1, 5, (40, K)), 0.0)
    t[3] = 0.0  # a sample with no applicable variant
    for alpha, lam, tau in ((1.0, 0.0, 0.05), (0.5, 0.3, 0.1)):
        _, g = mo.loss_grad(w, x, t, 0.3, alpha, lam, tau)
        eps = 1e-6
        for i in rng.choice(NP, 60, replace=False):
            wp, wm = w.copy(), w.copy()
            wp[i] += eps
            wm[i] -= eps
            fd = (mo.loss_grad(wp, x, t, 0.3, alpha, lam, tau)[0] - mo.loss_grad(wm, x, t, 0.3, alpha, lam, tau)[0]) / (
                2 * eps)
            assert abs(fd - g[i]) <= 1e-7 * max(1.0, np.abs(g).max()), (i, alpha, lam)


def test_bf16_rounding_oracle():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-5], dtype=np.float32)
    b = mo.bf16_bits(v)
    assert b.tolist()[:3] == [0x3F80, 0x3F80, 0x3F81]  # ties to even, above-half up
    assert np.all(np.abs(mo.bf16_to_f64(b) - v) <= np.abs(v) * 2 ** -8)


def _dev_problem(n, seed):
    import torch

    rng = np.random.default_rng(seed)
    w = selector.init_weights(seed) + rng.normal(0, 0.05, capi.lib().sparsep_mlp_nparams()).astype(np.float32)
    wb = mo.bf16_bits(w)
    x = rng.normal(0, 1, (n, 16)).astype(np.float32)
    t = np.where(rng.random((n, K)) < 0.5, rng.uniform(1, 50, (n, K)), 0.0).astype(np.float32)
    t[::17] = 0.0
    dev = torch.device("cuda")
    return (w, wb, x, t, torch.tensor(wb.view(np.int16), device=dev), torch.tensor(x, device=dev),
            torch.tensor(t, device=dev))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 63, 200, 1000])
@pytest.mark.parametrize("alpha,lam,tau", [(1.0, 0.0, 0.05), (0.5, 0.02, 0.05), (0.0, 0.5, 0.2)])
def test_gpu_forward_and_gradient_match_oracle(n, alpha, lam, tau):
    """The CUDA forward logits and loss / gradient (FP32 accumulate) against
    the FP64 oracle evaluated at the same BF16 weights."""
    import torch

    L = capi.lib()
    capi._batch_sigs(L)
    w, wb, x, t, dwb, dx, dt = _dev_problem(n, n)
    wq = mo.bf16_to_f64(wb)
    NP = wq.size
    logits = torch.zeros(n * K, device="cuda")
    capi.check(L.sparsep_mlp_forward(dwb.data_ptr(), dx.data_ptr(), n, logits.data_ptr(), None))
    _, _, z = mo.forward(wq, x.astype(np.float64), K)
    np.testing.assert_allclose(logits.cpu().numpy().reshape(n, K), z, rtol=1e-4, atol=1e-4 * np.abs(z).max())
    wscale = 0.05
    g = torch.zeros(NP, device="cuda")
    loss = torch.zeros(1, device="cuda")
    scratch = torch.zeros(int(L.sparsep_mlp_scratch_floats(n)), device="cuda")
    capi.check(L.sparsep_mlp_loss_grad(dwb.data_ptr(), dx.data_ptr(), dt.data_ptr(), n, wscale, alpha, lam, tau,
                                       g.data_ptr(), loss.data_ptr(), scratch.data_ptr(), None))
    lo, go = mo.loss_grad(wq, x, t, wscale, alpha, lam, tau)
    gg = g.cpu().numpy().astype(np.float64)
    assert abs(loss.item() - lo) <= 1e-4 * max(1.0, abs(lo))
    assert np.abs(gg - go).max() <= 1e-4 * max(np.abs(go).max(), 1e-12), np.abs(gg - go).max()
    # bit-identical on a second run (fixed-order reductions)
    g2 = torch.zeros_like(g)
    capi.check(L.sparsep_mlp_loss_grad(dwb.data_ptr(), dx.data_ptr(), dt.data_ptr(), n, wscale, alpha, lam, tau,
                                       g2.data_ptr(), loss.data_ptr(), scratch.data_ptr(), None))
    assert torch.equal(g, g2)


@pytest.mark.gpu
def test_gpu_adam_step_matches_formula():
    import torch

    L = capi.lib()
    capi._batch_sigs(L)
    rng = np.random.default_rng(1)
    NP = L.sparsep_mlp_nparams()
    w0 = rng.normal(0, 1, NP).astype(np.float32)
    g0 = rng.normal(0, 1, NP).astype(np.float32)
    w = torch.tensor(w0, device="cuda")
    wb = torch.zeros(NP, dtype=torch.int16, device="cuda")
    g = torch.tensor(g0, device="cuda")
    m = torch.zeros(NP, device="cuda")
    v = torch.zeros(NP, device="cuda")
    capi.check(L.sparsep_mlp_adam(w.data_ptr(), wb.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), 1, 1e-2, 0.9,
                                  0.999, 1e-8, 1e-3, None))
    mm = 0.1 * g0.astype(np.float64)
    vv = 0.001 * g0.astype(np.float64) ** 2
    want = w0 - 1e-2 * ((mm / 0.1) / (np.sqrt(vv / 0.001) + 1e-8) + 1e-3 * w0)
    np.testing.assert_allclose(w.cpu().numpy(), want, rtol=1e-5, atol=1e-6)
    assert np.array_equal(wb.cpu().numpy().view(np.uint16), mo.bf16_bits(w.cpu().numpy()))


@pytest.mark.gpu
def test_gpu_training_reduces_regret():
    """A few hundred full-batch steps on a synthetic timing table whose best
    variant is a function of the features: the loss falls and the picks beat
    a uniform choice."""
    rng = np.random.default_rng(7)
    n = 600
    feats = rng.normal(0, 1, (n, 16)).astype(np.float32)
    best = (np.floor((feats[:, 0] > 0) * 2 + (feats[:, 1] > 0)) * 5).astype(int)  # 0, 5, 10, 15
    times = rng.uniform(2.0, 3.0, (n, K)).astype(np.float32)
    times[np.arange(n), best] = 1.0
    times[:, 30:] = 0.0  # not applicable
    model = selector.train(feats, times, steps=400, lr=1e-2, seed=0, log=None)
    h = model["history"]
    assert h[-1, 1] < 0.3 * h[0, 1], h
    sel = selector.selector(model)
    pick = selector.picks(sel.scores(feats), times)
    assert np.mean(pick == best) > 0.9


def small_batch(dtype, nmats=24, seed=9):
    rng = np.random.default_rng(seed)
    out = []
    for m in range(nmats):
        n, rp, ci = sp.synth.selector_matrix(rng, sp.synth.SELECTOR_FAMILIES[m % 5], int(rng.integers(300, 3000)),
                                             float(rng.integers(2, 40)))
        vv = (rng.uniform(-1, 1, ci.size) if dtype == "f32" else rng.integers(-8, 9, ci.size)).astype(
            capi.DTYPES[dtype].np)
        k = int(rng.integers(1, 33))
        x = (rng.uniform(-1, 1, (n, k)) if dtype == "f32" else rng.integers(-8, 9, (n, k))).astype(
            capi.DTYPES[dtype].np)
        out.append((n, rp, ci, vv, k, x))
    return out


def check_batch(b, mats, data, dtype):
    for m, (n, rp, ci, vv, k, x) in enumerate(data):
        y = b.get_y(m)
        rows = np.repeat(np.arange(n, dtype=np.uint32), np.diff(rp.astype(np.int64)))
        for j in range(k):
            yo = oracle_spmv(mats[m], np.ascontiguousarray(x[:, j]))
            if dtype == "i32":
                assert np.array_equal(y[:, j], yo), (m, j)
            else:
                y_hi, a, cnt = hi_ref(rows, ci, vv.astype(np.float64), x[:, j].astype(np.float64), n)
                ok, err, bound = fp_bound_ok(y[:, j], y_hi, a, cnt, "f32")
                assert ok, (m, j)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f32", "i32"])
def test_batch_select_results_and_fallback(dtype):
    """The learned schedule changes no result; min_confidence above 1 sends
    every matrix to the exhaustive autotuner."""
    data = small_batch(dtype)
    mats = [sp.csr(dtype, n, n, rp, ci, vv) for (n, rp, ci, vv, k, x) in data]
    b = capi.Batch(dtype, mats, [d[4] for d in data])
    for m, d in enumerate(data):
        b.set_x(m, d[5])
    feats = b.features()
    for m, (n, rp, ci, vv, k, x) in enumerate(data):
        np.testing.assert_array_equal(feats[m], capi.features(n, n, rp, ci, k))
    model = selector.load() if selector.MODEL.exists() else selector.train(
        feats, np.ones((len(data), K), dtype=np.float32), steps=5, log=None)
    sel = selector.selector(model)
    ch, fb = b.select(sel, min_confidence=0.0)
    assert (fb == 0).all() and (ch >= 0).all()
    cand = capi.batch_candidates()
    assert all(cand[c].applies(d[4]) and b.applies(m, cand[c]) for m, (c, d) in enumerate(zip(ch, data)))
    b.execute()
    check_batch(b, mats, data, dtype)
    ch2, fb2 = b.select(sel, min_confidence=1.01, reps=1)
    assert (fb2 == 1).all()
    b.execute()
    check_batch(b, mats, data, dtype)


HELDOUT = selector.DATA / "heldout.npz"


@pytest.mark.gpu
@pytest.mark.skipif(not (selector.MODEL.exists() and HELDOUT.exists()), reason="no trained model committed")
def test_trained_model_gain_on_heldout():
    """On held-out matrices (timed on a B200 by the autotuner), the trained
    network's picks run within 10% of the exhaustive best in total and faster
    than the untuned default variant: what the network gains over the method
    without it."""
    model = selector.load()
    h = np.load(HELDOUT)
    res = selector.evaluate(selector.selector(model).scores(h["feats"]), h["times"], h["meta"][:, 3])
    assert res["regret_total"] <= 0.10, res
    assert res["speedup_vs_default"] > 1.0, res
    assert res["regret_total"] < res["default_regret_total"], res
    # the confidence is informative: falling back below 0.3 lowers the regret
    z = selector.selector(model).scores(h["feats"])
    t = h["times"]
    zz = np.where(t > 0, z, -np.inf)
    p = np.exp(zz - zz.max(axis=1, keepdims=True))
    conf = (p / p.sum(axis=1, keepdims=True)).max(axis=1)
    best = np.where(t > 0, t, np.inf).min(axis=1)
    pick = t[np.arange(len(t)), selector.picks(z, t)]
    fb = conf < 0.3
    assert 0.0 < fb.mean() < 0.5
    assert np.where(fb, best, pick).sum() / best.sum() - 1 < res["regret_total"]


HELDOUT_WIDE = selector.DATA / "heldout_wide.npz"


@pytest.mark.gpu
@pytest.mark.skipif(not (selector.MODEL.exists() and HELDOUT_WIDE.exists()), reason="no trained model committed")
def test_trained_model_gain_on_wider_matrices():
    """Held-out matrices of the wide range (rows 8k-2.1M, 2-128 nonzeros
    per row, up to 10 M nonzeros; 2,000 of the 22,000 training matrices come
    from that range, the rest from 1k-262k rows and 2-64 per row), timed on a
    B200 by the autotuner: the network's picks run within 10% of the
    exhaustive best in total and beat the default variant."""
    h = np.load(HELDOUT_WIDE)
    assert h["meta"][:, 1].max() > 1_000_000 and h["meta"][:, 2].max() > 4_000_000
    res = selector.evaluate(selector.selector(selector.load()).scores(h["feats"]), h["times"], h["meta"][:, 3])
    assert res["regret_total"] <= 0.10, res
    assert res["speedup_vs_default"] > 1.0, res
