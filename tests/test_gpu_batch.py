"""Batched multi-RHS SpMV: the persistent graph launch, the per-matrix
launches and every autotuner candidate against the oracle, column by column
(integers bit-exact, FP32 within the per-row gamma bound)."""
import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import fp_bound_ok, hi_ref, oracle_spmv

pytestmark = pytest.mark.gpu


def small_batch(dtype, nmats=30, seed=5):
    rng = np.random.default_rng(seed)
    kinds = ("uniform", "zipf", "banded")
    ks = [1, 2, 3, 4, 5, 8, 16, 32, 7, 33]
    out = []
    for m in range(nmats):
        n = int(rng.integers(200, 3000))
        rp, ci, vv = sp.synth.batch_matrix(rng, n, kinds[m % 3], capi.DTYPES[dtype].np)
        k = ks[m % len(ks)]
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
                assert ok, (m, j, np.nonzero(err > bound)[0][:5])


@pytest.mark.parametrize("dtype", ["f32", "i32"])
def test_batch_graph_and_per_matrix(dtype):
    data = small_batch(dtype)
    mats = [sp.csr(dtype, n, n, rp, ci, vv) for (n, rp, ci, vv, k, x) in data]
    b = sp.capi.Batch(dtype, mats, [d[4] for d in data])
    for m, d in enumerate(data):
        b.set_x(m, d[5])
    b.execute()
    check_batch(b, mats, data, dtype)
    b.execute()  # graph replay
    check_batch(b, mats, data, dtype)
    b.execute_per_matrix()
    check_batch(b, mats, data, dtype)
    t, ch = b.autotune(reps=2)
    assert (ch >= 0).all() and (t.max(axis=1) > 0).all()
    b.execute()
    check_batch(b, mats, data, dtype)


@pytest.mark.parametrize("dtype", ["f32", "i32"])
def test_batch_every_candidate(dtype):
    data = small_batch(dtype, nmats=10, seed=6)
    mats = [sp.csr(dtype, n, n, rp, ci, vv) for (n, rp, ci, vv, k, x) in data]
    b = sp.capi.Batch(dtype, mats, [d[4] for d in data])
    for m, d in enumerate(data):
        b.set_x(m, d[5])
    for v in sp.capi.batch_candidates():
        applied = False
        for m, d in enumerate(data):
            k = d[4]
            if v.applies(k):
                b.set_variant(m, v)
                applied = True
        if not applied:
            continue
        b.commit()
        b.execute()
        check_batch(b, mats, data, dtype)


def test_batch_rejects_bad_variants():
    data = small_batch("f32", nmats=2)
    mats = [sp.csr("f32", n, n, rp, ci, vv) for (n, rp, ci, vv, k, x) in data]
    b = sp.capi.Batch("f32", mats, [d[4] for d in data])
    bad = sp.capi.BatchVariant(1, 3, 2048, 0)  # lanes not a power of two
    with pytest.raises(sp.SparsepError):
        b.set_variant(0, bad)


@pytest.mark.parametrize("dtype", ["f32", "i32"])
def test_batch_wide_rhs(dtype):
    """k = 64, 128, 256 right-hand sides (SpMM-like), default and applicable
    candidate variants, every column against the oracle."""
    rng = np.random.default_rng(8)
    data = []
    for m, k in enumerate((64, 128, 256)):
        n = int(rng.integers(500, 1500))
        rp, ci, vv = sp.synth.batch_matrix(rng, n, ("uniform", "zipf", "banded")[m], capi.DTYPES[dtype].np)
        x = (rng.uniform(-1, 1, (n, k)) if dtype == "f32" else rng.integers(-8, 9, (n, k))).astype(
            capi.DTYPES[dtype].np)
        data.append((n, rp, ci, vv, k, x))
    mats = [sp.csr(dtype, n, n, rp, ci, vv) for (n, rp, ci, vv, k, x) in data]
    b = sp.capi.Batch(dtype, mats, [d[4] for d in data])
    for m, d in enumerate(data):
        b.set_x(m, d[5])
    b.execute()
    check_batch(b, mats, data, dtype)
    for v in sp.capi.batch_candidates():
        if not all(v.applies(d[4]) for d in data):
            continue
        for m in range(len(data)):
            b.set_variant(m, v)
        b.commit()
        b.execute()
        check_batch(b, mats, data, dtype)
