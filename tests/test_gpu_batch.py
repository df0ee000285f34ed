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
            if b.applies(m, v):
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
        if not all(b.applies(m, v) for m in range(len(data))):
            continue
        for m in range(len(data)):
            b.set_variant(m, v)
        b.commit()
        b.execute()
        check_batch(b, mats, data, dtype)


def long_row_batch(dtype, seed=11):
    """Matrices whose longest rows exceed one 5120-nonzero chunk (5121 up to
    50,000 nonzeros, so 2..10 chunk items per row) beside ordinary rows, with
    k = 1, 3, 16 and 33 right-hand sides."""
    rng = np.random.default_rng(seed)
    out = []
    for m, (k, long_lens) in enumerate(((1, (5121, 9000)), (3, (10240, 50000)), (16, (15361,)), (33, (5121, 20000)))):
        n = 60_000
        lens = rng.integers(1, 40, n)
        rows = rng.choice(n, len(long_lens), replace=False)
        lens[rows] = long_lens
        rp = np.zeros(n + 1, dtype=np.uint32)
        np.cumsum(lens, out=rp[1:])
        ci = np.concatenate([np.sort(rng.choice(n, int(l), replace=False)) for l in lens]).astype(np.uint32)
        np_t = capi.DTYPES[dtype].np
        vv = (rng.uniform(-1, 1, ci.size) if dtype == "f32" else rng.integers(-8, 9, ci.size)).astype(np_t)
        x = (rng.uniform(-1, 1, (n, k)) if dtype == "f32" else rng.integers(-8, 9, (n, k))).astype(np_t)
        out.append((n, rp, ci, vv, k, x))
    return out


@pytest.mark.parametrize("dtype", ["f32", "i32"])
def test_batch_long_rows(dtype):
    """Rows longer than a chunk run as one item per chunk on many CTAs; the
    last chunk to arrive sums the partial rows.  Results stay right over
    repeated graph launches, per-matrix launches, every applicable candidate
    and the autotuner's timing runs -- the rows' arrival counters return to
    zero after every launch."""
    data = long_row_batch(dtype)
    mats = [sp.csr(dtype, n, n, rp, ci, vv) for (n, rp, ci, vv, k, x) in data]
    b = sp.capi.Batch(dtype, mats, [d[4] for d in data])
    for m, d in enumerate(data):
        b.set_x(m, d[5])
    assert b.item_kinds()[1] == sum(-(-int(l) // 5120) for d in data for l in np.diff(d[1].astype(np.int64))
                                    if l > 5120)
    for _ in range(3):
        b.execute()
        check_batch(b, mats, data, dtype)
    b.execute_per_matrix()
    check_batch(b, mats, data, dtype)
    for v in sp.capi.batch_candidates()[::5]:
        for m, d in enumerate(data):
            if b.applies(m, v):
                b.set_variant(m, v)
        b.commit()
        b.execute()
        check_batch(b, mats, data, dtype)
    b.autotune(reps=1)
    b.execute()
    check_batch(b, mats, data, dtype)
    b.status()


@pytest.mark.parametrize("dtype", ["f32", "i32"])
def test_batch_window_items(dtype):
    """Banded matrices under the window variants: x tiles staged in shared
    memory (including spans just inside and beyond what the arena holds, so
    that window and ordinary items alternate), every column against the
    oracle."""
    rng = np.random.default_rng(12)
    data = []
    for m, (k, bw) in enumerate(((4, 8), (7, 64), (16, 200), (32, 90), (12, 1500))):
        n = int(rng.integers(5_000, 20_000))
        r = np.arange(n)
        lo = np.maximum(0, r - bw)
        hi = np.minimum(n, r + bw + 1)
        lens = np.minimum(hi - lo, rng.integers(4, 65, n))
        rp, ci = sp.synth.stratified_cols(rng, lens, lo, hi)
        np_t = capi.DTYPES[dtype].np
        vv = (rng.uniform(-1, 1, ci.size) if dtype == "f32" else rng.integers(-8, 9, ci.size)).astype(np_t)
        x = (rng.uniform(-1, 1, (n, k)) if dtype == "f32" else rng.integers(-8, 9, (n, k))).astype(np_t)
        data.append((n, rp, ci, vv, k, x))
    mats = [sp.csr(dtype, n, n, rp, ci, vv) for (n, rp, ci, vv, k, x) in data]
    b = sp.capi.Batch(dtype, mats, [d[4] for d in data])
    for m, d in enumerate(data):
        b.set_x(m, d[5])
    for v in sp.capi.batch_candidates():
        if not v.mode & 2 or not any(b.applies(m, v) for m in range(len(data))):
            continue
        for m, d in enumerate(data):
            b.set_variant(m, v if b.applies(m, v) else sp.capi.BatchVariant(1, 8, 0, 4))
        b.commit()
        nwin, _ = b.item_kinds()
        assert nwin > 0
        b.execute()
        check_batch(b, mats, data, dtype)


def block_matrix(rng, n, dtype, fill=0.8, half_bw=6):
    """Square matrix of 4 x 4 blocks around the diagonal (block columns within
    half_bw of the block row, each block's entries present with probability
    fill), n not a multiple of 4: the last block row and column are partial."""
    nb = (n + 3) // 4
    rows, cols = [], []
    for br in range(nb):
        for bc in range(max(0, br - half_bw), min(nb, br + half_bw + 1)):
            if rng.random() < 0.5:
                continue
            mask = rng.random((4, 4)) < fill
            rr, cc = np.nonzero(mask)
            rr, cc = rr + 4 * br, cc + 4 * bc
            ok = (rr < n) & (cc < n)
            rows.append(rr[ok])
            cols.append(cc[ok])
    r = np.concatenate(rows).astype(np.int64)
    c = np.concatenate(cols).astype(np.int64)
    key = np.unique(r * n + c)
    r, c = key // n, key % n
    rp = np.zeros(n + 1, dtype=np.uint32)
    np.cumsum(np.bincount(r, minlength=n), out=rp[1:])
    np_t = capi.DTYPES[dtype].np
    vv = (rng.uniform(-1, 1, c.size) if dtype == "f32" else rng.integers(-8, 9, c.size)).astype(np_t)
    return rp, c.astype(np.uint32), vv


@pytest.mark.parametrize("dtype", ["f32", "i32"])
def test_batch_block_items(dtype):
    """Block-structured matrices get a 4 x 4 BCSR copy and run under every
    block variant (mode 4) that fits their k, partial last blocks included;
    a scattered matrix gets none.  Every column against the oracle, then the
    autotuner over all candidates."""
    rng = np.random.default_rng(13)
    data = []
    for n, k in ((4001, 4), (2002, 16), (3003, 7), (1501, 32), (999, 12)):
        rp, ci, vv = block_matrix(rng, n, dtype)
        x = (rng.uniform(-1, 1, (n, k)) if dtype == "f32" else rng.integers(-8, 9, (n, k))).astype(
            capi.DTYPES[dtype].np)
        data.append((n, rp, ci, vv, k, x))
    n = 3000
    rp, ci, vv = sp.synth.batch_matrix(rng, n, "uniform", capi.DTYPES[dtype].np)
    data.append((n, rp, ci, vv, 8, rng.integers(-8, 9, (n, 8)).astype(capi.DTYPES[dtype].np)))
    mats = [sp.csr(dtype, n, n, rp, ci, vv) for (n, rp, ci, vv, k, x) in data]
    b = sp.capi.Batch(dtype, mats, [d[4] for d in data])
    for m, d in enumerate(data):
        b.set_x(m, d[5])
    blocks = [v for v in sp.capi.batch_candidates() if v.mode == 4]
    assert len(blocks) == 6
    assert not any(b.applies(len(data) - 1, v) for v in blocks)  # no copy for the scattered matrix
    for m in range(len(data) - 1):
        assert any(b.applies(m, v) for v in blocks), m
    ran = 0
    for v in blocks:
        use = [m for m in range(len(data)) if b.applies(m, v)]
        if not use:
            continue
        for m in range(len(data)):
            b.set_variant(m, v if m in use else sp.capi.BatchVariant(1, 8, 0, 4 if data[m][4] % 4 == 0 else 1))
        b.commit()
        b.execute()
        check_batch(b, mats, data, dtype)
        ran += len(use)
    assert ran >= 10
    b.autotune(reps=1)
    b.execute()
    check_batch(b, mats, data, dtype)
    b.status()
