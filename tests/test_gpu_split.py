"""Split 1D CSR plans: the heavy rows in column stripes whose x segment is
staged in shared memory (csr_stripes.cu), the other rows on the row kernel.

Against the oracle (the reference's spmv_host restated): integers bit-exact,
FP32 / FP64 within gamma_{n_r} * sum_j |a_rj x_j| of a long-double sum.  The
cases cover stripe rows cut into pieces (a row segment longer than a chunk),
a single stripe, every row heavy, no row heavy, ragged column counts (the
stripe's ragged tail loaded without reading past x), an x pointer that is not
16-byte aligned (ragged head), and the host-buffer path with its y bands."""
import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import fp_bound_ok, hi_ref, max_rel_err, oracle_spmv, random_x

pytestmark = pytest.mark.gpu
DT = list(capi.DTYPES)
TORCH = {"i8": "int8", "i16": "int16", "i32": "int32", "i64": "int64", "f32": "float32", "f64": "float64"}


def lengths_matrix(rng, nrows, ncols, lens, dtype):
    """Sorted triplets with the given row lengths (distinct columns per row)."""
    rows, cols = [], []
    for r, k in enumerate(lens):
        k = int(min(k, ncols))
        if k == 0:
            continue
        c = np.sort(rng.choice(ncols, size=k, replace=False))
        rows.append(np.full(k, r, np.uint32))
        cols.append(c.astype(np.uint32))
    rows = np.concatenate(rows) if rows else np.zeros(0, np.uint32)
    cols = np.concatenate(cols) if cols else np.zeros(0, np.uint32)
    dt = np.dtype(capi.DTYPES[dtype].np)
    if dt.kind == "f":
        vals = rng.uniform(-1, 1, rows.size).astype(dt)
    else:
        lo, hi = (-128, 127) if dt.itemsize == 1 else (-30000, 30000)
        vals = rng.integers(lo, hi + 1, rows.size).astype(dt)
    return rows, cols, vals


def scenario(name, dtype, seed=0):
    rng = np.random.default_rng(seed)
    if name == "mixed":  # short rows, empty rows and heavy rows, ragged ncols
        nrows, ncols = 5000, 200_003
        lens = rng.integers(0, 9, nrows)
        heavy = rng.choice(nrows, 120, replace=False)
        lens[heavy] = rng.integers(64, 3000, heavy.size)
        lens[0], lens[-1] = 2500, 700  # heavy first and last rows
        thr = 64
    elif name == "pieces":  # stripe rows longer than a chunk
        nrows, ncols = 300, 140_001
        lens = rng.integers(0, 20, nrows)
        lens[7], lens[150] = 120_000, 30_000
        thr = 1000
    elif name == "one_stripe":  # x narrower than a stripe
        nrows, ncols = 4000, 5003
        lens = rng.integers(0, 40, nrows)
        thr = 8
    elif name == "all_heavy":  # no light nonzeros
        nrows, ncols = 700, 90_017
        lens = rng.integers(1, 300, nrows)
        thr = 1
    else:  # "none_heavy": a threshold above every row
        nrows, ncols = 2000, 100_000
        lens = rng.integers(0, 30, nrows)
        thr = 10_000
    r, c, v = lengths_matrix(rng, nrows, ncols, lens, dtype)
    x = random_x(rng, ncols, dtype)
    return nrows, ncols, (r, c, v), x, thr


def check_y(A, trip, x, y, label):
    if A.dtype in ("f32", "f64"):
        r, c, v = trip
        y_hi, a, cnt = hi_ref(r, c, v.astype(np.float64), x.astype(np.float64), int(A.s.nrows))
        ok, err, bound = fp_bound_ok(y, y_hi, a, cnt, A.dtype)
        assert ok, f"{label}: FP bound violated at rows {np.nonzero(err > bound)[0][:5]}"
        print(f"{label}: max |dy|/sum|ax| = {max_rel_err(y, y_hi, a):.3e}")
    else:
        y_or = oracle_spmv(A, x)
        bad = np.nonzero(y != y_or)[0]
        assert bad.size == 0, f"{label}: {bad.size} rows differ, first {bad[:5]}"


def run_device_offset(plan, x, nrows, dtype):
    """execute_device with x at an element offset of 1 (not 16-byte aligned)."""
    import torch

    tdt = getattr(torch, TORCH[dtype])
    xb = torch.zeros(x.size + 1, dtype=tdt, device="cuda")
    xb[1:] = torch.from_numpy(np.ascontiguousarray(x)).to(tdt).cuda()
    yd = torch.full((nrows,), 7, dtype=tdt, device="cuda")
    plan.run_device(xb.data_ptr() + xb.element_size(), yd.data_ptr(), 0)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("name", ["mixed", "pieces", "one_stripe", "all_heavy", "none_heavy"])
def test_split_forced(dtype, name):
    nrows, ncols, trip, x, thr = scenario(name, dtype, seed=len(name))
    r, c, v = trip
    A = sp.csr(dtype, nrows, ncols, *sp.synth.to_csr(nrows, r, c, v))
    plan = sp.Plan(A, sp.default_opts(heavy_rows=thr))
    variant = plan.info.variant.decode()
    lens = np.bincount(r.astype(np.int64), minlength=nrows)
    assert ("heavy>=" in variant) == bool((lens >= thr).any()), variant
    y_host = plan.run_host(x)
    check_y(A, trip, x, y_host, f"split {name} {dtype} {variant}")
    y_dev = run_device_offset(plan, x, nrows, dtype)
    assert y_dev.tobytes() == y_host.tobytes(), "device path with an unaligned x differs from the host path"
    y_again = plan.run_host(x)
    assert y_again.tobytes() == y_host.tobytes(), "split plan is not deterministic"
    plan.free()


@pytest.mark.parametrize("dtype", ["i8", "i32", "i64"])
def test_split_equals_unsplit_integers(dtype):
    nrows, ncols, trip, x, thr = scenario("mixed", dtype, seed=5)
    r, c, v = trip
    A = sp.csr(dtype, nrows, ncols, *sp.synth.to_csr(nrows, r, c, v))
    ys = [sp.Plan(A, sp.default_opts(heavy_rows=h)).run_host(x) for h in (thr, -1)]
    assert np.array_equal(ys[0], ys[1])
