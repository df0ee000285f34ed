"""Host-buffer path with y copied back in row bands while the kernel runs.

1D CSR plans with at least 1 MB of y split their items into up to 4 row bands;
sparsep_execute_host copies each band to the host as soon as the kernel has
counted all of the band's items.  Every element type, with empty rows and long
rows (chunked items) spread over the bands, through pageable and pinned host
buffers: y identical to the device path bit for bit, and to the oracle (integer
types bit-exact, FP within the per-row gamma bound)."""
import ctypes as C

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import fp_bound_ok, hi_ref, oracle_spmv, random_x

pytestmark = pytest.mark.gpu


def case(dtype, ybytes, seed=0, ncols=65536):
    rng = np.random.default_rng(seed)
    es = np.dtype(capi.DTYPES[dtype].np).itemsize
    n = ybytes // es
    lens = rng.integers(0, 4, n)  # a quarter of the rows empty
    longs = np.linspace(n // 17, n - 1, 9).astype(np.int64)
    lens[longs] = rng.integers(5000, 20000, longs.size)  # chunked into long-row items
    rows = np.repeat(np.arange(n, dtype=np.uint32), lens)
    cols = rng.integers(0, ncols, rows.size, dtype=np.uint32)
    vals = random_x(rng, rows.size, dtype)
    x = random_x(rng, ncols, dtype)
    A = sp.csr(dtype, n, ncols, *sp.synth.to_csr(n, rows, cols, vals))
    return A, (rows, cols, vals), x


def run_pinned(plan, x, n, dtype):
    import torch

    tdt = {"i8": torch.int8, "i16": torch.int16, "i32": torch.int32, "i64": torch.int64, "f32": torch.float32,
           "f64": torch.float64}[dtype]
    hx = torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
    hy = torch.full((n,), 7, dtype=tdt).pin_memory()
    capi.check(capi.lib().sparsep_execute_host(plan.h, C.c_void_p(hx.data_ptr()), C.c_void_p(hy.data_ptr())),
               "execute_host")
    return hy.numpy().copy()


def run_device(plan, x, n):
    import torch

    xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    yd = torch.zeros(n + 64, dtype=xd.dtype, device="cuda")
    plan.run_device(xd.data_ptr(), yd.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return yd[:n].cpu().numpy()


@pytest.mark.parametrize("dtype", list(capi.DTYPES))
@pytest.mark.parametrize("o", [dict(), dict(nr_parts=2048, part_balance=capi.BAL_NNZ)])
def test_banded_host_path(dtype, o):
    A, (r, c, v), x = case(dtype, 4 << 20)
    n = int(A.s.nrows)
    plan = sp.Plan(A, sp.default_opts(**o))
    assert plan.info.y_bands == 4, plan.info.y_bands
    y_dev = run_device(plan, x, n)
    for i in range(3):  # repeated, device calls between: the band counters keep counting across calls
        assert np.array_equal(plan.run_host(x), y_dev)
        assert np.array_equal(run_pinned(plan, x, n, dtype), y_dev)
        if i == 1:
            assert np.array_equal(run_device(plan, x, n), y_dev)
    t = plan.timings()
    assert t[2] > 0 and t[3] >= 0
    plan.free()
    if dtype in ("f32", "f64"):
        y_hi, a, cnt = hi_ref(r, c, v.astype(np.float64), x.astype(np.float64), n)
        ok, err, bound = fp_bound_ok(y_dev, y_hi, a, cnt, dtype)
        assert ok, int(np.argmax(err - bound))
    else:
        assert np.array_equal(y_dev, oracle_spmv(A, x))


@pytest.mark.parametrize("ybytes,bands", [(1 << 20, 2), ((1 << 20) - 4, 0), (3 << 19, 3)])
def test_band_count(ybytes, bands):
    A, _, x = case("f32", ybytes, seed=1)
    plan = sp.Plan(A)
    assert plan.info.y_bands == bands
    assert np.array_equal(plan.run_host(x), run_device(plan, x, int(A.s.nrows)))
    plan.free()


def test_many_calls_and_changing_x():
    """60 host calls on one plan with a new x each time: every call returns its
    own product (no band copy may be satisfied by an earlier call's counts)."""
    A, (r, c, v), _ = case("i32", 4 << 20, seed=3)
    n = int(A.s.nrows)
    plan = sp.Plan(A)
    assert plan.info.y_bands == 4
    rng = np.random.default_rng(9)
    for i in range(60):
        x = random_x(rng, int(A.s.ncols), "i32")
        y = run_pinned(plan, x, n, "i32") if i % 2 else plan.run_host(x)
        if i % 10 == 0:
            assert np.array_equal(y, oracle_spmv(A, x)), i
        else:
            assert np.array_equal(y, run_device(plan, x, n)), i
    plan.free()


def test_no_bands_outside_1d_csr():
    A, (r, c, v), x = case("i32", 2 << 20, seed=2)
    n = int(A.s.nrows)
    for M, o in [(A, dict(pipeline=1)), (A, dict(sync=capi.SYNC_ATOMIC)), (sp.cooe("i32", n, int(A.s.ncols), r, c, v), {})]:
        plan = sp.Plan(M, sp.default_opts(**o))
        assert plan.info.y_bands == 0, (M.kind, o)
        assert np.array_equal(plan.run_host(x), oracle_spmv(A, x))
        plan.free()
