"""GPU parity: every format / scheme / option through the C-ABI against the oracle.

Integer element types must match the oracle (the reference's spmv_host
restated) bit for bit.  FP32 / FP64 must satisfy, per row,
    |y_gpu - y_exact| <= gamma_{n_r} * sum_j |a_rj x_j|,   gamma_n = n u / (1 - n u)
(u = 2^-24 / 2^-53), with y_exact from a long-double compensated sum; the
max error against that FP64-or-better oracle is printed for every case."""
import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import fp_bound_ok, hi_ref, max_rel_err, oracle_spmv, random_triplets, random_x

pytestmark = pytest.mark.gpu
DT = list(capi.DTYPES)


def check(A: capi.HostMatrix, trip, x, opts=None, label=""):
    plan = sp.Plan(A, opts)
    y = plan.run_host(x)
    y_or = oracle_spmv(A, x)
    if A.dtype in ("f32", "f64"):
        r, c, v = trip
        y_hi, a, cnt = hi_ref(r, c, v.astype(np.float64), x.astype(np.float64), int(A.s.nrows))
        ok, err, bound = fp_bound_ok(y, y_hi, a, cnt, A.dtype)
        assert ok, f"{label}: FP bound violated at rows {np.nonzero(err > bound)[0][:5]}"
        ok2, _, _ = fp_bound_ok(y_or, y_hi, a, cnt, A.dtype)
        assert ok2
        print(f"{label} {plan.info.variant.decode()}: max |dy|/sum|ax| = {max_rel_err(y, y_hi, a):.3e}")
    else:
        bad = np.nonzero(y != y_or)[0]
        assert bad.size == 0, f"{label}: {bad.size} rows differ, first {bad[:5]} gpu={y[bad[:5]]} ref={y_or[bad[:5]]}"
    plan.free()
    return y


def make(dtype, seed=0, nrows=3001, ncols=2903, density=0.004, long_row=11, empty_frac=0.15):
    rng = np.random.default_rng(seed)
    r, c, v = random_triplets(rng, nrows, ncols, density, dtype, long_row=long_row, empty_frac=empty_frac)
    x = random_x(rng, ncols, dtype)
    return nrows, ncols, (r, c, v), x


OPTS_1D = [dict(), dict(sync=capi.SYNC_ATOMIC), dict(nr_parts=7, part_balance=capi.BAL_ROW),
           dict(nr_parts=64, part_balance=capi.BAL_NNZ, worker_balance=capi.BAL_NNZ),
           dict(nr_parts=33, part_balance=capi.BAL_NNZ_ELEM), dict(lanes=1), dict(lanes=32, nr_workers=4),
           dict(pipeline=1), dict(pipeline=1, item_nnz=2048), dict(item_nnz=2048), dict(nr_workers=16),
           dict(nr_workers=4)]


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("oi", range(len(OPTS_1D)))
def test_csr_1d(dtype, oi):
    nrows, ncols, trip, x = make(dtype, seed=1)
    r, c, v = trip
    A = sp.csr(dtype, nrows, ncols, *sp.synth.to_csr(nrows, r, c, v))
    check(A, trip, x, sp.default_opts(**OPTS_1D[oi]), f"csr {dtype} {OPTS_1D[oi]}")


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("oi", range(len(OPTS_1D)))
def test_coo_1d(dtype, oi):
    nrows, ncols, trip, x = make(dtype, seed=2)
    r, c, v = trip
    A = sp.cooe(dtype, nrows, ncols, r, c, v)
    check(A, trip, x, sp.default_opts(**OPTS_1D[oi]), f"cooe {dtype} {OPTS_1D[oi]}")


@pytest.mark.parametrize("dtype", ["i32", "f32"])
def test_coo_soa_unsorted(dtype):
    nrows, ncols, trip, x = make(dtype, seed=3)
    r, c, v = trip
    p = np.random.default_rng(0).permutation(r.size)
    A = sp.coo(dtype, nrows, ncols, r[p], c[p], v[p])
    check(A, trip, x, None, f"coo-soa {dtype}")


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("rb,cb", [(4, 4), (8, 8), (2, 2), (3, 5)])
@pytest.mark.parametrize("oi", [0, 1, 2, 3, 4])
def test_bcsr_bcoo_1d(dtype, rb, cb, oi):
    opts = [dict(), dict(sync=capi.SYNC_ATOMIC), dict(nr_parts=9, part_balance=capi.BAL_BLOCK),
            dict(nr_parts=21, part_balance=capi.BAL_NNZ), dict(lanes=2)][oi]
    nrows, ncols, trip, x = make(dtype, seed=4, nrows=1203, ncols=1101, density=0.01)
    r, c, v = trip
    Acsr = sp.csr(dtype, nrows, ncols, *sp.synth.to_csr(nrows, r, c, v))
    B = sp.convert("csr2bcsr", Acsr, rb, cb)
    check(B, trip, x, sp.default_opts(**opts), f"bcsr{rb}x{cb} {dtype} {opts}")
    O = sp.convert("bcsr2bcoo", B)
    o2 = dict(opts)
    if o2.get("part_balance") == capi.BAL_NNZ:
        o2["part_balance"] = capi.BAL_NNZ_ELEM
    check(O, trip, x, sp.default_opts(**o2), f"bcoo{rb}x{cb} {dtype} {o2}")


TWO_D = ["cooe2dcsr", "cooe2rbdcsr", "cooe2bdcsr", "cooe2dcoo", "cooe2rbdcoo", "cooe2bdcoo"]


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("conv", TWO_D)
@pytest.mark.parametrize("hv", [(4, 3), (16, 8), (1, 1)])
@pytest.mark.parametrize("oi", [0, 1, 2, 3])
def test_2d(dtype, conv, hv, oi):
    opts = [dict(), dict(sync=capi.SYNC_ATOMIC), dict(stage_x=0), dict(nr_parts=1)][oi]
    nrows, ncols, trip, x = make(dtype, seed=5)
    r, c, v = trip
    C = sp.cooe(dtype, nrows, ncols, r, c, v)
    D = sp.convert(conv, C, *hv)
    check(D, trip, x, sp.default_opts(**opts), f"{conv} {hv} {dtype} {opts}")


TWO_D_BLOCK = [("cooe2dcsr", "dcsr2dbcsr"), ("cooe2dcsr", "dcsr2dbcoo"), ("cooe2rbdcsr", "rbdcsr2rbdbcsr"),
               ("cooe2rbdcsr", "rbdcsr2rbdbcoo"), ("cooe2bdcsr", "bdcsr2bdbcsr"), ("cooe2bdcsr", "bdcsr2bdbcoo")]


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("c1,c2", TWO_D_BLOCK)
@pytest.mark.parametrize("hv,blk", [((4, 3), (4, 4)), ((3, 5), (8, 8)), ((2, 2), (3, 2))])
@pytest.mark.parametrize("oi", [0, 1])
def test_2d_block(dtype, c1, c2, hv, blk, oi):
    opts = [dict(), dict(sync=capi.SYNC_ATOMIC)][oi]
    nrows, ncols, trip, x = make(dtype, seed=6, nrows=1201, ncols=1307, density=0.01)
    r, c, v = trip
    C = sp.cooe(dtype, nrows, ncols, r, c, v)
    D = sp.convert(c2, sp.convert(c1, C, *hv), *blk)
    check(D, trip, x, sp.default_opts(**opts), f"{c2} {hv} {blk} {dtype} {opts}")


# ---------------------------------------------------------------- edge cases
@pytest.mark.parametrize("dtype", ["i8", "i32", "f32", "f64"])
@pytest.mark.parametrize("kind", ["csr", "cooe", "bcsr", "bcoo"])
def test_single_long_row(dtype, kind):
    """One row holding every nonzero: CSR long-row chunks, COO/BCOO carries."""
    rng = np.random.default_rng(7)
    nrows, ncols = 64, 100_003
    c = np.sort(rng.choice(ncols, 60_000, replace=False)).astype(np.uint32)
    r = np.full(c.size, 17, dtype=np.uint32)
    v = random_x(rng, c.size, dtype)
    x = random_x(rng, ncols, dtype)
    trip = (r, c, v)
    if kind == "csr":
        A = sp.csr(dtype, nrows, ncols, *sp.synth.to_csr(nrows, r, c, v))
    elif kind == "cooe":
        A = sp.cooe(dtype, nrows, ncols, r, c, v)
    else:
        A = sp.convert("csr2bcsr", sp.csr(dtype, nrows, ncols, *sp.synth.to_csr(nrows, r, c, v)), 4, 4)
        if kind == "bcoo":
            A = sp.convert("bcsr2bcoo", A)
    for o in (dict(), dict(sync=capi.SYNC_ATOMIC), dict(pipeline=1), dict(pipeline=1, item_nnz=2048)):
        check(A, trip, x, sp.default_opts(**o), f"long-row {kind} {dtype} {o}")


@pytest.mark.parametrize("kind", ["csr", "cooe", "bcsr", "bcoo", "dcsr", "bdcoo"])
def test_empty_matrix(kind):
    nrows, ncols = 40, 33
    r = np.zeros(0, np.uint32)
    c = np.zeros(0, np.uint32)
    v = np.zeros(0, np.float32)
    x = np.ones(ncols, np.float32)
    if kind == "csr":
        A = sp.csr("f32", nrows, ncols, *sp.synth.to_csr(nrows, r, c, v))
    elif kind in ("bcsr", "bcoo"):
        A = sp.convert("csr2bcsr", sp.csr("f32", nrows, ncols, *sp.synth.to_csr(nrows, r, c, v)), 4, 4)
        if kind == "bcoo":
            A = sp.convert("bcsr2bcoo", A)
    else:
        A = sp.cooe("f32", nrows, ncols, r, c, v)
        if kind != "cooe":
            A = sp.convert("cooe2" + kind, A, 3, 2)
    y = sp.Plan(A).run_host(x)
    assert y.shape == (nrows,) and not y.any()


@pytest.mark.parametrize("dtype", ["i8", "i16"])
def test_narrow_int_wraparound(dtype):
    """Sums overflow int8/int16 many times over; results wrap exactly."""
    nrows, ncols = 500, 700
    rng = np.random.default_rng(8)
    r, c, v = random_triplets(rng, nrows, ncols, 0.2, dtype, empty_frac=0.0)
    info = np.iinfo(capi.DTYPES[dtype].np)
    v = np.full(r.size, info.max, dtype=capi.DTYPES[dtype].np)
    x = np.full(ncols, info.max, dtype=capi.DTYPES[dtype].np)
    for kind in ("csr", "cooe"):
        A = sp.csr(dtype, nrows, ncols, *sp.synth.to_csr(nrows, r, c, v)) if kind == "csr" else \
            sp.cooe(dtype, nrows, ncols, r, c, v)
        for o in (dict(), dict(sync=capi.SYNC_ATOMIC)):
            check(A, (r, c, v), x, sp.default_opts(**o), f"wrap {kind} {dtype} {o}")


def test_one_shot_and_device_paths():
    """sparsep_spmv_* (one-shot, host buffers) and execute_device (torch buffers) agree."""
    import torch
    nrows, ncols, trip, x = make("f32", seed=9)
    r, c, v = trip
    A = sp.csr("f32", nrows, ncols, *sp.synth.to_csr(nrows, r, c, v))
    y1 = sp.spmv(A, x)
    plan = sp.Plan(A)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty(nrows, dtype=torch.float32, device="cuda")
    plan.run_device(xd.data_ptr(), yd.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(y1, yd.cpu().numpy())  # same plan layout -> same order -> identical
    t = plan.timings()
    assert len(t) == 5 and t[0] > 0


def test_concurrent_plans_from_host_threads():
    """Plans built and executed from four host threads at once (x-staged 2D
    tiles and the TMA pipeline set kernel attributes on first use): every
    result equals the oracle."""
    import concurrent.futures as cf

    def one(i):
        dtype = ("i32", "f32", "i64", "f64")[i % 4]
        nrows, ncols, trip, x = make(dtype, seed=40 + i, nrows=2500 + 100 * i, ncols=2300, density=0.005)
        r, c, v = trip
        A = sp.cooe(dtype, nrows, ncols, r, c, v)
        out = []
        for M, o in ((sp.convert("cooe2dcsr", A, 4, 3), {}),
                     (sp.csr(dtype, nrows, ncols, *sp.synth.to_csr(nrows, r, c, v)), dict(pipeline=1))):
            out.append((dtype, sp.Plan(M, sp.default_opts(**o)).run_host(x), oracle_spmv(M, x), trip, x, nrows))
        return out

    with cf.ThreadPoolExecutor(4) as ex:
        results = [r for rs in ex.map(one, range(8)) for r in rs]
    for dtype, y, yo, (r, c, v), x, nrows in results:
        if np.dtype(capi.DTYPES[dtype].np).kind != "f":
            assert np.array_equal(y, yo)
        else:
            y_hi, a, cnt = hi_ref(r, c, v.astype(np.float64), x.astype(np.float64), nrows)
            assert fp_bound_ok(y, y_hi, a, cnt, dtype)[0]
