"""Failure paths, made to happen on purpose without faulting the GPU.

- A bounded device wait that runs out: with sparsep_test_wait_fault on, the
  kernels with a staging wait add, after their own copies have landed, one
  wait that nothing completes.  The call must report SPARSEP_ETIMEDOUT, and
  the next call with the switch off must succeed with the oracle's result.
- A device allocation that fails: sparsep_test_fail_alloc(n) fails the n-th
  allocation; every n up to the last allocation of the object must give
  SPARSEP_ENOMEM and leave the library holding no more device memory than
  before (plans, 2D plans, the batch, CG, the device converters).  The
  reference's answer to both is an abort (DPU_ASSERT)."""
import ctypes as C

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import oracle_spmv, random_triplets, random_x

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def switches_off():
    L = capi.lib()
    L.sparsep_test_wait_fault(0)
    L.sparsep_test_fail_alloc(0)
    yield
    L.sparsep_test_wait_fault(0)
    L.sparsep_test_fail_alloc(0)


def staged_2d(dtype="i32"):
    rng = np.random.default_rng(7)
    nrows, ncols = 3000, 2500
    r, c, v = random_triplets(rng, nrows, ncols, 0.004, dtype, long_row=5)
    x = random_x(rng, ncols, dtype)
    D = sp.convert("cooe2rbdcsr", sp.cooe(dtype, nrows, ncols, r, c, v), 4, 8)
    return D, x


def test_plan_staging_wait_runs_out_and_recovers():
    D, x = staged_2d()
    plan = sp.Plan(D, sp.default_opts(stage_x=1))
    assert plan.info.stage_x == 1
    L = capi.lib()
    L.sparsep_test_wait_fault(1)
    with pytest.raises(capi.SparsepError) as e:
        plan.run_host(x)
    assert e.value.status == capi.ETIMEDOUT
    L.sparsep_test_wait_fault(0)
    y = plan.run_host(x)
    assert np.array_equal(y, oracle_spmv(D, x))
    plan.free()


def test_batch_wait_runs_out_and_recovers():
    rng = np.random.default_rng(3)
    mats, data = [], []
    for m in range(6):
        n = int(rng.integers(500, 3000))
        rp, ci, vv = sp.synth.batch_matrix(rng, n, ("uniform", "zipf", "banded")[m % 3], np.int32)
        k = int(rng.integers(1, 9))
        x = rng.integers(-8, 9, (n, k)).astype(np.int32)
        mats.append(sp.csr("i32", n, n, rp, ci, vv))
        data.append((n, k, x))
    b = capi.Batch("i32", mats, [d[1] for d in data])
    for m, (n, k, x) in enumerate(data):
        b.set_x(m, x)
    L = capi.lib()
    for run in (b.execute, b.execute_per_matrix):
        L.sparsep_test_wait_fault(1)
        with pytest.raises(capi.SparsepError) as e:
            run()  # no stream: synchronous, returns the batch's status
        assert e.value.status == capi.ETIMEDOUT
        L.sparsep_test_wait_fault(0)
        run()
        for m, (n, k, x) in enumerate(data):
            y = b.get_y(m)
            for j in range(k):
                assert np.array_equal(y[:, j], oracle_spmv(mats[m], np.ascontiguousarray(x[:, j])))
    b.free()


def fails_cleanly(make, free, limit=80, holds=True):
    """make() under a failure of the n-th allocation for n = 1, 2, ... until it
    succeeds: each failure is ENOMEM and leaves the live count unchanged
    (holds: the object made keeps device memory until free)."""
    L = capi.lib()
    base = L.sparsep_test_live_allocations()
    for n in range(1, limit):
        L.sparsep_test_fail_alloc(n)
        try:
            obj = make()
        except capi.SparsepError as e:
            assert e.status == capi.ENOMEM, (n, e)
            assert L.sparsep_test_live_allocations() == base, f"allocation {n} failed and left memory held"
            continue
        L.sparsep_test_fail_alloc(0)
        assert (L.sparsep_test_live_allocations() > base) == holds
        free(obj)
        assert L.sparsep_test_live_allocations() == base
        return n - 1  # allocations the object makes
    raise AssertionError("object still failing after the limit")


def test_alloc_failures_plans():
    rng = np.random.default_rng(1)
    nrows, ncols = 4000, 3500
    r, c, v = random_triplets(rng, nrows, ncols, 0.003, "f32", long_row=9)
    A = sp.csr("f32", nrows, ncols, *sp.synth.to_csr(nrows, r, c, v))
    E = sp.cooe("f32", nrows, ncols, r, c, v)
    D = sp.convert("cooe2bdcsr", E, 4, 4)
    B = sp.convert("csr2bcsr", A, 4, 4)
    for M, o in ((A, {}), (A, dict(heavy_rows=8)), (E, {}), (D, {}), (B, {}), (A, dict(pipeline=1))):
        n = fails_cleanly(lambda: sp.Plan(M, sp.default_opts(**o)), lambda p: p.free())
        assert n >= 5, (M.kind, o, n)


def test_alloc_failures_batch_cg_converters():
    rng = np.random.default_rng(2)
    mats, ks = [], []
    for m in range(4):
        n = int(rng.integers(300, 2000))
        rp, ci, vv = sp.synth.batch_matrix(rng, n, "uniform", np.float32)
        mats.append(sp.csr("f32", n, n, rp, ci, vv))
        ks.append(m + 1)
    fails_cleanly(lambda: capi.Batch("f32", mats, ks), lambda b: b.free())

    # CG on an SPD plan (a shifted 1D Laplacian)
    n = 3000
    trip = [(i, j, 4.0 if i == j else -1.0) for i in range(n) for j in (i - 1, i, i + 1) if 0 <= j < n]
    rows, cols, vals = (np.array(t) for t in zip(*trip))
    S = sp.csr("f64", n, n, *sp.synth.to_csr(n, rows.astype(np.uint32), cols.astype(np.uint32), vals))
    plan = sp.Plan(S)
    fails_cleanly(lambda: capi.CG(plan), lambda c: c.free())
    plan.free()

    # device COO -> CSR and the device BCSR layout (their scratch)
    import torch

    nnz, nr = 20000, 3000
    rr = rng.integers(0, nr, nnz).astype(np.int32)
    cc = rng.integers(0, 2000, nnz).astype(np.int32)
    vv = rng.uniform(-1, 1, nnz).astype(np.float32)
    dr, dc, dv = (torch.from_numpy(a).cuda() for a in (rr, cc, vv))
    rp = torch.zeros(nr + 1, dtype=torch.int32, device="cuda")
    co = torch.zeros(nnz, dtype=torch.int32, device="cuda")
    vo = torch.zeros(nnz, dtype=torch.float32, device="cuda")
    L = capi.lib()
    f = L.sparsep_coo2csr_device_f32
    f.argtypes = [C.c_void_p] * 3 + [C.c_uint32, C.c_uint32] + [C.c_void_p] * 4

    def c2c():
        capi.check(f(dr.data_ptr(), dc.data_ptr(), dv.data_ptr(), nnz, nr, rp.data_ptr(), co.data_ptr(),
                     vo.data_ptr(), None), "coo2csr_device")
        return None

    fails_cleanly(c2c, lambda _: None, holds=False)
    fails_cleanly(lambda: capi.BcsrLayout(rp.data_ptr(), co.data_ptr(), nr, 2000, nnz, 4, 4),
                  lambda lay: lay.free())
