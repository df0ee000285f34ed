"""Several right-hand sides on one plan (sparsep_opts.nrhs = k): x is
ncols x k and y nrows x k, row-major.  Every column must equal the oracle's
single-vector result (INT32 bit for bit, FP32 within the per-row gamma bound),
through the host path and the device path; the kinds without a multi-RHS
kernel answer ENOSYS."""
import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import fp_bound_ok, hi_ref, oracle_spmv, random_triplets

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["f32", "i32"])
@pytest.mark.parametrize("k", [2, 7, 32, 64, 256])
def test_plan_nrhs_every_column(dtype, k):
    import torch

    rng = np.random.default_rng(k)
    nrows, ncols = 2500, 2300
    r, c, v = random_triplets(rng, nrows, ncols, 0.004, dtype, long_row=17)
    if dtype == "i32":
        v = rng.integers(-8, 9, v.size).astype(np.int32)
    A = sp.csr(dtype, nrows, ncols, *sp.synth.to_csr(nrows, r, c, v))
    X = (rng.uniform(-1, 1, (ncols, k)) if dtype == "f32" else rng.integers(-8, 9, (ncols, k))).astype(
        capi.DTYPES[dtype].np)
    plan = sp.Plan(A, sp.default_opts(nrhs=k))
    assert plan.info.nrhs == k
    Y = plan.run_host(X)
    xd = torch.from_numpy(X).cuda()
    yd = torch.zeros((nrows, k), dtype=xd.dtype, device="cuda")
    s = torch.cuda.Stream()
    plan.run_device(xd.data_ptr(), yd.data_ptr(), s.cuda_stream)
    s.synchronize()
    assert np.array_equal(yd.cpu().numpy(), Y), "device and host paths differ"
    for j in range(k):
        xj = np.ascontiguousarray(X[:, j])
        if dtype == "i32":
            assert np.array_equal(Y[:, j], oracle_spmv(A, xj)), j
        else:
            y_hi, a, cnt = hi_ref(r, c, v.astype(np.float64), xj.astype(np.float64), nrows)
            ok, err, bound = fp_bound_ok(Y[:, j], y_hi, a, cnt, "f32")
            assert ok, (j, np.nonzero(err > bound)[0][:5])
    plan.free()


def test_plan_nrhs_unsupported_kinds():
    rng = np.random.default_rng(0)
    r, c, v = random_triplets(rng, 300, 300, 0.02, "f64")
    A = sp.csr("f64", 300, 300, *sp.synth.to_csr(300, r, c, v))
    with pytest.raises(capi.SparsepError) as e:
        sp.Plan(A, sp.default_opts(nrhs=4))
    assert e.value.status == capi.ENOSYS
    E = sp.cooe("f32", 300, 300, r, c, v.astype(np.float32))
    with pytest.raises(capi.SparsepError) as e:
        sp.Plan(E, sp.default_opts(nrhs=4))
    assert e.value.status == capi.ENOSYS
    B = sp.csr("f32", 300, 300, *sp.synth.to_csr(300, r, c, v.astype(np.float32)))
    with pytest.raises(capi.SparsepError) as e:
        sp.Plan(B, sp.default_opts(nrhs=4, nr_parts=8))
    assert e.value.status == capi.ENOSYS
