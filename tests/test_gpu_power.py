"""Power iteration on a plan (sparsep_power_*): one iteration -- SpMV, Rayleigh
quotient, norm, normalisation -- captured as a CUDA graph and replayed.  The
dominant eigenvalue against SciPy's ARPACK and against the same iteration in
FP64 numpy; the eigenvector residual; bit-identical reruns; 1D CSR and
2D-tiled plans."""
import numpy as np
import pytest
import scipy.sparse as ssp
import scipy.sparse.linalg as sla

import sparsep_b200 as sp
from sparsep_b200 import capi

pytestmark = pytest.mark.gpu


def matrix(n=6000, seed=0):
    """Symmetric, dominant eigenvalue near 10 with a gap of about 4."""
    rng = np.random.default_rng(seed)
    d = rng.uniform(0.0, 5.0, n)
    d[n // 3] = 10.0
    R = ssp.random(n, n, density=4.0 / n, random_state=seed, format="csr")
    A = (ssp.diags(d) + 0.05 * (R + R.T)).tocsr()
    A.sort_indices()
    return A


def host(A, dtype, layout):
    n = A.shape[0]
    T = capi.DTYPES[dtype].np
    M = sp.csr(dtype, n, n, A.indptr.astype(np.uint32), A.indices.astype(np.uint32), A.data.astype(T))
    if layout == "csr":
        return M
    rows = np.repeat(np.arange(n, dtype=np.uint32), np.diff(A.indptr))
    return sp.convert("cooe2rbdcsr", sp.cooe(dtype, n, n, rows, A.indices.astype(np.uint32), A.data.astype(T)), 4, 4)


def numpy_power(A, x0, iters):
    p = x0 / np.linalg.norm(x0)
    lam = 0.0
    for _ in range(iters):
        q = A @ p
        lam = p @ q
        p = q / np.linalg.norm(q)
    return lam, p


@pytest.mark.parametrize("dtype,tol", [("f64", 1e-12), ("f32", 1e-6)])
@pytest.mark.parametrize("layout", ["csr", "rbdcsr"])
def test_power_dominant_eigenvalue(dtype, tol, layout):
    import torch

    A = matrix()
    n = A.shape[0]
    want = float(sla.eigsh(A, k=1, which="LA", return_eigenvectors=False)[0])
    plan = sp.Plan(host(A, dtype, layout))
    pw = capi.PowerIteration(plan)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    x0 = np.random.default_rng(1).uniform(-1, 1, n)
    dx = torch.tensor(x0, dtype=tdt, device="cuda")
    lam, it = pw.run(dx.data_ptr(), max_iters=2000, rel_tol=tol, check_every=5)
    assert 0 < it < 2000, it
    assert abs(lam - want) <= (1e-9 if dtype == "f64" else 1e-4) * abs(want), (lam, want)
    v = dx.cpu().numpy().astype(np.float64)
    assert abs(np.linalg.norm(v) - 1.0) < (1e-12 if dtype == "f64" else 1e-5)
    assert np.linalg.norm(A @ v - lam * v) <= (1e-5 if dtype == "f64" else 5e-3) * abs(lam)
    # the same iteration count in FP64 numpy from the same start
    lam_np, _ = numpy_power(A, x0, it)
    assert abs(lam - lam_np) <= (1e-12 if dtype == "f64" else 1e-5) * abs(lam_np)
    # rerun from the same start: bit-identical
    dx2 = torch.tensor(x0, dtype=tdt, device="cuda")
    lam2, it2 = pw.run(dx2.data_ptr(), max_iters=2000, rel_tol=tol, check_every=5)
    assert it2 == it and lam2 == lam and torch.equal(dx, dx2)
    pw.free()
    plan.free()


def test_power_zero_start_and_integer_plan():
    import torch

    A = matrix(500)
    plan = sp.Plan(host(A, "f64", "csr"))
    pw = capi.PowerIteration(plan)
    dx = torch.zeros(500, dtype=torch.float64, device="cuda")
    lam, it = pw.run(dx.data_ptr(), max_iters=50, check_every=5)
    assert lam == 0.0 and it == 5  # A p = 0: stops at the first read
    pw.free()
    plan.free()
    n = 100
    M = sp.csr("i32", n, n, np.arange(n + 1, dtype=np.uint32), np.arange(n, dtype=np.uint32), np.ones(n, np.int32))
    ip = sp.Plan(M)
    with pytest.raises(capi.SparsepError) as e:
        capi.PowerIteration(ip)
    assert e.value.status == capi.ENOSYS
    ip.free()
