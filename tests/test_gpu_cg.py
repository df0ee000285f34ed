"""Conjugate gradient on a plan (sparsep_cg_*): the iterative caller of the
SpMV, one iteration captured as a CUDA graph and replayed.  Checked against
SciPy's direct solve on a shifted 2D Laplacian, bit-identical across solves,
on 1D CSR and 2D-tiled plans."""
import numpy as np
import pytest
import scipy.sparse as ssp
import scipy.sparse.linalg as sla

import sparsep_b200 as sp
from sparsep_b200 import capi

pytestmark = pytest.mark.gpu


def laplacian(g, shift=0.05):
    t = ssp.diags([-1.0, 2.0, -1.0], [-1, 0, 1], shape=(g, g))
    A = (ssp.kron(ssp.eye(g), t) + ssp.kron(t, ssp.eye(g)) + shift * ssp.eye(g * g)).tocsr()
    A.sort_indices()
    return A


def host(A, dtype):
    n = A.shape[0]
    return sp.csr(dtype, n, n, A.indptr.astype(np.uint32), A.indices.astype(np.uint32),
                  A.data.astype(capi.DTYPES[dtype].np))


@pytest.mark.parametrize("dtype,tol", [("f64", 1e-10), ("f32", 1e-5)])
@pytest.mark.parametrize("layout", ["csr", "bdcsr"])
def test_cg_matches_direct_solve(dtype, tol, layout):
    import torch

    g = 80
    A = laplacian(g)
    n = g * g
    rng = np.random.default_rng(1)
    b = rng.uniform(-1, 1, n)
    want = sla.spsolve(A.tocsc(), b)
    M = host(A, dtype)
    if layout == "bdcsr":
        rp = M.arrays["rowptr"]
        rows = np.repeat(np.arange(n, dtype=np.uint32), np.diff(rp[: n + 1].astype(np.int64)))
        M = sp.convert("cooe2bdcsr", sp.cooe(dtype, n, n, rows, A.indices.astype(np.uint32),
                                              A.data.astype(capi.DTYPES[dtype].np)), 4, 4)
    plan = sp.Plan(M)
    cg = capi.CG(plan)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    db = torch.tensor(b, dtype=tdt, device="cuda")
    dx = torch.zeros(n, dtype=tdt, device="cuda")
    it, res = cg.solve(db.data_ptr(), dx.data_ptr(), max_iters=4000, rel_tol=tol, check_every=25)
    assert res <= tol and 0 < it < 4000, (it, res)
    x = dx.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(A @ x - b) / np.linalg.norm(b) <= 10 * tol
    assert np.abs(x - want).max() <= (1e-7 if dtype == "f64" else 5e-2) * np.abs(want).max()
    # the same solve again (graph replayed from the same start): bit-identical
    dx2 = torch.zeros_like(dx)
    it2, res2 = cg.solve(db.data_ptr(), dx2.data_ptr(), max_iters=4000, rel_tol=tol, check_every=25)
    assert it2 == it and res2 == res and torch.equal(dx, dx2)
    cg.free()


def test_cg_rejects_integer_and_rectangular_plans():
    A = laplacian(8)
    with pytest.raises(capi.SparsepError) as e:
        capi.CG(sp.Plan(host(A, "i32")))
    assert e.value.status == capi.ENOSYS
    R = sp.csr("f32", 3, 4, np.array([0, 1, 2, 3], np.uint32), np.array([0, 1, 3], np.uint32),
               np.ones(3, np.float32))
    with pytest.raises(capi.SparsepError) as e:
        capi.CG(sp.Plan(R))
    assert e.value.status == capi.EINVAL
