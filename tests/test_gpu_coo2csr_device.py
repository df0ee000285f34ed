"""COO -> CSR on the device (sparsep_coo2csr_device_*): the same arrays as the
host converter (the reference's counting sort: rows ascending, input order
kept inside a row), for unsorted input with duplicates and empty rows."""
import ctypes as C

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi

pytestmark = pytest.mark.gpu
TORCH = {"i8": "int8", "i16": "int16", "i32": "int32", "i64": "int64", "f32": "float32", "f64": "float64"}


def device_coo2csr(dtype, nrows, rows, cols, vals):
    import torch

    L = capi.lib()
    f = getattr(L, f"sparsep_coo2csr_device_{dtype}")
    f.argtypes = [C.c_void_p] * 3 + [C.c_uint32, C.c_uint32] + [C.c_void_p] * 4
    tdt = getattr(torch, TORCH[dtype])
    nnz = len(rows)
    dr = torch.tensor(rows.astype(np.int64), dtype=torch.int64).to(torch.int32).cuda()
    dc = torch.tensor(cols.astype(np.int64), dtype=torch.int64).to(torch.int32).cuda()
    dv = torch.from_numpy(np.ascontiguousarray(vals)).to(tdt).cuda()
    rp = torch.zeros(nrows + 1, dtype=torch.int32, device="cuda")
    co = torch.zeros(max(nnz, 1), dtype=torch.int32, device="cuda")
    vo = torch.zeros(max(nnz, 1), dtype=tdt, device="cuda")
    capi.check(f(dr.data_ptr(), dc.data_ptr(), dv.data_ptr(), nnz, nrows, rp.data_ptr(), co.data_ptr(),
                 vo.data_ptr(), None), "coo2csr_device")
    return (rp.cpu().numpy().view(np.uint32), co.cpu().numpy().view(np.uint32)[:nnz],
            vo.cpu().numpy()[:nnz])


@pytest.mark.parametrize("dtype", list(capi.DTYPES))
@pytest.mark.parametrize("nrows,nnz", [(1, 50), (37, 0), (37, 400), (5000, 60000), (70001, 300000)])
def test_device_coo2csr_equals_host(dtype, nrows, nnz):
    rng = np.random.default_rng(nrows + nnz)
    ncols = 911
    rows = rng.integers(0, nrows, nnz).astype(np.uint32)
    rows[: nnz // 5] = rows[0] if nnz else rows[: nnz // 5]  # a heavy row
    rng.shuffle(rows)
    cols = rng.integers(0, ncols, nnz).astype(np.uint32)
    cols[1::7] = cols[::7][: len(cols[1::7])]  # duplicates of (row, col) pairs are allowed
    dt = np.dtype(capi.DTYPES[dtype].np)
    vals = (rng.uniform(-1, 1, nnz) if dt.kind == "f" else rng.integers(-100, 100, nnz)).astype(dt)
    H = sp.convert("coo2csr", sp.coo(dtype, nrows, ncols, rows, cols, vals))
    rp, co, vo = device_coo2csr(dtype, nrows, rows, cols, vals)
    n = int(H.s.nnz)
    assert np.array_equal(rp, np.ctypeslib.as_array(H.s.rowptr, (nrows + 1,)))
    if n:
        assert np.array_equal(co, np.ctypeslib.as_array(H.s.colind, (n,)))
        assert np.array_equal(vo, np.ctypeslib.as_array(H.s.values, (n,)))


def test_device_coo2csr_rejects_rows_out_of_range():
    rows = np.array([0, 3, 9], dtype=np.uint32)
    with pytest.raises(capi.SparsepError) as e:
        device_coo2csr("f32", 5, rows, np.zeros(3, np.uint32), np.ones(3, np.float32))
    assert e.value.status == capi.EINVAL


@pytest.mark.parametrize("dtype", ["i32", "f32", "f64"])
def test_device_pipeline_coo_to_plan_to_spmv(dtype):
    """Device COO -> device CSR -> plan from device arrays -> SpMV: the same y
    as a plan built from the host CSR (same arrays, same kernel)."""
    import torch

    rng = np.random.default_rng(21)
    nrows, ncols, nnz = 3000, 2700, 40000
    rows = rng.integers(0, nrows, nnz).astype(np.uint32)
    cols = rng.integers(0, ncols, nnz).astype(np.uint32)
    dt = np.dtype(capi.DTYPES[dtype].np)
    vals = (rng.uniform(-1, 1, nnz) if dt.kind == "f" else rng.integers(-9, 10, nnz)).astype(dt)
    x = (rng.uniform(-1, 1, ncols) if dt.kind == "f" else rng.integers(-9, 10, ncols)).astype(dt)
    L = capi.lib()
    f = getattr(L, f"sparsep_coo2csr_device_{dtype}")
    f.argtypes = [C.c_void_p] * 3 + [C.c_uint32, C.c_uint32] + [C.c_void_p] * 4
    tdt = getattr(torch, TORCH[dtype])
    dr = torch.from_numpy(rows.view(np.int32)).cuda()
    dc = torch.from_numpy(cols.view(np.int32)).cuda()
    dv = torch.from_numpy(vals).cuda()
    rp = torch.zeros(nrows + 1, dtype=torch.int32, device="cuda")
    co = torch.zeros(nnz, dtype=torch.int32, device="cuda")
    vo = torch.zeros(nnz, dtype=tdt, device="cuda")
    capi.check(f(dr.data_ptr(), dc.data_ptr(), dv.data_ptr(), nnz, nrows, rp.data_ptr(), co.data_ptr(),
                 vo.data_ptr(), None))
    P = capi.Plan.from_device_csr(dtype, nrows, ncols, nnz, rp.data_ptr(), co.data_ptr(), vo.data_ptr())
    del rp, co, vo  # the plan holds its own copies
    torch.cuda.synchronize()
    y = P.run_host(x)
    H = sp.Plan(sp.convert("coo2csr", sp.coo(dtype, nrows, ncols, rows, cols, vals))).run_host(x)
    assert np.array_equal(y, H)


def test_plan_from_device_csr_rejects_bad_columns():
    import torch

    rp = torch.tensor([0, 1, 2], dtype=torch.int32, device="cuda")
    co = torch.tensor([0, 7], dtype=torch.int32, device="cuda")
    vo = torch.ones(2, device="cuda")
    with pytest.raises(capi.SparsepError) as e:
        capi.Plan.from_device_csr("f32", 2, 5, 2, rp.data_ptr(), co.data_ptr(), vo.data_ptr())
    assert e.value.status == capi.EINVAL
