"""CSR -> BCSR on the device (sparsep_bcsr_layout_device + sparsep_csr2bcsr_device_*):
the same browptr / bcolind / bval / nnz_per_block as the host converter (the
reference's csr2bcsr + sortBCSRMatrix + countNNZperBlockBCSRMatrix), for rows
with unsorted and duplicate columns, explicit zeros, empty rows and shapes
that are not multiples of the block; a plan from the device arrays
(sparsep_plan_bcsr_device_*) computes what a plan from the host BCSR does."""
import time

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import random_x, struct_arrays

pytestmark = pytest.mark.gpu
TORCH = {"i8": "int8", "i16": "int16", "i32": "int32", "i64": "int64", "f32": "float32", "f64": "float64"}


def host_csr(dtype, nrows, ncols, rng, per_row=6, long_rows=0):
    lens = rng.integers(0, 2 * per_row, nrows)
    lens[rng.random(nrows) < 0.2] = 0
    if long_rows:
        lens[rng.choice(nrows, long_rows, replace=False)] = rng.integers(500, 3000, long_rows)
    rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)
    nnz = int(rowptr[-1])
    colind = rng.integers(0, ncols, nnz).astype(np.uint32)  # unsorted, duplicates possible
    dup = rng.random(nnz) < 0.05  # some explicit repeats of the previous entry's column
    dup[:1] = False
    colind[dup] = colind[np.nonzero(dup)[0] - 1]
    vals = random_x(rng, nnz, dtype)
    vals[rng.random(nnz) < 0.1] = 0  # explicit zeros
    return sp.csr(dtype, nrows, ncols, rowptr, colind, vals), rowptr, colind, vals


def device_bcsr(dtype, nrows, ncols, rowptr, colind, vals, rb, cb):
    import torch

    tdt = getattr(torch, TORCH[dtype])
    drp = torch.from_numpy(rowptr.view(np.int32)).cuda()
    dci = torch.from_numpy(colind.view(np.int32).copy() if colind.size else np.zeros(1, np.int32)).cuda()
    dv = torch.from_numpy(np.ascontiguousarray(vals) if vals.size else np.zeros(1, vals.dtype)).to(tdt).cuda()
    L = capi.BcsrLayout(drp.data_ptr(), dci.data_ptr(), nrows, ncols, int(rowptr[-1]), rb, cb)
    nb = L.nblocks
    bp = torch.full((L.nbr + 1,), -1, dtype=torch.int32, device="cuda")
    bc = torch.full((max(nb, 1),), -1, dtype=torch.int32, device="cuda")
    bv = torch.full((max(nb, 1) * rb * cb,), 7, dtype=tdt, device="cuda")
    npb = torch.full((max(nb, 1),), -1, dtype=torch.int32, device="cuda")
    L.fill(dtype, dv.data_ptr(), bp.data_ptr(), bc.data_ptr(), bv.data_ptr(), npb.data_ptr())
    L.free()
    return nb, bp, bc, bv, npb


def compare(dtype, A, nb, bp, bc, bv, npb, rb, cb):
    H = sp.convert("csr2bcsr", A, rb, cb)
    h = struct_arrays("bcsr", dtype, H.s)
    assert nb == int(H.s.num_blocks)
    assert np.array_equal(bp.cpu().numpy().view(np.uint32), h["browptr"])
    assert np.array_equal(bc.cpu().numpy().view(np.uint32)[:nb], h["bcolind"])
    assert bv.cpu().numpy()[: nb * rb * cb].tobytes() == h["bval"].tobytes()
    assert np.array_equal(npb.cpu().numpy().view(np.uint32)[:nb], h["nnz_per_block"])
    return H


@pytest.mark.parametrize("dtype", list(capi.DTYPES))
@pytest.mark.parametrize("rb,cb", [(4, 4), (8, 8), (2, 3), (16, 16), (1, 1)])
@pytest.mark.parametrize("nrows,ncols", [(1, 1), (37, 53), (5003, 4001)])
def test_device_csr2bcsr_equals_host(dtype, rb, cb, nrows, ncols):
    rng = np.random.default_rng(nrows * 31 + rb * 7 + cb)
    A, rowptr, colind, vals = host_csr(dtype, nrows, ncols, rng, long_rows=2 if nrows > 100 else 0)
    nb, bp, bc, bv, npb = device_bcsr(dtype, nrows, ncols, rowptr, colind, vals, rb, cb)
    compare(dtype, A, nb, bp, bc, bv, npb, rb, cb)


def test_empty_matrix():
    rowptr = np.zeros(10, np.uint32)
    nb, bp, *_ = device_bcsr("f32", 9, 9, rowptr, np.zeros(0, np.uint32), np.zeros(0, np.float32), 4, 4)
    assert nb == 0 and np.array_equal(bp.cpu().numpy(), np.zeros(4, np.int32))


@pytest.mark.parametrize("bad", ["column", "rowptr_end", "rowptr_order"])
def test_invalid_input_is_einval(bad):
    import torch

    rowptr = np.array([0, 2, 3, 5], np.uint32)
    colind = np.array([0, 1, 2, 3, 4], np.uint32)
    if bad == "column":
        colind[3] = 5  # ncols = 5
    elif bad == "rowptr_end":
        rowptr[-1] = 4
    else:
        rowptr[1:3] = [3, 2]
    drp = torch.from_numpy(rowptr.view(np.int32)).cuda()
    dci = torch.from_numpy(colind.view(np.int32)).cuda()
    with pytest.raises(capi.SparsepError) as e:
        capi.BcsrLayout(drp.data_ptr(), dci.data_ptr(), 3, 5, 5, 2, 2)
    assert e.value.status == capi.EINVAL


@pytest.mark.parametrize("dtype", ["i8", "i32", "f32", "f64"])
@pytest.mark.parametrize("o", [dict(), dict(nr_parts=64, part_balance=capi.BAL_NNZ),
                               dict(nr_parts=64, part_balance=capi.BAL_BLOCK)])
def test_plan_from_device_bcsr(dtype, o):
    import torch

    rng = np.random.default_rng(5)
    nrows, ncols, rb, cb = 20011, 19997, 4, 4
    A, rowptr, colind, vals = host_csr(dtype, nrows, ncols, rng, long_rows=3)
    nb, bp, bc, bv, npb = device_bcsr(dtype, nrows, ncols, rowptr, colind, vals, rb, cb)
    H = compare(dtype, A, nb, bp, bc, bv, npb, rb, cb)
    x = random_x(rng, ncols, dtype)
    want = sp.Plan(H, sp.default_opts(**o)).run_host(x)
    p = capi.Plan.from_device_bcsr(dtype, nrows, ncols, rb, cb, nb, int(rowptr[-1]), bp.data_ptr(), bc.data_ptr(),
                                   bv.data_ptr(), npb.data_ptr(), sp.default_opts(**o))
    del bp, bc, bv, npb
    torch.cuda.synchronize()
    assert np.array_equal(p.run_host(x), want)
    p.free()


def test_banded_fullsize_timing():
    """The 2,097,152-row block-banded matrix (FP32, 4 x 4): the device converter
    against the host one, arrays equal."""
    import torch

    B = sp.synth.block_banded(rb=4, cb=4, dtype=np.float32)
    r, c, v = sp.synth.bcsr_triplets(B)
    keep = v != 0
    r, c, v = r[keep], c[keep], v[keep]
    o = np.lexsort((c, r))
    n = B["nrows"]
    rowptr, colind, vals = sp.synth.to_csr(n, r[o], c[o], v[o])
    A = sp.csr("f32", n, B["ncols"], rowptr, colind, vals)
    t0 = time.perf_counter()
    H = sp.convert("csr2bcsr", A, 4, 4)
    host_s = time.perf_counter() - t0
    drp = torch.from_numpy(rowptr.view(np.int32)).cuda()
    dci = torch.from_numpy(colind.view(np.int32)).cuda()
    dv = torch.from_numpy(vals).cuda()
    ts = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L = capi.BcsrLayout(drp.data_ptr(), dci.data_ptr(), n, B["ncols"], int(rowptr[-1]), 4, 4)
        nb = L.nblocks
        bp = torch.empty(L.nbr + 1, dtype=torch.int32, device="cuda")
        bc = torch.empty(nb, dtype=torch.int32, device="cuda")
        bv = torch.empty(nb * 16, dtype=torch.float32, device="cuda")
        npb = torch.empty(nb, dtype=torch.int32, device="cuda")
        L.fill("f32", dv.data_ptr(), bp.data_ptr(), bc.data_ptr(), bv.data_ptr(), npb.data_ptr())
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
        L.free()
    h = struct_arrays("bcsr", "f32", H.s)
    assert nb == int(H.s.num_blocks)
    assert np.array_equal(bc.cpu().numpy().view(np.uint32), h["bcolind"])
    assert bv.cpu().numpy().tobytes() == h["bval"].tobytes()
    assert np.array_equal(npb.cpu().numpy().view(np.uint32), h["nnz_per_block"])
    assert np.array_equal(bp.cpu().numpy().view(np.uint32), h["browptr"])
    print(f"\ncsr2bcsr 4x4, {int(rowptr[-1])} nnz, {nb} blocks: host {host_s:.2f} s, device "
          f"{min(ts) * 1e3:.1f} ms (layout + fill + output allocation)")
