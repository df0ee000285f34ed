"""The allocation-free entry point (sparsep_spmv_cooe_f32_noalloc).

It serves callers that cannot allocate device memory when they multiply (a
pool or arena owning the device heap, work issued between another
component's stream operations).  This file is named to run last: it checks
the entry point through the C-ABI against the planned COO entry point on two
calls in a row -- bit for bit, since both cut the same items and add the same
carries in the same order, and within the FP32 bound the parity tests use --
for a mixed matrix, no nonzeros, one nonzero, exactly one and two full items
and trailing empty rows, and that sizes past its fixed scratch are refused.  It passes alone in a fresh process and
after the other tests."""
import ctypes as C

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import fp_bound_ok, hi_ref, random_triplets, random_x

pytestmark = pytest.mark.gpu


def _entry():
    f = capi.lib().sparsep_spmv_cooe_f32_noalloc
    f.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _case(name):
    rng = np.random.default_rng(21)
    if name == "mixed":
        nrows, ncols = 20011, 17003
        r, c, v = random_triplets(rng, nrows, ncols, 0.002, "f32", long_row=3, empty_frac=0.2)
        # a long row crossing many 4096-nonzero items exercises the carries
        extra = np.sort(rng.choice(ncols, 12000, replace=False)).astype(np.uint32)
        keep = r != 9
        r = np.concatenate([r[keep], np.full(extra.size, 9, np.uint32)])
        c = np.concatenate([c[keep], extra])
        v = np.concatenate([v[keep], rng.uniform(-1, 1, extra.size).astype(np.float32)])
    elif name == "empty":  # nnz = 0: y is cleared
        nrows, ncols = 300, 200
        r = c = np.zeros(0, np.uint32)
        v = np.zeros(0, np.float32)
    elif name == "one":  # a single nonzero, a single item
        nrows, ncols = 50, 40
        r, c, v = np.array([17], np.uint32), np.array([5], np.uint32), np.array([0.75], np.float32)
    elif name == "one_item_exact":  # exactly one full item of 4096 nonzeros
        nrows, ncols = 1000, 900
        r = np.sort(rng.integers(0, nrows, 4096)).astype(np.uint32)
        c = rng.integers(0, ncols, 4096).astype(np.uint32)
        v = rng.uniform(-1, 1, 4096).astype(np.float32)
    elif name == "two_items_exact":  # 8192 nonzeros: an item boundary inside a row
        nrows, ncols = 700, 900
        r = np.sort(rng.integers(0, nrows, 8192)).astype(np.uint32)
        c = rng.integers(0, ncols, 8192).astype(np.uint32)
        v = rng.uniform(-1, 1, 8192).astype(np.float32)
    else:  # "trailing_empty": the last nonzero's row far below nrows
        nrows, ncols = 90000, 3000
        r = np.sort(rng.integers(0, 5000, 30000)).astype(np.uint32)
        c = rng.integers(0, ncols, r.size).astype(np.uint32)
        v = rng.uniform(-1, 1, r.size).astype(np.float32)
    order = np.lexsort((c, r))
    return nrows, ncols, r[order], c[order], v[order], random_x(rng, ncols, "f32")


@pytest.mark.parametrize("name", ["mixed", "empty", "one", "one_item_exact", "two_items_exact", "trailing_empty"])
def test_noalloc_matches_planned_entry_point(name):
    import torch

    nrows, ncols, r, c, v, x = _case(name)
    A = sp.cooe("f32", nrows, ncols, r, c, v)
    y_ref = sp.Plan(A).run_host(x)  # the existing (planned, allocating) entry point

    el = A.arrays["nnzs"][: max(r.size, 1)]
    d_el = torch.from_numpy(np.ascontiguousarray(el).view(np.uint8).copy()).cuda()
    d_x = torch.from_numpy(x).cuda()
    d_y = torch.full((nrows,), float("nan"), dtype=torch.float32, device="cuda")
    f = _entry()
    stream = torch.cuda.current_stream().cuda_stream
    y_hi, a, cnt = hi_ref(r, c, v.astype(np.float64), x.astype(np.float64), nrows)
    for call in range(2):
        st = f(d_el.data_ptr(), r.size, nrows, ncols, d_x.data_ptr(), d_y.data_ptr(), stream)
        assert st == 0, capi.lib().sparsep_strerror(st)
        torch.cuda.synchronize()
        y = d_y.cpu().numpy()
        ok, err, bound = fp_bound_ok(y, y_hi, a, cnt, "f32")
        assert ok, f"call {call}: FP32 bound violated at rows {np.nonzero(err > bound)[0][:5]}"
        # the planned path cuts the same 4096-nonzero items and adds the same
        # carries in the same order: the sums are identical bit for bit
        assert y.tobytes() == y_ref.tobytes(), f"call {call}: differs from the planned entry point"
        d_y.fill_(float("nan"))


def test_noalloc_rejects_sizes_past_its_scratch():
    import torch

    d = torch.zeros(64, dtype=torch.float32, device="cuda")
    f = _entry()
    st = f(d.data_ptr(), (1 << 28) + 1, 4, 4, d.data_ptr(), d.data_ptr(), None)
    assert st == capi.ERANGE
