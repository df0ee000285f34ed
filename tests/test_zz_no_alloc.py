"""The allocation-free entry point (sparsep_spmv_cooe_f32_noalloc).

It serves callers that cannot allocate device memory when they multiply (a
pool or arena owning the device heap, work issued between another
component's stream operations).  This file is named to run last: it checks
the entry point through the C-ABI against the planned COO entry point on two
calls in a row, within the FP32 bound the parity tests use, and that sizes
past its fixed scratch are refused.  It passes alone in a fresh process and
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


def test_noalloc_matches_planned_entry_point():
    import torch

    rng = np.random.default_rng(21)
    nrows, ncols = 20011, 17003
    r, c, v = random_triplets(rng, nrows, ncols, 0.002, "f32", long_row=3, empty_frac=0.2)
    # a long row crossing many 4096-nonzero items exercises the carries
    extra = np.sort(rng.choice(ncols, 12000, replace=False)).astype(np.uint32)
    keep = r != 9
    r = np.concatenate([r[keep], np.full(extra.size, 9, np.uint32)])
    c = np.concatenate([c[keep], extra])
    v = np.concatenate([v[keep], rng.uniform(-1, 1, extra.size).astype(np.float32)])
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    x = random_x(rng, ncols, "f32")
    A = sp.cooe("f32", nrows, ncols, r, c, v)
    y_ref = sp.Plan(A).run_host(x)  # the existing (planned, allocating) entry point

    el = A.arrays["nnzs"][: r.size]
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
        # same item split as the planned path: the same sums in the same order
        assert np.allclose(y, y_ref, rtol=0, atol=float(np.max(bound)) * 2)
        d_y.fill_(float("nan"))


def test_noalloc_rejects_sizes_past_its_scratch():
    import torch

    d = torch.zeros(64, dtype=torch.float32, device="cuda")
    f = _entry()
    st = f(d.data_ptr(), (1 << 28) + 1, 4, 4, d.data_ptr(), d.data_ptr(), None)
    assert st == capi.ERANGE
