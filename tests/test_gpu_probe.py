"""The gather-floor probe reads x at the given indices: its per-thread sums
add up to the sum of x over the index stream."""
import ctypes as C

import numpy as np
import pytest

from sparsep_b200 import capi

pytestmark = pytest.mark.gpu


def test_probe_gather_sums_x_at_indices():
    import torch

    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, 10000).astype(np.float32)
    idx = rng.integers(0, x.size, 300001).astype(np.uint32)
    L = capi.lib()
    L.sparsep_probe_gather_f32.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    di = torch.from_numpy(idx.view(np.int32)).cuda()
    dx = torch.from_numpy(x).cuda()
    out = torch.zeros(37 * 512, device="cuda")
    capi.check(L.sparsep_probe_gather_f32(di.data_ptr(), idx.size, dx.data_ptr(), out.data_ptr(), 37, None))
    torch.cuda.synchronize()
    want = float(x[idx].astype(np.float64).sum())
    assert abs(float(out.double().sum()) - want) <= 1e-3 * np.abs(x[idx]).sum() ** 0.5 + 1e-2
