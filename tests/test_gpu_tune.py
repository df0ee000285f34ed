"""Single-matrix exhaustive autotuner: every candidate plan (format x 1D/2D
scheme x balance x sync x lanes) runs, integer results agree bit for bit
across all of them, FP results agree to rounding, and the fastest is chosen."""
import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi, tune

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["i32", "f32"])
def test_autotune_small(dtype):
    n, m, r, c, v, x = sp.synth.uniform_rows(3000, 2800, 9, 5, capi.DTYPES[dtype].np)
    A = sp.csr(dtype, n, m, *sp.synth.to_csr(n, r, c, v))
    best, recs = tune.autotune(A, x, reps=2, grids=((2, 3), (8, 8)), blocks=(4,), log=None)
    ok = [q for q in recs if q.get("status") == 0]
    kinds = {q["kind"] for q in ok}
    assert {"csr", "cooe", "bcsr", "bcoo", "dcsr", "rbdcsr", "bdcsr", "dcoo", "rbdcoo", "bdcoo"} <= kinds
    assert len(ok) == len(recs), [q for q in recs if q.get("status") != 0][:3]
    if dtype == "i32":
        assert all(q["matches_first"] for q in ok)
    else:
        assert max(q["max_rel_diff_vs_first"] for q in ok) < 1e-5
    assert best is not None and best["us"] == min(q["us"] for q in ok)
