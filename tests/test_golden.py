"""Golden vectors: outputs of the reference's own converters + spmv_host
(tests/golden/golden.npz, made by tests/golden/make_golden.py from the
reference compiled in oracle/_ref).  The oracle replays each case through
this library's converters and must match bit for bit (CPU); the GPU path must
match bit for bit for integers and within 2 gamma_n sum|a x| for FP (the
reference sums each row sequentially in the element type, the GPU in another
order)."""
from pathlib import Path

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import fp_bound_ok, hi_ref, oracle_spmv

G = np.load(Path(__file__).resolve().parent / "golden" / "golden.npz")
CASES = sorted({k.rsplit("/", 2)[0] + "/" + k.rsplit("/", 2)[1] for k in G.files})
NROWS, NCOLS = 57, 61
BLOCK_CONV = {"dbcsr": ("cooe2dcsr", "dcsr2dbcsr"), "dbcoo": ("cooe2dcsr", "dcsr2dbcoo"),
              "rbdbcsr": ("cooe2rbdcsr", "rbdcsr2rbdbcsr"), "rbdbcoo": ("cooe2rbdcsr", "rbdcsr2rbdbcoo"),
              "bdbcsr": ("cooe2bdcsr", "bdcsr2bdbcsr"), "bdbcoo": ("cooe2bdcsr", "bdcsr2bdbcoo")}


def build(case):
    """The case's struct through this library's converters (the same chain the
    reference's host program runs)."""
    name, dtype = case.split("/")
    g = {f: G[f"{case}/{f}"] for f in ("rows", "cols", "vals", "x", "y", "params")}
    prm = [int(v) for v in g["params"]]
    r, c, v = g["rows"], g["cols"], g["vals"]
    if name == "csr":
        return sp.convert("coo2csr", sp.coo(dtype, NROWS, NCOLS, r, c, v)), g
    if name.startswith("bcsr") or name.startswith("bcoo"):
        B = sp.convert("csr2bcsr", sp.convert("coo2csr", sp.coo(dtype, NROWS, NCOLS, r, c, v)), *prm)
        return (B if name.startswith("bcsr") else sp.convert("bcsr2bcoo", B)), g
    A = sp.cooe(dtype, NROWS, NCOLS, r, c, v)
    if name == "cooe":
        sp.sort_cooe(A)
        return A, g
    if name in BLOCK_CONV:
        c1, c2 = BLOCK_CONV[name]
        return sp.convert(c2, sp.convert(c1, A, prm[0], prm[1]), prm[2], prm[3]), g
    return sp.convert(f"cooe2{name}", A, *prm), g


def test_golden_cases_present():
    assert len(CASES) == 17 * 6


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_golden(case):
    A, g = build(case)
    assert np.array_equal(oracle_spmv(A, g["x"]), g["y"]), case


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_gpu_matches_reference_golden(case):
    A, g = build(case)
    y = sp.spmv(A, g["x"])
    dtype = case.split("/")[1]
    if np.dtype(capi.DTYPES[dtype].np).kind != "f":
        assert np.array_equal(y, g["y"]), case
    else:
        y_hi, a, cnt = hi_ref(g["rows"], g["cols"], g["vals"].astype(np.float64), g["x"].astype(np.float64), NROWS)
        ok, err, bound = fp_bound_ok(y, g["y"].astype(np.float64), a, cnt, dtype, factor=2.0)
        assert ok, (case, float((err / np.maximum(bound, 1e-300)).max()))
