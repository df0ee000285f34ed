"""Parity at the benchmark configurations' full sizes (GPU against the oracle,
which handles these sizes in well under a second per SpMV).

  uniform8  4096 x 4096, 8 distinct uniform columns per row, INT32, CSR 1D
            nnz-balanced: bit-exact.
  zipf      1,048,576^2, 16,777,216 nonzeros, Zipf(2.0) row lengths, FP32 and
            FP64; CSR and COO, 1D row- and nnz-balanced, 2D equal (D, 256
            tiles), row-band (RBD, 1024 tiles) and variable (BD, 4096 tiles):
            every row within gamma_{n_i} sum_j |a_ij x_j| of a long-double
            compensated sum.
  banded    2,097,152 rows, block-banded, BCSR and BCOO 4x4 and 8x8, block-
            and nnz-balanced, INT8 / INT16 / INT64 bit-exact, FP32 within the
            per-row bound against an FP64 evaluation of the same blocks.
"""
import functools

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import fp_bound_ok, hi_ref, oracle_spmv

pytestmark = pytest.mark.gpu
PARTS = 2048  # parts as the reference's 2048-DPU runs (one part = one CTA)


def opts(**kw):
    return sp.default_opts(**kw)


# ---------------------------------------------------------------------------
# uniform8, INT32
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("o", [dict(), dict(nr_parts=64, part_balance=capi.BAL_NNZ),
                               dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ, worker_balance=capi.BAL_NNZ)])
def test_uniform8_int32_csr_bit_exact(o):
    n, m, r, c, v, x = sp.synth.uniform_rows(4096, 4096, 8, 0, np.int32)
    A = sp.csr("i32", n, m, *sp.synth.to_csr(n, r, c, v))
    assert np.array_equal(sp.spmv(A, x, opts(**o)), oracle_spmv(A, x))


# ---------------------------------------------------------------------------
# zipf, FP32 / FP64
# ---------------------------------------------------------------------------
@functools.lru_cache(maxsize=2)
def zipf(dtype):
    npdt = capi.DTYPES[dtype].np
    n, m, r, c, v, x = sp.synth.zipf_rows(seed=1, dtype=npdt)
    y_hi, a, cnt = hi_ref(r, c, v.astype(np.float64), x.astype(np.float64), n)
    return n, m, r, c, v, x, (y_hi, a, cnt)


ZIPF = [("csr", "", (), dict()),
        ("csr", "", (), dict(nr_parts=PARTS, part_balance=capi.BAL_ROW)),
        ("csr", "", (), dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ, worker_balance=capi.BAL_NNZ)),
        ("cooe", "", (), dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ_ELEM)),
        ("cooe", "", (), dict(sync=capi.SYNC_ATOMIC)),
        ("cooe", "", (), dict(nr_parts=PARTS, part_balance=capi.BAL_ROW)),
        ("cooe", "cooe2dcsr", (16, 16), dict()),
        ("cooe", "cooe2rbdcsr", (32, 32), dict()),
        ("cooe", "cooe2bdcsr", (64, 64), dict()),
        ("cooe", "cooe2bdcsr", (64, 64), dict(sync=capi.SYNC_ATOMIC)),
        ("cooe", "cooe2dcoo", (16, 16), dict()),
        ("cooe", "cooe2bdcoo", (64, 64), dict())]


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("case", range(len(ZIPF)))
def test_zipf_fullsize_within_bound(dtype, case):
    base, conv, args, o = ZIPF[case]
    n, m, r, c, v, x, (y_hi, a, cnt) = zipf(dtype)
    if base == "csr":
        A = sp.csr(dtype, n, m, *sp.synth.to_csr(n, r, c, v))
    else:
        A = sp.cooe(dtype, n, m, r, c, v)
        if conv:
            A = sp.convert(conv, A, *args)
    y = sp.spmv(A, x, opts(**o))
    ok, err, bound = fp_bound_ok(y, y_hi, a, cnt, dtype)
    assert ok, (A.kind, o, int(np.argmax(err - bound)))


# ---------------------------------------------------------------------------
# banded, BCSR / BCOO
# ---------------------------------------------------------------------------
@functools.lru_cache(maxsize=1)
def banded(dtype, rb):
    B = sp.synth.block_banded(rb=rb, cb=rb, dtype=capi.DTYPES[dtype].np)
    A = capi.bcsr(dtype, B["nrows"], B["ncols"], rb, rb, B["browptr"], B["bcolind"], B["bval"], B["nnz"],
                  B["nnz_per_block"])
    return B, A


BANDED = [("bcsr", dict(nr_parts=PARTS, part_balance=capi.BAL_BLOCK)),
          ("bcsr", dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ)),
          ("bcoo", dict(nr_parts=PARTS, part_balance=capi.BAL_BLOCK)),
          ("bcoo", dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ_ELEM))]


@pytest.mark.parametrize("dtype", ["i8", "i16", "i64", "f32"])
@pytest.mark.parametrize("rb", [4, 8])
def test_banded_fullsize(dtype, rb):
    B, A = banded(dtype, rb)
    x = B["x"]
    O = sp.convert("bcsr2bcoo", A)
    if dtype != "f32":
        want = oracle_spmv(A, x)
    else:
        # FP64 evaluation of the same blocks, and of |blocks| x |x| for the bound
        A64 = capi.bcsr("f64", B["nrows"], B["ncols"], rb, rb, B["browptr"], B["bcolind"],
                        B["bval"].astype(np.float64), B["nnz"], B["nnz_per_block"])
        Aabs = capi.bcsr("f64", B["nrows"], B["ncols"], rb, rb, B["browptr"], B["bcolind"],
                         np.abs(B["bval"].astype(np.float64)), B["nnz"], B["nnz_per_block"])
        y64 = oracle_spmv(A64, x.astype(np.float64))
        yabs = oracle_spmv(Aabs, np.abs(x.astype(np.float64)))
        cnt = np.repeat(np.diff(B["browptr"].astype(np.int64)) * rb, rb)[: B["nrows"]]
    for kind, o in BANDED:
        M = A if kind == "bcsr" else O
        y = sp.spmv(M, x, opts(**o))
        if dtype != "f32":
            assert np.array_equal(y, want), (kind, o)
        else:
            ok, err, bound = fp_bound_ok(y, y64, yabs, cnt, "f32")
            assert ok, (kind, o, int(np.argmax(err - bound)))
