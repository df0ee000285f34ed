"""Pins the oracle and the host converters against the reference's own code.

The reference's support headers and spmv_host are compiled from the reference
tree into oracle/_ref (oracle/build_ref.py).  Every test here compares, on the
same seeded inputs:
  * the library's converter output with the reference converter's, array by
    array (bit-exact), and
  * the oracle's SpMV with the reference's spmv_host on the reference-built
    struct (bit-exact for every element type: same loop order, same types).
Skipped where oracle/_ref is absent; tests/golden carries the same pins as
committed vectors."""
import ctypes as C

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import (REF_DIR, assert_same_struct, oracle_spmv, random_triplets, random_x, ref_lib, ref_spmv,
                     ref_struct)

DT = list(capi.DTYPES)
needs_ref = pytest.mark.skipif(not REF_DIR.exists(), reason="oracle/_ref not built (reference tree absent)")


def _coo_soa(dtype, nrows, ncols, rows, cols, vals, shuffle_rng=None):
    if shuffle_rng is not None:
        p = shuffle_rng.permutation(rows.size)
        rows, cols, vals = rows[p], cols[p], vals[p]
    return sp.coo(dtype, nrows, ncols, rows, cols, vals)


@needs_ref
@pytest.mark.parametrize("dtype", DT)
def test_csr_pipeline(dtype):
    rng = np.random.default_rng(10)
    nrows, ncols = 203, 197
    r, c, v = random_triplets(rng, nrows, ncols, 0.05, dtype, long_row=7)
    B = _coo_soa(dtype, nrows, ncols, r, c, v, shuffle_rng=rng)
    L = ref_lib("1D/CSR-row", dtype)
    L.ref_coo2csr.restype = C.c_void_p
    Aref = ref_struct("csr", dtype, L.ref_coo2csr(B.ref))
    A = sp.convert("coo2csr", B)
    assert_same_struct("csr", dtype, A.s, Aref.s)
    x = random_x(rng, ncols, dtype)
    assert np.array_equal(oracle_spmv(A, x), ref_spmv(L, Aref, x))


@needs_ref
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("rb,cb", [(4, 4), (8, 8), (2, 2), (3, 5)])
def test_bcsr_bcoo_pipeline(dtype, rb, cb):
    rng = np.random.default_rng(11 + rb)
    nrows, ncols = 130, 150
    r, c, v = random_triplets(rng, nrows, ncols, 0.06, dtype, long_row=3)
    B = _coo_soa(dtype, nrows, ncols, r, c, v, shuffle_rng=rng)
    L = ref_lib("1D/BCSR-nnz", dtype)
    L.ref_coo2csr.restype = C.c_void_p
    L.ref_csr2bcsr.restype = C.c_void_p
    Cref = L.ref_coo2csr(B.ref)
    Bref = ref_struct("bcsr", dtype, L.ref_csr2bcsr(C.c_void_p(Cref), rb, cb))
    A = sp.convert("csr2bcsr", sp.convert("coo2csr", B), rb, cb)
    assert_same_struct("bcsr", dtype, A.s, Bref.s)
    x = random_x(rng, ncols, dtype)
    assert np.array_equal(oracle_spmv(A, x), ref_spmv(L, Bref, x))
    # BCOO
    L2 = ref_lib("1D/BCOO-nnz", dtype)
    L2.ref_coo2csr.restype = C.c_void_p
    L2.ref_csr2bcoo.restype = C.c_void_p
    Oref = ref_struct("bcoo", dtype, L2.ref_csr2bcoo(C.c_void_p(L2.ref_coo2csr(B.ref)), rb, cb))
    O = sp.convert("bcsr2bcoo", A)
    assert_same_struct("bcoo", dtype, O.s, Oref.s)
    assert np.array_equal(oracle_spmv(O, x), ref_spmv(L2, Oref, x))


def _sorted_cooe(dtype, rng, nrows=161, ncols=173, density=0.05, nonzero=False):
    r, c, v = random_triplets(rng, nrows, ncols, density, dtype, long_row=5, nonzero=nonzero)
    return sp.cooe(dtype, nrows, ncols, r, c, v), (r, c, v)


@needs_ref
@pytest.mark.parametrize("dtype", DT)
def test_cooe_sort_and_spmv(dtype):
    rng = np.random.default_rng(12)
    nrows, ncols = 161, 173
    r, c, v = random_triplets(rng, nrows, ncols, 0.05, dtype, long_row=5)
    p = rng.permutation(r.size)
    A = sp.cooe(dtype, nrows, ncols, r[p], c[p], v[p])
    Aref = sp.cooe(dtype, nrows, ncols, r[p], c[p], v[p])
    L = ref_lib("1D/COO-nnz", dtype)
    L.ref_sort(Aref.ref)
    sp.sort_cooe(A)
    assert_same_struct("cooe", dtype, A.s, Aref.s)
    x = random_x(rng, ncols, dtype)
    assert np.array_equal(oracle_spmv(A, x), ref_spmv(L, Aref, x))


TWO_D = [("2D/DCSR", "cooe2dcsr", "dcsr"), ("2D/RBDCSR", "cooe2rbdcsr", "rbdcsr"),
         ("2D/BDCSR", "cooe2bdcsr", "bdcsr"), ("2D/DCOO", "cooe2dcoo", "dcoo"),
         ("2D/RBDCOO", "cooe2rbdcoo", "rbdcoo"), ("2D/BDCOO", "cooe2bdcoo", "bdcoo")]


@needs_ref
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("d,conv,kind", TWO_D)
@pytest.mark.parametrize("h,v", [(4, 3), (2, 8), (1, 1)])
def test_2d_pipeline(dtype, d, conv, kind, h, v):
    rng = np.random.default_rng(13)
    A, _ = _sorted_cooe(dtype, rng)
    L = ref_lib(d, dtype)
    L.ref_convert.restype = C.c_void_p
    Dref = ref_struct(kind, dtype, L.ref_convert(A.ref, h, v))
    D = sp.convert(conv, A, h, v)
    assert_same_struct(kind, dtype, D.s, Dref.s)
    x = random_x(rng, A.s.ncols, dtype)
    assert np.array_equal(oracle_spmv(D, x), ref_spmv(L, Dref, x))


TWO_D_BLOCK = [("2D/DBCSR", "cooe2dcsr", "dcsr2dbcsr", "dbcsr"), ("2D/DBCOO", "cooe2dcsr", "dcsr2dbcoo", "dbcoo"),
               ("2D/RBDBCSR-nnz", "cooe2rbdcsr", "rbdcsr2rbdbcsr", "rbdbcsr"),
               ("2D/RBDBCOO-nnz", "cooe2rbdcsr", "rbdcsr2rbdbcoo", "rbdbcoo"),
               ("2D/BDBCSR-nnz", "cooe2bdcsr", "bdcsr2bdbcsr", "bdbcsr"),
               ("2D/BDBCOO-nnz", "cooe2bdcsr", "bdcsr2bdbcoo", "bdbcoo")]


@needs_ref
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("d,c1,c2,kind", TWO_D_BLOCK)
@pytest.mark.parametrize("h,v,rb,cb", [(4, 3, 4, 4), (2, 5, 2, 2), (3, 2, 8, 8)])
def test_2d_block_pipeline(dtype, d, c1, c2, kind, h, v, rb, cb):
    rng = np.random.default_rng(14)
    # the reference's block counters assert that no stored value is zero
    # (countNNZperBlockDBCSRMatrix, spmv/2D/DBCSR/support/matrix.h:521-557)
    A, _ = _sorted_cooe(dtype, rng, nonzero=True)
    L = ref_lib(d, dtype)
    L.ref_convert.restype = C.c_void_p
    Dref = ref_struct(kind, dtype, L.ref_convert(A.ref, h, v, rb, cb))
    D = sp.convert(c2, sp.convert(c1, A, h, v), rb, cb)
    assert_same_struct(kind, dtype, D.s, Dref.s)
    x = random_x(rng, A.s.ncols, dtype)
    assert np.array_equal(oracle_spmv(D, x), ref_spmv(L, Dref, x))


@needs_ref
@pytest.mark.parametrize("parts", [1, 3, 8, 64])
def test_partitions_vs_reference(parts):
    rng = np.random.default_rng(15)
    nrows, ncols = 300, 120
    r, c, v = random_triplets(rng, nrows, ncols, 0.05, "i32", long_row=17)
    A = sp.convert("coo2csr", sp.coo("i32", nrows, ncols, r, c, v))
    rp = A.arrays["_src"]  # keep alive
    L = capi.lib()
    mine = (C.c_uint32 * (parts + 2))()
    ref = (C.c_uint32 * (parts + 2))()
    Lr = ref_lib("1D/CSR-row", "i32")
    Lr.ref_partition_by_row(A.ref, parts, ref)
    L.sparsep_partition_by_row(nrows, parts, mine)
    assert list(mine)[: parts + 1] == list(ref)[: parts + 1]
    Ln = ref_lib("1D/CSR-nnz", "i32")
    Ln.ref_partition_by_nnz(A.ref, parts, ref)
    L.sparsep_partition_by_nnz(A.s.rowptr, nrows, parts, mine)
    assert list(mine)[: parts + 1] == list(ref)[: parts + 1]
    del rp
    # BCSR block-row splits by nnz and by blocks
    Bm = sp.convert("csr2bcsr", A, 4, 4)
    Lb = ref_lib("1D/BCSR-nnz", "i32")
    Lb.ref_partition_by_nnz(Bm.ref, parts, ref)
    L.sparsep_partition_block_rows(Bm.s.browptr, Bm.s.num_block_rows, Bm.s.nnz_per_block, parts, mine)
    if parts > 1:
        assert list(mine)[: parts + 1] == list(ref)[: parts + 1]
    Lk = ref_lib("1D/BCSR-block", "i32")
    Lk.ref_partition_by_blocks(Bm.ref, parts, ref)
    L.sparsep_partition_block_rows(Bm.s.browptr, Bm.s.num_block_rows, None, parts, mine)
    assert list(mine)[: parts + 1] == list(ref)[: parts + 1]


def _write_mtx(path, nrows, ncols, entries, comments=("%%MatrixMarket matrix coordinate real general",)):
    with open(path, "w") as f:
        for cmt in comments:
            f.write(cmt + "\n")
        f.write(f"{nrows} {ncols} {len(entries)}\n")
        for r, c in entries:
            f.write(f"{r + 1} {c + 1} 1.5\n")


@needs_ref
@pytest.mark.parametrize("dtype", DT)
def test_reader_vs_reference(tmp_path, dtype):
    rng = np.random.default_rng(16)
    nrows, ncols = 37, 29
    r, c, _ = random_triplets(rng, nrows, ncols, 0.1, "i32")
    path = tmp_path / "m.mtx"
    _write_mtx(path, nrows, ncols, list(zip(r.tolist(), c.tolist())))
    libc = C.CDLL(None)
    # SoA reader (CSR family, padded)
    L = ref_lib("1D/CSR-row", dtype)
    L.ref_read.restype = C.c_void_p
    libc.srand(1)
    Rref = ref_struct("coo", dtype, L.ref_read(str(path).encode()))
    libc.srand(1)
    R = sp.read_mtx(path, dtype, "coo")
    assert_same_struct("coo", dtype, R.s, Rref.s)
    # AoS reader (COO / 2D family)
    L2 = ref_lib("1D/COO-nnz", dtype)
    L2.ref_read.restype = C.c_void_p
    libc.srand(1)
    Eref = ref_struct("cooe", dtype, L2.ref_read(str(path).encode()))
    libc.srand(1)
    E = sp.read_mtx(path, dtype, "cooe")
    assert_same_struct("cooe", dtype, E.s, Eref.s)
    # BCSR family reader: no padding
    L3 = ref_lib("1D/BCSR-nnz", dtype)
    L3.ref_read.restype = C.c_void_p
    libc.srand(1)
    Nref = ref_struct("coo", dtype, L3.ref_read(str(path).encode()))
    libc.srand(1)
    N = sp.read_mtx(path, dtype, "coo_nopad")
    assert_same_struct("coo", dtype, N.s, Nref.s)
