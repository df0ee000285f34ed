"""Test helpers: the CPU oracle (oracle/liboracle.so), the reference's own
host code (oracle/_ref, when built) and the FP error bound."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

import sparsep_b200 as sp
from sparsep_b200 import capi

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
REF_DIR = ORACLE_DIR / "_ref"
_oracle = None


def oracle() -> C.CDLL:
    global _oracle
    if _oracle is None:
        so = ORACLE_DIR / "liboracle.so"
        src = ORACLE_DIR / "sparsep_oracle.c"
        if not so.exists() or so.stat().st_mtime < src.stat().st_mtime:
            subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "liboracle.so"], check=True)
        _oracle = C.CDLL(str(so))
    return _oracle


def ref_lib(d: str, dtype: str):
    """Reference shim library for directory d (e.g. '1D/CSR-row') or None."""
    name = d.replace("/", "_").replace("-", "_")
    so = REF_DIR / f"libref_{name}_{dtype}.so"
    return C.CDLL(str(so)) if so.exists() else None


def ylen_ref(kind: str, s) -> int:
    """Length of y_host the reference allocates for this struct."""
    if kind in ("bcsr", "bcoo"):
        return int(s.num_block_rows * s.row_block_size)
    if kind in ("dcsr", "dcoo"):
        return int(s.horz_partitions * s.tile_height)
    if kind in ("dbcsr", "dbcoo"):
        return int(s.horz_partitions * s.tile_height + s.row_block_size)
    if kind in ("rbdbcsr", "rbdbcoo", "bdbcsr", "bdbcoo"):
        return int(s.nrows + s.row_block_size)
    return int(s.nrows)


def xlen_ref(kind: str, s) -> int:
    """Columns of x the reference reads (block formats read whole blocks)."""
    n = int(s.ncols)
    if kind in ("dbcsr", "dbcoo"):
        return int(s.vert_partitions * s.tile_width + s.col_block_size) + 8
    if kind in ("rbdbcsr", "rbdbcoo"):
        return n + int(s.tile_width + s.col_block_size) + 8
    if kind in ("bdbcsr", "bdbcoo"):
        return n + int(s.max_tile_width + s.col_block_size) + 8
    if kind in ("dcsr", "dcoo"):
        return int(s.vert_partitions * s.tile_width) + 8
    return n + 16


def padded_x(kind: str, A: capi.HostMatrix, x: np.ndarray) -> np.ndarray:
    xp = np.zeros(max(xlen_ref(kind, A.s), x.size), dtype=x.dtype)
    xp[: x.size] = x
    return xp


def oracle_spmv(A: capi.HostMatrix, x: np.ndarray) -> np.ndarray:
    if A.kind == "coo":
        # the reference never multiplies the unsorted SoA COO directly: it
        # converts it with coo2csr first (spmv/1D/CSR-row/host/app.c:101-103)
        return oracle_spmv(sp.convert("coo2csr", A), x)
    dt = capi.DTYPES[A.dtype]
    xp = padded_x(A.kind, A, np.ascontiguousarray(x, dtype=dt.np))
    y = np.zeros(ylen_ref(A.kind, A.s) + 8, dtype=dt.np)
    f = getattr(oracle(), f"oracle_spmv_{A.kind}_{A.dtype}")
    f(y.ctypes.data_as(C.c_void_p), A.ref, xp.ctypes.data_as(C.c_void_p))
    return y[: int(A.s.nrows)]


def ref_spmv(lib: C.CDLL, A: capi.HostMatrix, x: np.ndarray) -> np.ndarray:
    dt = capi.DTYPES[A.dtype]
    xp = padded_x(A.kind, A, np.ascontiguousarray(x, dtype=dt.np))
    y = np.zeros(ylen_ref(A.kind, A.s) + 8, dtype=dt.np)
    lib.ref_spmv(y.ctypes.data_as(C.c_void_p), A.ref, xp.ctypes.data_as(C.c_void_p))
    return y[: int(A.s.nrows)]


def hi_ref(rows, cols, vals, x, nrows):
    """(y_hi, sum|a x|, terms per row) from triplets, long-double Neumaier sums."""
    o = oracle()
    n = len(rows)
    r = np.ascontiguousarray(rows, dtype=np.uint32)
    c = np.ascontiguousarray(cols, dtype=np.uint32)
    v = np.ascontiguousarray(vals, dtype=np.float64)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(nrows, dtype=np.float64)
    a = np.zeros(nrows, dtype=np.float64)
    cnt = np.zeros(nrows, dtype=np.uint32)
    o.oracle_ref_triplets(C.c_uint64(n), r.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p),
                          v.ctypes.data_as(C.c_void_p), xx.ctypes.data_as(C.c_void_p), C.c_uint32(nrows),
                          y.ctypes.data_as(C.c_void_p), a.ctypes.data_as(C.c_void_p), cnt.ctypes.data_as(C.c_void_p))
    return y, a, cnt


def gamma(n, u):
    n = np.asarray(n, dtype=np.float64)
    return n * u / (1.0 - n * u)


def fp_bound_ok(y, y_hi, abs_sum, cnt, dtype: str, factor: float = 1.0):
    """|y - y_hi| <= factor * gamma_{n_r} * sum|a x| (+ half an ulp of y_hi).

    The bound is the classical dot-product bound for any summation order
    (with or without FMA); y_hi is exact to ~2^-64 relative, so its own
    rounding to double is the only extra term."""
    u = 2.0 ** -24 if dtype == "f32" else 2.0 ** -53
    err = np.abs(y.astype(np.float64) - y_hi)
    bound = factor * gamma(np.maximum(cnt, 1), u) * abs_sum + np.abs(y_hi) * 2.0 ** -53 + 1e-300
    bad = err > bound
    return (not bad.any()), err, bound


def max_rel_err(y, y_hi, abs_sum):
    d = np.abs(y.astype(np.float64) - y_hi)
    s = np.maximum(abs_sum, 1e-300)
    return float((d / s).max()) if d.size else 0.0


def _arr(p, n, dtype):
    n = int(n)
    if n == 0:
        return np.zeros(0, dtype=dtype)
    if not p:
        raise AssertionError("null array pointer")
    return np.ctypeslib.as_array(p, shape=(n,)).copy().view(dtype) if dtype is not None else \
        np.ctypeslib.as_array(p, shape=(n,)).copy()


def struct_arrays(kind: str, dtype: str, s) -> dict:
    """Scalar fields and arrays (with their reference lengths) of a struct."""
    out = {}
    for name, ct in s._fields_:
        if not name.startswith("_") and ct in (C.c_uint32, C.c_uint64):
            out[name] = int(getattr(s, name))
    T = capi.DTYPES[dtype].np
    g = lambda f, n: _arr(getattr(s, f), n, None)  # noqa: E731
    if kind in ("csr",):
        out.update(rowptr=g("rowptr", s.nrows + 1), colind=g("colind", s.nnz), values=g("values", s.nnz))
    elif kind == "coo":
        out.update(rowindx=g("rowindx", s.nnz), colind=g("colind", s.nnz), values=g("values", s.nnz))
    elif kind == "cooe":
        out.update(rows=g("rows", s.nrows), nnzs=g("nnzs", s.nnz))
    elif kind in ("bcsr", "bcoo"):
        nb, bs = int(s.num_blocks), int(s.row_block_size * s.col_block_size)
        out.update(bval=g("bval", nb * bs), nnz_per_block=g("nnz_per_block", nb))
        if kind == "bcsr":
            out.update(browptr=g("browptr", s.num_block_rows + 1), bcolind=g("bcolind", nb))
        else:
            out.update(bind=g("bind", nb))
    elif kind == "dcsr":
        P = s.npartitions
        out.update(nnzs_per_partition=g("nnzs_per_partition", P), drowptr=g("drowptr", P * (s.tile_height + 1)),
                   dcolind=g("dcolind", s.nnz), dval=g("dval", s.nnz))
    elif kind in ("rbdcsr", "bdcsr"):
        V = s.vert_partitions
        out.update(nnzs_per_vert_partition=g("nnzs_per_vert_partition", V),
                   drowptr=g("drowptr", V * (s.nrows + 1)), dcolind=g("dcolind", s.nnz), dval=g("dval", s.nnz))
        if kind == "bdcsr":
            out.update(vert_tile_widths=g("vert_tile_widths", V + 1), nnzs_per_column=g("nnzs_per_column", s.ncols))
    elif kind == "dcoo":
        out.update(nnzs_per_partition=g("nnzs_per_partition", s.npartitions), nnzs=g("nnzs", s.nnz))
    elif kind in ("rbdcoo", "bdcoo"):
        V = s.vert_partitions
        out.update(nnzs_per_vert_partition=g("nnzs_per_vert_partition", V), nnzs=g("nnzs", s.nnz))
        if kind == "bdcoo":
            out.update(vert_tile_widths=g("vert_tile_widths", V + 1), nnzs_per_column=g("nnzs_per_column", s.ncols))
    elif kind in ("dbcsr", "dbcoo", "rbdbcsr", "rbdbcoo", "bdbcsr", "bdbcoo"):
        nb, bs = int(s.nblocks), int(s.row_block_size * s.col_block_size)
        P = s.npartitions
        out.update(bval=g("bval", nb * bs), nnz_per_block=g("nnz_per_block", nb))
        if kind.startswith("d"):
            out.update(nnzs_per_partition=g("nnzs_per_partition", P), blocks_per_partition=g("blocks_per_partition", P))
        else:
            out.update(nnzs_per_vert_partition=g("nnzs_per_vert_partition", P),
                       blocks_per_vert_partition=g("blocks_per_vert_partition", P))
        if kind.startswith("bd"):
            out.update(vert_tile_widths=g("vert_tile_widths", P + 1), nnzs_per_column=g("nnzs_per_column", s.ncols))
        if kind.endswith("bcsr"):
            out.update(browptr=g("browptr", P * (s.num_block_rows + 1)), bcolind=g("bcolind", nb))
        else:
            out.update(bind=g("bind", nb))
    return out


def assert_same_struct(kind, dtype, a, b):
    A, B = struct_arrays(kind, dtype, a), struct_arrays(kind, dtype, b)
    assert A.keys() == B.keys()
    for k in A:
        if isinstance(A[k], int):
            assert A[k] == B[k], f"{kind}.{k}: {A[k]} != {B[k]}"
        elif A[k].dtype.names:
            for f in A[k].dtype.names:
                assert np.array_equal(A[k][f], B[k][f]), f"{kind}.{k}.{f} differs"
        else:
            assert A[k].tobytes() == B[k].tobytes(), f"{kind}.{k} differs"


def ref_struct(kind: str, dtype: str, p: int) -> capi.HostMatrix:
    """Wrap a struct pointer returned by a reference shim (never freed)."""
    st = capi.STRUCTS[dtype][kind]
    s = C.cast(C.c_void_p(p), C.POINTER(st)).contents
    return capi.HostMatrix(kind, dtype, s, {})


def random_triplets(rng, nrows, ncols, density, dtype, long_row=None, empty_frac=0.1, unique=True, nonzero=False):
    """Random sparse triplets with empty rows and an optional long row, sorted by (row, col)."""
    rows, cols = [], []
    for r in range(nrows):
        if rng.random() < empty_frac:
            continue
        k = rng.binomial(ncols, density)
        if long_row is not None and r == long_row:
            k = ncols // 2
        c = rng.choice(ncols, size=min(k, ncols), replace=False) if unique else rng.integers(0, ncols, k)
        rows.extend([r] * len(c))
        cols.extend(sorted(c))
    rows = np.asarray(rows, dtype=np.uint32)
    cols = np.asarray(cols, dtype=np.uint32)
    dt = np.dtype(capi.DTYPES[dtype].np)
    if dt.kind == "f":
        vals = rng.uniform(-1, 1, rows.size).astype(dt)
    else:
        lo, hi = (-128, 127) if dt.itemsize == 1 else (-30000, 30000)
        vals = rng.integers(lo, hi + 1, rows.size).astype(dt)
    if nonzero:
        vals[vals == 0] = 1
    return rows, cols, vals


def random_x(rng, n, dtype):
    dt = np.dtype(capi.DTYPES[dtype].np)
    if dt.kind == "f":
        return rng.uniform(-1, 1, n).astype(dt)
    lo, hi = (-128, 127) if dt.itemsize == 1 else (-30000, 30000)
    return rng.integers(lo, hi + 1, n).astype(dt)
