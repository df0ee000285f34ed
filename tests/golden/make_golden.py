"""Generate tests/golden/golden.npz: outputs of the reference's own host SpMV.

For every SpMV kind of the reference (1D CSR / COO / BCSR / BCOO and the 2D
D / RBD / BD tilings of CSR, COO, BCSR, BCOO) and every element type, a small
seeded matrix (with an empty row band and one long row) is converted by the
reference's OWN converters and multiplied by the reference's OWN spmv_host,
both compiled from the reference tree into oracle/_ref by oracle/build_ref.py.
The fixture keeps the input triplets, x, the conversion parameters and y, so
tests can replay the pipeline through this library without the reference
tree.  Run from the repository root where oracle/_ref exists:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import sparsep_b200 as sp  # noqa: E402
from sparsep_b200 import capi  # noqa: E402
from helpers import random_triplets, random_x, ref_lib, ref_spmv, ref_struct  # noqa: E402

OUT = Path(__file__).resolve().parent / "golden.npz"

# (case name, reference directory, kind, params); params: h, v for 2D tilings,
# rb, cb for blocks
CASES = [
    ("csr", "1D/CSR-row", "csr", ()),
    ("cooe", "1D/COO-nnz", "cooe", ()),
    ("bcsr4x4", "1D/BCSR-nnz", "bcsr", (4, 4)),
    ("bcsr3x5", "1D/BCSR-nnz", "bcsr", (3, 5)),
    ("bcoo4x4", "1D/BCOO-nnz", "bcoo", (4, 4)),
    ("dcsr", "2D/DCSR", "dcsr", (3, 4)),
    ("rbdcsr", "2D/RBDCSR", "rbdcsr", (3, 4)),
    ("bdcsr", "2D/BDCSR", "bdcsr", (3, 4)),
    ("dcoo", "2D/DCOO", "dcoo", (3, 4)),
    ("rbdcoo", "2D/RBDCOO", "rbdcoo", (3, 4)),
    ("bdcoo", "2D/BDCOO", "bdcoo", (3, 4)),
    ("dbcsr", "2D/DBCSR", "dbcsr", (2, 3, 4, 4)),
    ("dbcoo", "2D/DBCOO", "dbcoo", (2, 3, 4, 4)),
    ("rbdbcsr", "2D/RBDBCSR-nnz", "rbdbcsr", (2, 3, 4, 4)),
    ("rbdbcoo", "2D/RBDBCOO-nnz", "rbdbcoo", (2, 3, 4, 4)),
    ("bdbcsr", "2D/BDBCSR-nnz", "bdbcsr", (2, 3, 4, 4)),
    ("bdbcoo", "2D/BDBCOO-nnz", "bdbcoo", (2, 3, 4, 4)),
]
NROWS, NCOLS = 57, 61


def reference_struct(kind, L, dtype, rows, cols, vals, params):
    """The reference's converters, from the triplets, as the reference's host
    program chains them."""
    if kind in ("csr", "bcsr", "bcoo"):
        B = sp.coo(dtype, NROWS, NCOLS, rows, cols, vals)
        L.ref_coo2csr.restype = C.c_void_p
        c = L.ref_coo2csr(B.ref)
        if kind == "csr":
            return ref_struct("csr", dtype, c), B
        if kind == "bcsr":
            L.ref_csr2bcsr.restype = C.c_void_p
            return ref_struct("bcsr", dtype, L.ref_csr2bcsr(C.c_void_p(c), *params)), B
        L.ref_csr2bcoo.restype = C.c_void_p
        return ref_struct("bcoo", dtype, L.ref_csr2bcoo(C.c_void_p(c), *params)), B
    A = sp.cooe(dtype, NROWS, NCOLS, rows, cols, vals)
    if kind == "cooe":  # shuffled triplets, sorted by the reference's sortCOOMatrix
        L.ref_sort(A.ref)
        return A, A
    L.ref_convert.restype = C.c_void_p  # 2D: the converters take (row, col)-sorted COO
    return ref_struct(kind, dtype, L.ref_convert(A.ref, *params)), A


def main():
    data = {}
    for ci, (name, d, kind, params) in enumerate(CASES):
        for di, dtype in enumerate(capi.DTYPES):
            rng = np.random.default_rng(1000 + 10 * ci + di)
            block2d = kind in ("dbcsr", "dbcoo", "rbdbcsr", "rbdbcoo", "bdbcsr", "bdbcoo")
            # the reference's 2D block counters assert that no stored value is
            # zero (spmv/2D/DBCSR/support/matrix.h:521-557)
            rows, cols, vals = random_triplets(rng, NROWS, NCOLS, 0.08, dtype, long_row=9, nonzero=block2d)
            if kind in ("csr", "bcsr", "bcoo", "cooe"):
                p = rng.permutation(rows.size)
                rows, cols, vals = rows[p], cols[p], vals[p]
            x = random_x(rng, NCOLS, dtype)
            L = ref_lib(d, dtype)
            if L is None:
                raise SystemExit(f"oracle/_ref is missing {d} {dtype}: run oracle/build_ref.py")
            Aref, _keep = reference_struct(kind, L, dtype, rows, cols, vals, params)
            y = ref_spmv(L, Aref, x)
            key = f"{name}/{dtype}"
            data[key + "/rows"] = rows.astype(np.uint32)
            data[key + "/cols"] = cols.astype(np.uint32)
            data[key + "/vals"] = vals
            data[key + "/x"] = x
            data[key + "/y"] = y
            data[key + "/params"] = np.array(params, dtype=np.uint32)
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(CASES) * len(capi.DTYPES)} cases)")


if __name__ == "__main__":
    main()
