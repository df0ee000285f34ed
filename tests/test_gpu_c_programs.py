"""A compiled reference-style C program, run end to end on the GPU.

tests/ref_app.c reads a Matrix Market file with the reference's own reader
name (readCOOMatrix), converts it with coo2csr / csr2bcsr / bcsr2bcoo,
multiplies through the C-ABI as CSR (one-shot over 64 nnz-balanced parts, and
a plan run twice on host buffers), BCSR 4x4, BCOO 4x4 and the plan variant
the learned selector picks (sparsep_opts.autotune = 1), and writes its
arrays.  The results must equal the oracle's (the reference's spmv_host
restated) on the CSR the program built: integers bit for bit, FP32 / FP64
within the per-row gamma bound of a long-double sum."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import fp_bound_ok, hi_ref, oracle_spmv

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
MACRO = {"i8": "INT8", "i16": "INT16", "i32": "INT32", "i64": "INT64", "f32": "FP32", "f64": "FP64"}


def write_mtx(path, nrows, ncols, rows, cols):
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern general\n")
        f.write(f"{nrows} {ncols} {len(rows)}\n")
        for r, c in zip(rows, cols):
            f.write(f"{r + 1} {c + 1}\n")


@pytest.mark.parametrize("dtype", list(MACRO))
def test_reference_style_program_runs(tmp_path, dtype):
    exe = tmp_path / "ref_app"
    lib_dir = ROOT / "sparsep_b200"
    subprocess.run(["gcc", "-std=c11", "-O2", f"-I{ROOT / 'include'}", "-DSPARSEP_REFERENCE_NAMES",
                    f"-D{MACRO[dtype]}", str(ROOT / "tests" / "ref_app.c"), f"-L{lib_dir}", "-lsparsep_b200",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    rng = np.random.default_rng(11)
    nrows, ncols = 1500, 1300
    key = np.unique(rng.integers(0, nrows * ncols, 12000))
    rows, cols = key // ncols, key % ncols
    order = rng.permutation(rows.size)  # the file in any order
    mtx = tmp_path / "m.mtx"
    write_mtx(mtx, nrows, ncols, rows[order], cols[order])
    out = subprocess.run([str(exe), str(mtx), str(tmp_path / "o")], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    n, m, nnz = (int(v) for v in out.stdout.split())
    T = capi.DTYPES[dtype].np
    ld = lambda name, dt: np.fromfile(tmp_path / f"o.{name}", dtype=dt)  # noqa: E731
    rp, ci, vv, x = ld("rowptr", np.uint32), ld("colind", np.uint32), ld("values", T), ld("x", T)
    assert rp.size == n + 1 and ci.size == nnz == rows.size
    A = sp.csr(dtype, n, m, rp, ci, vv)
    for name in ("y_csr", "y_plan", "y_bcsr", "y_bcoo", "y_auto"):
        y = ld(name, T)
        if dtype in ("f32", "f64"):
            r = np.repeat(np.arange(n, dtype=np.uint32), np.diff(rp.astype(np.int64)))
            y_hi, a, cnt = hi_ref(r, ci, vv.astype(np.float64), x.astype(np.float64), n)
            ok, err, bound = fp_bound_ok(y, y_hi, a, cnt, dtype)
            assert ok, (name, np.nonzero(err > bound)[0][:5])
        else:
            assert np.array_equal(y, oracle_spmv(A, x)), name
