"""C-ABI surface (no GPU needed): the library loads and exports every
function include/sparsep.h declares; host-side error handling returns status
codes instead of aborting."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    out = subprocess.run(["gcc", "-E", "-P", "-x", "c", str(ROOT / "include" / "sparsep.h")], capture_output=True,
                         text=True, check=True).stdout
    names = set(re.findall(r"\b(sparsep_\w+)\s*\(", out))
    return sorted(names)


def test_exports_every_declared_symbol():
    L = capi.lib()
    names = declared_functions()
    assert len(names) > 300, len(names)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing[:10]


def test_version_and_strerror():
    L = capi.lib()
    assert b"sm_100a" in L.sparsep_version()
    for st in (0, -5, -12, -19, -22, -38, -34, -110, -9):
        assert L.sparsep_strerror(st)


def test_options_validation_without_gpu():
    # invalid options are rejected before any device call
    A = sp.csr("f32", 2, 2, np.array([0, 1, 2]), np.array([0, 1]), np.array([1.0, 2.0], np.float32))
    h = C.c_void_p()
    for bad in (dict(lanes=3), dict(lanes=64), dict(nr_workers=17), dict(sync=9), dict(part_balance=7)):
        o = sp.default_opts(**bad)
        st = capi.lib().sparsep_plan_csr_f32(A.ref, C.byref(o), C.byref(h))
        assert st == capi.EINVAL, (bad, st)
    assert capi.lib().sparsep_plan_csr_f32(None, None, C.byref(h)) in (capi.EINVAL, capi.ENODEV)


@pytest.mark.parametrize("content", [
    "",                                   # empty file
    "% only a comment\n",                # no header
    "3 3 2\n1 1 5\n",                     # fewer entries than declared
    "3 3 1\n1 1 5\n2 2 5\n",              # more entries than declared
    "3 3 1\n0 1 5\n",                     # 0-based index
    "3 3 1\n4 1 5\n",                     # row out of range
    "3 3 1\n1\n",                         # truncated entry
])
def test_malformed_mtx(tmp_path, content):
    p = tmp_path / "bad.mtx"
    p.write_text(content)
    for flavour in ("coo", "cooe", "coo_nopad"):
        with pytest.raises(sp.SparsepError) as e:
            sp.read_mtx(p, "f32", flavour)
        assert e.value.status == capi.EBADF


def test_missing_file():
    with pytest.raises(sp.SparsepError) as e:
        sp.read_mtx("/nonexistent/x.mtx", "i32")
    assert e.value.status == capi.EBADF


def test_converter_validation():
    # unsorted AoS input is rejected by the 2D converters (they assume sortCOOMatrix ran)
    A = sp.cooe("f32", 4, 4, np.array([2, 1]), np.array([0, 0]), np.array([1, 1], np.float32))
    with pytest.raises(sp.SparsepError):
        sp.convert("cooe2dcsr", A, 2, 2)
    # zero block size
    B = sp.csr("f32", 2, 2, np.array([0, 1, 2]), np.array([0, 1]), np.array([1.0, 2.0], np.float32))
    with pytest.raises(sp.SparsepError):
        sp.convert("csr2bcsr", B, 0, 4)
    # column index out of range
    Cx = sp.coo("f32", 2, 2, np.array([0]), np.array([5]), np.array([1.0], np.float32))
    with pytest.raises(sp.SparsepError):
        sp.convert("coo2csr", Cx)


def test_partition_entry_points():
    L = capi.lib()
    s = (C.c_uint32 * 5)()
    assert L.sparsep_partition_by_row(10, 4, s) == 0
    assert list(s) == [0, 3, 6, 8, 10]
    e = (C.c_uint64 * 4)()
    assert L.sparsep_partition_by_elem(10, 3, e) == 0
    assert list(e) == [0, 4, 7, 10]
    assert L.sparsep_partition_by_row(10, 0, s) == capi.EINVAL


@pytest.mark.parametrize("macro", ["INT8", "INT16", "INT32", "INT64", "FP32", "FP64"])
def test_compat_header_builds_reference_style_code(tmp_path, macro):
    """A reference-style host program (struct CSRMatrix, val_dt, -D<TYPE>)
    compiles against include/sparsep_compat.h and links to the library."""
    out = tmp_path / "compat"
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", f"-I{ROOT / 'include'}", f"-D{macro}",
                        str(ROOT / "tests" / "compat_check.c"), f"-L{ROOT / 'sparsep_b200'}", "-lsparsep_b200",
                        "-o", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("macro", ["INT8", "INT16", "INT32", "INT64", "FP32", "FP64"])
def test_reference_names_build(tmp_path, macro):
    """An unmodified-style reference host program that calls readCOOMatrix,
    coo2csr, csr2bcsr, bcsr2bcoo and free*Matrix by the reference's own names
    and signatures (tests/ref_app.c, -DSPARSEP_REFERENCE_NAMES) compiles
    warning-free and links to the library; tests/test_gpu_c_programs.py runs it."""
    out = tmp_path / "ref_app"
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}",
                        "-DSPARSEP_REFERENCE_NAMES", f"-D{macro}", str(ROOT / "tests" / "ref_app.c"),
                        f"-L{ROOT / 'sparsep_b200'}", "-lsparsep_b200", "-o", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_api_example_builds(tmp_path):
    """A C caller of the batch, selector, CG and value-reader entry points
    (tests/api_example.c) compiles warning-free and links to the library."""
    out = tmp_path / "api_example"
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}",
                        str(ROOT / "tests" / "api_example.c"), f"-L{ROOT / 'sparsep_b200'}", "-lsparsep_b200",
                        "-o", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_plan_info_layout_matches_header(tmp_path):
    """capi.PlanInfo mirrors sparsep_plan_info field for field (size and the
    offsets of every field, from a C program compiled against the header)."""
    names = [f[0] for f in capi.PlanInfo._fields_]
    src = tmp_path / "layout.c"
    src.write_text("#include <stddef.h>\n#include <stdio.h>\n#include \"sparsep.h\"\nint main(void) {\n"
                   '  printf("%zu", sizeof(sparsep_plan_info));\n'
                   + "".join(f'  printf(" %zu", offsetof(sparsep_plan_info, {n}));\n' for n in names)
                   + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(capi.PlanInfo)] + [getattr(capi.PlanInfo, n).offset for n in names]
    assert got == want
