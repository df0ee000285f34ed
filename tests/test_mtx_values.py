"""Matrix Market with values (sparsep_read_mtx_values_*): the file's own
values, symmetric / skew-symmetric expansion, pattern files as ones, and the
error codes for what it does not read.  No reference counterpart (the
reference reader replaces values by rand()%4+1; tests/test_reference_pins.py
pins that one)."""
import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi
from helpers import oracle_spmv


def write(tmp_path, text, name="m.mtx"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def arrays(A):
    n = int(A.s.nnz)
    return ([A.s.rowindx[i] for i in range(n)], [A.s.colind[i] for i in range(n)],
            [A.s.values[i] for i in range(n)])


def test_real_general_with_comments(tmp_path):
    f = write(tmp_path, "%%MatrixMarket matrix coordinate real general\n% a comment\n\n3 4 3\n"
                        "1 1 2.5\n3 4 -1e-3\n  2 2   7\n")
    A = sp.read_mtx(f, "f64", "values")
    assert (A.s.nrows, A.s.ncols, A.s.nnz) == (3, 4, 3)
    assert arrays(A) == ([0, 2, 1], [0, 3, 1], [2.5, -1e-3, 7.0])


def test_symmetric_expansion(tmp_path):
    f = write(tmp_path, "%%MatrixMarket matrix coordinate integer symmetric\n3 3 3\n1 1 4\n2 1 -2\n3 2 5\n")
    A = sp.read_mtx(f, "i32", "values")
    assert arrays(A) == ([0, 1, 0, 2, 1], [0, 0, 1, 1, 2], [4, -2, -2, 5, 5])


def test_skew_symmetric_and_pattern(tmp_path):
    f = write(tmp_path, "%%MatrixMarket matrix coordinate real skew-symmetric\n2 2 1\n2 1 1.5\n")
    assert arrays(sp.read_mtx(f, "f32", "values")) == ([1, 0], [0, 1], [1.5, -1.5])
    f = write(tmp_path, "%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n2 1\n3 3\n", "p.mtx")
    assert arrays(sp.read_mtx(f, "f32", "values")) == ([1, 0, 2], [0, 1, 2], [1.0, 1.0, 1.0])


def test_no_banner_is_real_general(tmp_path):
    f = write(tmp_path, "2 2 2\n1 2 0.5\n2 1 -0.25\n")
    assert arrays(sp.read_mtx(f, "f64", "values")) == ([0, 1], [1, 0], [0.5, -0.25])


def test_integer_types_round_and_wrap(tmp_path):
    f = write(tmp_path, "%%MatrixMarket matrix coordinate real general\n1 3 3\n1 1 300\n1 2 -1.6\n1 3 2.5\n")
    assert arrays(sp.read_mtx(f, "i8", "values"))[2] == [44, -2, 3]
    assert arrays(sp.read_mtx(f, "i64", "values"))[2] == [300, -2, 3]


@pytest.mark.parametrize("text,status", [
    ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n", capi.ENOSYS),
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", capi.ENOSYS),
    ("%%MatrixMarket matrix coordinate real hermitian\n1 1 1\n1 1 1\n", capi.ENOSYS),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n", capi.EBADF),
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n", capi.EBADF),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1\n", capi.EBADF),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1\n2 2 2\n", capi.EBADF),
    ("%%MatrixMarket vector coordinate real general\n2 2 1\n1 1 1\n", capi.EBADF),
])
def test_errors(tmp_path, text, status):
    with pytest.raises(capi.SparsepError) as e:
        sp.read_mtx(write(tmp_path, text), "f32", "values")
    assert e.value.status == status


def test_missing_file():
    with pytest.raises(capi.SparsepError) as e:
        sp.read_mtx("/nonexistent/file.mtx", "f32", "values")
    assert e.value.status == capi.EBADF


def test_spmv_of_a_read_symmetric_matrix(tmp_path):
    rng = np.random.default_rng(3)
    n = 40
    D = np.triu(rng.uniform(-1, 1, (n, n)) * (rng.random((n, n)) < 0.2))
    lines = [f"{j + 1} {i + 1} {float(D[i, j]):.17g}" for i in range(n) for j in range(i, n) if D[i, j] != 0]
    f = write(tmp_path, f"%%MatrixMarket matrix coordinate real symmetric\n{n} {n} {len(lines)}\n" + "\n".join(lines))
    A = sp.convert("coo2csr", sp.read_mtx(f, "f64", "values"))
    full = D + np.triu(D, 1).T
    x = rng.uniform(-1, 1, n)
    np.testing.assert_allclose(oracle_spmv(A, x), full @ x, rtol=1e-12, atol=1e-12)
