"""The batched multi-RHS path at its benchmark size: 512 CSR matrices, rows
log-uniform in [1k, 256k], uniform / Zipf / banded, 1-32 right-hand sides
each (seed 3), FP32 and INT32.

Every column of every matrix is checked against the oracle (the reference's
CSR spmv_host restated, run once per matrix and right-hand side on all host
cores) for four schedules of the same batch: plain per-matrix launches, the
one-launch queue with default, learned and exhaustively autotuned variants.
INT32 must match bit for bit; FP32 must satisfy, per row,
|y - y_oracle| <= 2 gamma_n sum_j |a_rj x_j| (both are sums of the same
products, each within gamma_n of the exact value; sum |a x| is the oracle's
own sum of |a| |x|, covered by a 1.01 factor)."""
import concurrent.futures as cf
import ctypes as C
import os

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi, selector
from helpers import oracle

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def oracle_columns(dtype, w, mats):
    """Oracle y (and sum |a||x| for FP32) of every matrix and right-hand side."""
    o = oracle()
    f = getattr(o, f"oracle_spmv_csr_{dtype}")
    np_dt = capi.DTYPES[dtype].np
    abs_mats = [sp.csr(dtype, d["n"], d["n"], d["rowptr"], d["colind"], np.abs(d["values"])) for d in w] \
        if dtype == "f32" else None

    def one(m):
        d = w[m]
        n, k = d["n"], d["k"]
        y = np.zeros((n, k), np_dt)
        ya = np.zeros((n, k), np_dt) if abs_mats else None
        buf = np.zeros(n + 8, np_dt)
        for j in range(k):
            x = np.zeros(n + 16, np_dt)
            x[:n] = d["x"][:, j]
            f(buf.ctypes.data_as(C.c_void_p), mats[m].ref, x.ctypes.data_as(C.c_void_p))
            y[:, j] = buf[:n]
            if abs_mats:
                x[:n] = np.abs(d["x"][:, j])
                f(buf.ctypes.data_as(C.c_void_p), abs_mats[m].ref, x.ctypes.data_as(C.c_void_p))
                ya[:, j] = buf[:n]
        return y, ya

    with cf.ThreadPoolExecutor(os.cpu_count() or 4) as ex:  # ctypes releases the GIL during each call
        return list(ex.map(one, range(len(w))))


def check_all(dtype, b, w, ref, label):
    u = 2.0 ** -24
    worst = 0.0
    for m, d in enumerate(w):
        y = b.get_y(m)
        y_or, y_abs = ref[m]
        if dtype == "i32":
            bad = np.argwhere(y != y_or)
            assert bad.size == 0, f"{label}: matrix {m} differs at (row, column) {bad[:3].tolist()}"
        else:
            n_r = np.diff(d["rowptr"].astype(np.int64)).astype(np.float64)[:, None]
            g = np.maximum(n_r, 1) * u / (1 - np.maximum(n_r, 1) * u)
            bound = 1.01 * 2 * g * y_abs.astype(np.float64) + 1e-300
            r = np.abs(y.astype(np.float64) - y_or.astype(np.float64)) / bound
            worst = max(worst, float(r.max()) if r.size else 0.0)
            assert (r <= 1.0).all(), f"{label}: matrix {m} outside the bound at {np.argwhere(r > 1)[:3].tolist()}"
    print(f"{label}: {len(w)} matrices, max |y - y_oracle| / (2 gamma_n sum|ax|) = {worst:.3g}")


@pytest.mark.parametrize("dtype", ["f32", "i32"])
def test_batch_512_every_column(dtype):
    w = sp.synth.batch_workload(nmats=512, dtype=capi.DTYPES[dtype].np)
    mats = [sp.csr(dtype, d["n"], d["n"], d["rowptr"], d["colind"], d["values"]) for d in w]
    b = capi.Batch(dtype, mats, [d["k"] for d in w])
    for m, d in enumerate(w):
        b.set_x(m, d["x"])
    ref = oracle_columns(dtype, w, mats)

    b.execute_per_matrix()
    check_all(dtype, b, w, ref, f"{dtype} plain per-matrix")
    b.execute()
    b.status()
    check_all(dtype, b, w, ref, f"{dtype} queue, default variants")
    b.select(selector.selector(selector.load()), min_confidence=0.0)
    b.execute()
    b.status()
    check_all(dtype, b, w, ref, f"{dtype} queue, learned variants")
    b.autotune(reps=1)
    b.execute()
    b.status()
    check_all(dtype, b, w, ref, f"{dtype} queue, autotuned variants")
    b.free()
