"""1D row sharding over ranks (sparsep_b200.shard), on the CPU with gloo and
world size 2: rows split by the reference's partition_by_nnz, each rank's
slice multiplied with the x assembled by the all-gather of every rank's x
slice; the ranks' y slices put together equal the whole product.  The
multiply here is the test's own (numpy, exact for integers); the GPU plan of
a slice is covered by tests/test_gpu_shard.py."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def matrix(seed=0, n=3001):
    rng = np.random.default_rng(seed)
    lens = np.minimum(rng.zipf(2.0, n) * 3, 800)
    rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)
    colind = rng.integers(0, n, int(rowptr[-1])).astype(np.uint32)
    values = rng.integers(-8, 9, colind.size).astype(np.int64)
    x = rng.integers(-8, 9, n).astype(np.int64)
    return n, rowptr, colind, values, x


def csr_mul(rowptr, colind, values, x):
    rows = np.repeat(np.arange(len(rowptr) - 1), np.diff(rowptr.astype(np.int64)))
    return np.bincount(rows, weights=values * x[colind], minlength=len(rowptr) - 1).astype(np.int64)


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    from sparsep_b200 import shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    n, rowptr, colind, values, x = matrix()
    b = shard.row_bounds(rowptr, n, world)
    r0, r1 = int(b[rank]), int(b[rank + 1])
    A = shard.row_slice("i64", n, n, rowptr, colind, values, r0, r1)
    xs = torch.from_numpy(x[r0:r1].copy())
    xfull = shard.gather_x(xs, b, rank).numpy()
    rp = np.ctypeslib.as_array(A.s.rowptr, (r1 - r0 + 1,)).copy()
    ci = np.ctypeslib.as_array(A.s.colind, (int(A.s.nnz),)).copy() if A.s.nnz else np.zeros(0, np.uint32)
    va = np.ctypeslib.as_array(A.s.values, (int(A.s.nnz),)).copy() if A.s.nnz else np.zeros(0, np.int64)
    out[rank] = (b.tolist(), np.array_equal(xfull, x), csr_mul(rp, ci, va, xfull).tolist())
    dist.destroy_process_group()


def test_two_ranks_row_shards_assemble_the_product():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    n, rowptr, colind, values, x = matrix()
    b = res[0][0]
    assert b == res[1][0] and b[0] == 0 and b[-1] == n
    nnz = np.diff(rowptr.astype(np.int64)[b])
    assert abs(int(nnz[0]) - int(nnz[1])) <= int(np.diff(rowptr.astype(np.int64)).max())  # balanced by nonzeros
    assert res[0][1] and res[1][1], "the all-gather did not rebuild x"
    y = np.concatenate([np.array(res[0][2]), np.array(res[1][2])])
    assert np.array_equal(y, csr_mul(rowptr, colind, values, x))


def test_row_bounds_match_the_reference_partition():
    sys.path.insert(0, str(ROOT))
    from sparsep_b200 import shard

    n, rowptr, _, _, _ = matrix(seed=1)
    for parts in (1, 2, 3, 8):
        b = shard.row_bounds(rowptr, n, parts)
        assert len(b) == parts + 1 and b[0] == 0 and b[-1] == n and np.all(np.diff(b) >= 0)
