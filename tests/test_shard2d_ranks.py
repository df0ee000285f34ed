"""2D tile sharding over a P x Q grid of ranks (sparsep_b200.shard), on the CPU
with gloo: rank (p, q) holds the tile of row block p (rows split by
partition_by_nnz) and column segment q (equal widths) with local column
indices, multiplies it with its own x segment only, and the reduce-scatter of
the partial row blocks over the row block's Q ranks hands every rank its
sub-slice of y; all sub-slices together equal the whole product.  The
multiply here is the test's own (numpy, exact for integers); the GPU plans of
tiles are covered by tests/test_gpu_shard.py."""
import datetime
import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

from test_shard_ranks import _free_port, csr_mul, matrix

ROOT = Path(__file__).resolve().parents[1]


def _rank(rank, world, grid, port, out):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    from sparsep_b200 import shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    P, Q = grid
    p, q = divmod(rank, Q)
    n, rowptr, colind, values, x = matrix(seed=2, n=2501)
    rb, cb = shard.row_bounds(rowptr, n, P), shard.col_bounds(n, Q)
    r0, r1, c0, c1 = int(rb[p]), int(rb[p + 1]), int(cb[q]), int(cb[q + 1])
    A = shard.tile_slice("i64", rowptr, colind, values, r0, r1, c0, c1)
    nz = int(A.s.nnz)
    rp = np.ctypeslib.as_array(A.s.rowptr, (r1 - r0 + 1,)).copy()
    ci = np.ctypeslib.as_array(A.s.colind, (nz,)).copy() if nz else np.zeros(0, np.uint32)
    va = np.ctypeslib.as_array(A.s.values, (nz,)).copy() if nz else np.zeros(0, np.int64)
    local_ok = bool(nz == 0 or int(ci.max()) < c1 - c0)
    part_y = csr_mul(rp, ci, va, x[c0:c1])  # only this rank's x segment
    w, a, b = shard.y_split(r1 - r0, Q, q)
    part = torch.zeros(Q * w, dtype=torch.int64)
    part[: r1 - r0] = torch.from_numpy(part_y)
    groups = shard.row_block_groups(P, Q)
    ys = shard.reduce_partial(part, Q, q, r1 - r0, groups[p])
    out[rank] = (r0 + a, r0 + b, ys.tolist(), nz, local_ok)
    dist.destroy_process_group()


@pytest.mark.parametrize("grid", [(1, 2), (2, 1), (2, 2)])
def test_grid_tiles_reduce_scatter_to_the_product(grid):
    world = grid[0] * grid[1]
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, grid, port, out), nprocs=world, join=True)
        res = dict(out)
    n, rowptr, colind, values, x = matrix(seed=2, n=2501)
    want = csr_mul(rowptr, colind, values, x)
    y = np.full(n, -(1 << 62), dtype=np.int64)
    for r in range(world):
        y0, y1, ys, _, local_ok = res[r]
        assert local_ok, "tile column indices are not local to the segment"
        assert len(ys) == y1 - y0
        y[y0:y1] = ys
    assert sum(res[r][3] for r in range(world)) == int(rowptr[-1])  # the tiles hold every nonzero once
    assert np.array_equal(y, want)


def test_col_bounds_and_y_split():
    sys.path.insert(0, str(ROOT))
    from sparsep_b200 import shard

    for ncols, parts in ((10, 3), (7, 7), (5, 8), (1_000_003, 4)):
        b = shard.col_bounds(ncols, parts)
        assert b[0] == 0 and b[-1] == ncols and len(b) == parts + 1 and np.all(np.diff(b) >= 0)
        assert np.diff(b).max() - np.diff(b).min() <= 1
    for rows, Q in ((7, 3), (0, 2), (1, 4), (12, 4)):
        pieces = [shard.y_split(rows, Q, q) for q in range(Q)]
        assert all(p[0] == pieces[0][0] for p in pieces)
        assert pieces[0][1] == 0 and pieces[-1][2] == rows
        assert all(pieces[q][2] == pieces[q + 1][1] for q in range(Q - 1))
