"""Row-sharded (1D) and tile-sharded (2D) SpMV over several GPUs (one
process per GPU); the 2D grid is described further down.

The reference's 1D scheme partitions rows over NR_DPUS DPUs with
partition_by_nnz (spmv/1D/CSR-row/support/partition.h:35-77, the CSR-nnz
variant) and broadcasts the whole x to every DPU before each SpMV
(spmv/1D/CSR-row/host/app.c:256-262).  Here the parts are GPUs: rank r owns
rows [b_r, b_{r+1}) of a square matrix, a plan of that row slice (all
columns) on its own GPU, and the same slice of x and y.  One SpMV is an
all-gather of the x slices over NCCL (torch.distributed; every slice padded
to the largest, since the collective moves equal-sized pieces) followed by
the local SpMV into the rank's slice of y -- no reduction, since no row is
split between ranks.  The collective runs on the plan's stream ordering: the
gather is enqueued on the current stream and the SpMV after it.

The partition, the slicing and the gather are plain host logic and run on
any backend (the tests use gloo on the CPU with world size 2); the SpMV is
the library's plan.  No TMA or bulk load in this path reads another GPU's
memory: x crosses NVLink only inside the NCCL collective.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi


def row_bounds(rowptr: np.ndarray, nrows: int, parts: int) -> np.ndarray:
    """parts + 1 row boundaries balancing nonzeros, the reference's
    partition_by_nnz at row granularity (sparsep_partition_by_nnz)."""
    rp = np.ascontiguousarray(rowptr[: nrows + 1], dtype=np.uint32)
    split = np.zeros(parts + 2, dtype=np.uint32)
    capi.check(capi.lib().sparsep_partition_by_nnz(rp.ctypes.data_as(C.POINTER(C.c_uint32)), nrows, parts,
                                                    split.ctypes.data_as(C.POINTER(C.c_uint32))),
               "partition_by_nnz")
    return split[: parts + 1].astype(np.int64)


def row_slice(dtype: str, nrows: int, ncols: int, rowptr, colind, values, r0: int, r1: int) -> capi.HostMatrix:
    """Rows [r0, r1) of a CSR matrix as a CSR of r1 - r0 rows over all columns."""
    a, b = int(rowptr[r0]), int(rowptr[r1])
    rp = (np.asarray(rowptr[r0: r1 + 1], dtype=np.int64) - a).astype(np.uint32)
    return capi.csr(dtype, r1 - r0, ncols, rp, np.asarray(colind[a:b]), np.asarray(values[a:b]))


def gather_x(x_slice, bounds: np.ndarray, rank: int, group=None):
    """The whole x on every rank from each rank's slice: an all-gather of the
    slices padded to the largest (torch tensors on the backend's device)."""
    import torch
    import torch.distributed as dist

    world = len(bounds) - 1
    widths = np.diff(bounds)
    wmax = int(widths.max())
    pad = torch.zeros(wmax, dtype=x_slice.dtype, device=x_slice.device)
    pad[: x_slice.numel()] = x_slice
    out = torch.empty(world * wmax, dtype=x_slice.dtype, device=x_slice.device)
    dist.all_gather_into_tensor(out, pad, group=group)
    return torch.cat([out[p * wmax: p * wmax + int(widths[p])] for p in range(world)])


class ShardedCSR:
    """This rank's part of a square CSR matrix sharded by rows over the
    process group: its plan, its rows and the matching slice of x and y."""

    def __init__(self, dtype: str, n: int, rowptr, colind, values, rank: int, world: int,
                 opts: capi.Opts | None = None, group=None):
        self.dtype, self.n, self.rank, self.world, self.group = dtype, n, rank, world, group
        self.bounds = row_bounds(rowptr, n, world)
        self.r0, self.r1 = int(self.bounds[rank]), int(self.bounds[rank + 1])
        self.A = row_slice(dtype, n, n, rowptr, colind, values, self.r0, self.r1)
        self.plan = capi.Plan(self.A, opts)

    def spmv(self, x_slice, y_slice, stream=None):
        """y_slice = rows [r0, r1) of A x, from every rank's x slice (device
        tensors of this rank's GPU); collective: every rank calls it."""
        import torch

        x = gather_x(x_slice, self.bounds, self.rank, self.group)
        s = stream or torch.cuda.current_stream()
        self.plan.run_device(x.data_ptr(), y_slice.data_ptr(), s.cuda_stream)
        return y_slice

    def free(self):
        self.plan.free()


# ---------------------------------------------------------------------------
# 2D tiles over a P x Q grid of ranks
# ---------------------------------------------------------------------------
# The reference's 2D schemes give every DPU one tile of the matrix (a row
# stripe crossed with a column segment), send each DPU only the x segment of
# its tile's columns (spmv/2D/DCSR/host/app.c:308-315) and add the partial y
# of the tiles of one row stripe on the host (spmv/2D/BDCSR/host/app.c:437-447).
# Here rank r = p * Q + q holds the tile of row block p (rows split by nonzeros,
# the reference's partition_by_nnz with P parts) and column segment q (Q
# equal-width segments), planned on its GPU with column indices local to the
# segment.  One SpMV is the tile's SpMV on the rank's x segment into a partial
# row block, then a reduce-scatter (sum) of the partial row blocks over the Q
# ranks of row block p: each of them ends up with its own sub-slice of y.  x
# never crosses between GPUs; the y partials do, once, inside the collective.

def col_bounds(ncols: int, parts: int) -> np.ndarray:
    """parts + 1 column boundaries of equal-width segments."""
    return np.array([ncols * q // parts for q in range(parts + 1)], dtype=np.int64)


def tile_slice(dtype: str, rowptr, colind, values, r0: int, r1: int, c0: int, c1: int) -> capi.HostMatrix:
    """The tile A[r0:r1, c0:c1] as a CSR of r1 - r0 rows over c1 - c0 columns,
    column indices local to the segment (row order and in-row order kept)."""
    a, b = int(rowptr[r0]), int(rowptr[r1])
    ci = np.asarray(colind[a:b]).astype(np.int64)
    keep = (ci >= c0) & (ci < c1)
    rows = np.repeat(np.arange(r1 - r0), np.diff(np.asarray(rowptr[r0: r1 + 1], dtype=np.int64)))
    rp = np.zeros(r1 - r0 + 1, dtype=np.uint32)
    np.cumsum(np.bincount(rows[keep], minlength=r1 - r0), out=rp[1:])
    return capi.csr(dtype, r1 - r0, c1 - c0, rp, (ci[keep] - c0).astype(np.uint32), np.asarray(values[a:b])[keep])


def y_split(block_rows: int, Q: int, q: int) -> tuple[int, int, int]:
    """Reduce-scatter layout of a row block of block_rows rows over Q ranks:
    the padded piece width w and rank q's rows [a, b) inside the block."""
    w = max(1, -(-block_rows // Q))
    return w, min(q * w, block_rows), min((q + 1) * w, block_rows)


def reduce_partial(partial, Q: int, q: int, block_rows: int, group=None):
    """Sum of the Q ranks' partial row blocks (each a tensor of Q * w entries,
    the first block_rows meaningful), scattered: rank q's rows of y."""
    import torch
    import torch.distributed as dist

    w, a, b = y_split(block_rows, Q, q)
    out = torch.empty(w, dtype=partial.dtype, device=partial.device)
    dist.reduce_scatter_tensor(out, partial, group=group)
    return out[: b - a]


def row_block_groups(P: int, Q: int):
    """One process group per row block (ranks p * Q .. p * Q + Q - 1), created
    in the same order on every rank, as torch.distributed requires."""
    import torch.distributed as dist

    return [dist.new_group(list(range(p * Q, p * Q + Q))) for p in range(P)]


class ShardedCSR2D:
    """Rank (p, q) of a P x Q grid over a square CSR matrix: its tile's plan,
    its x segment and its sub-slice of y."""

    def __init__(self, dtype: str, n: int, rowptr, colind, values, rank: int, world: int, grid: tuple[int, int],
                 opts: capi.Opts | None = None):
        P, Q = grid
        if P * Q != world:
            raise ValueError(f"grid {P}x{Q} does not match world size {world}")
        self.dtype, self.n, self.P, self.Q = dtype, n, P, Q
        self.p, self.q = divmod(rank, Q)
        self.rb = row_bounds(rowptr, n, P)
        self.cb = col_bounds(n, Q)
        self.r0, self.r1 = int(self.rb[self.p]), int(self.rb[self.p + 1])
        self.c0, self.c1 = int(self.cb[self.q]), int(self.cb[self.q + 1])
        self.A = tile_slice(dtype, rowptr, colind, values, self.r0, self.r1, self.c0, self.c1)
        self.plan = capi.Plan(self.A, opts)
        self.groups = row_block_groups(P, Q)
        self.w, a, b = y_split(self.r1 - self.r0, Q, self.q)
        self.y0, self.y1 = self.r0 + a, self.r0 + b  # this rank's rows of y

    def spmv(self, x_seg, y_sub, stream=None):
        """y_sub = rows [y0, y1) of A x from this rank's x segment x[c0:c1]
        (device tensors of this rank's GPU); collective over the row block."""
        import torch

        part = torch.zeros(self.Q * self.w, dtype=y_sub.dtype, device=y_sub.device)
        s = stream or torch.cuda.current_stream()
        self.plan.run_device(x_seg.data_ptr(), part.data_ptr(), s.cuda_stream)
        y_sub.copy_(reduce_partial(part, self.Q, self.q, self.r1 - self.r0, self.groups[self.p]))
        return y_sub

    def free(self):
        self.plan.free()
