"""1D row-sharded SpMV over several GPUs (one process per GPU).

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
