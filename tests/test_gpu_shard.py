"""The row-sharded SpMV on the GPU with one rank (NCCL, world size 1): the
plan of the rank's row slice after the all-gather of x gives the oracle's y
(INT32 bit for bit).  The multi-rank logic runs in tests/test_shard_ranks.py
(gloo, world size 2); this run has a single GPU."""
import datetime
import os
import socket

import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi, shard
from helpers import oracle_spmv, random_triplets, random_x

pytestmark = pytest.mark.gpu


def test_one_rank_sharded_spmv():
    import torch
    import torch.distributed as dist

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(4)
        n = 5000
        r, c, v = random_triplets(rng, n, n, 0.003, "i32", long_row=3)
        x = random_x(rng, n, "i32")
        rp, ci, vv = sp.synth.to_csr(n, r, c, v)
        S = shard.ShardedCSR("i32", n, rp, ci, vv, rank=0, world=1)
        xs = torch.from_numpy(x).cuda()
        ys = torch.zeros(S.r1 - S.r0, dtype=torch.int32, device="cuda")
        S.spmv(xs, ys)
        torch.cuda.synchronize()
        A = sp.csr("i32", n, n, rp, ci, vv)
        assert np.array_equal(ys.cpu().numpy(), oracle_spmv(A, x))
        S.free()
    finally:
        dist.destroy_process_group()


def test_grid_tiles_on_the_gpu_sum_to_the_product():
    """The plans of every tile of a 3 x 4 grid (local column indices, each
    multiplied with its own x segment on the GPU), summed per row block on the
    host, give the oracle's y (INT32 bit for bit): the per-rank part of the 2D
    scheme, without the collective."""
    import torch

    rng = np.random.default_rng(5)
    n = 6000
    r, c, v = random_triplets(rng, n, n, 0.002, "i32", long_row=2)
    x = random_x(rng, n, "i32")
    rp, ci, vv = sp.synth.to_csr(n, r, c, v)
    P, Q = 3, 4
    rb, cb = shard.row_bounds(rp, n, P), shard.col_bounds(n, Q)
    y = np.zeros(n, dtype=np.int64)
    for p in range(P):
        for q in range(Q):
            r0, r1, c0, c1 = int(rb[p]), int(rb[p + 1]), int(cb[q]), int(cb[q + 1])
            T = shard.tile_slice("i32", rp, ci, vv, r0, r1, c0, c1)
            plan = capi.Plan(T, None)
            xs = torch.from_numpy(x[c0:c1].copy()).cuda()
            ys = torch.zeros(r1 - r0, dtype=torch.int32, device="cuda")
            plan.run_device(xs.data_ptr(), ys.data_ptr(), torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            y[r0:r1] += ys.cpu().numpy().astype(np.int64)
            plan.free()
    A = sp.csr("i32", n, n, rp, ci, vv)
    want = oracle_spmv(A, x).astype(np.int64)
    assert np.array_equal(((y + (1 << 31)) % (1 << 32) - (1 << 31)), want)


def test_one_rank_tile_sharded_spmv():
    """ShardedCSR2D end to end with NCCL on one GPU (grid 1 x 1: the tile is
    the whole matrix, the reduce-scatter a group of one)."""
    import torch
    import torch.distributed as dist

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(6)
        n = 4000
        r, c, v = random_triplets(rng, n, n, 0.003, "f32", long_row=2)
        x = random_x(rng, n, "f32")
        rp, ci, vv = sp.synth.to_csr(n, r, c, v)
        S = shard.ShardedCSR2D("f32", n, rp, ci, vv, rank=0, world=1, grid=(1, 1))
        xs = torch.from_numpy(x[S.c0:S.c1].copy()).cuda()
        ys = torch.zeros(S.y1 - S.y0, dtype=torch.float32, device="cuda")
        S.spmv(xs, ys)
        torch.cuda.synchronize()
        A = sp.csr("f32", n, n, rp, ci, vv)
        P = capi.Plan(A, None)
        yd = torch.zeros(n, dtype=torch.float32, device="cuda")
        P.run_device(torch.from_numpy(x).cuda().data_ptr(), yd.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert np.array_equal(ys.cpu().numpy(), yd.cpu().numpy())  # the same tile, the same plan
        S.free()
        P.free()
    finally:
        dist.destroy_process_group()
