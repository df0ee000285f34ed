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
