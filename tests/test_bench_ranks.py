"""The multi-rank bench path on CPU (gloo, world size 2): each replica's time
reduces to the slowest rank's, and the whole-job value counts every rank's
bytes over that time."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    slow = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")  # rank 1 is the slow one
    dist.barrier()
    out[rank] = (slow, bench.whole_job_gbs(1000, 4, slow, world))
    dist.destroy_process_group()


def test_two_ranks_max_and_whole_job_value():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0
    # 2 ranks x 1000 B x 4 steps over 15 ms
    assert res[0][1] == pytest.approx(2 * 1000 * 4 / 15e-3 / 1e9)


def test_single_rank_passthrough():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.whole_job_gbs(2e9, 10, 1000.0, 1) == pytest.approx(20.0)
