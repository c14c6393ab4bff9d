"""The multi-GPU path is replicas (one independent copy of the workload per
rank): bench.py's rank combination, run as two gloo ranks on the CPU."""
import os
import socket
import sys

import torch.multiprocessing as mp

from conftest import REPO


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, REPO)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    local_ms = [40.0, 55.0][rank]  # rank 1 is the slow one
    r = bench.combine_ranks(local_ms, cells=1000, steps=10, world=world, dist=dist)
    out[rank] = (r["ms"], r["value"])
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    for rank in range(world):
        ms, value = res[rank]
        assert ms == 55.0
        assert abs(value - world * 1000 * 10 / 0.055) < 1e-6


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, REPO)
    import bench

    r = bench.combine_ranks(20.0, cells=500, steps=4, world=1)
    assert r["ms"] == 20.0 and abs(r["value"] - 500 * 4 / 0.02) < 1e-9
