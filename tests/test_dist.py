"""CPU test of the replica plumbing of bench.py --gpus N (world size 2, gloo):
each rank builds its own replica of the workload (a different seed), the
barrier completes, and the step time is the maximum over ranks. The path has
no data-path collective (replicas only); this is all the N > 1 host logic."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(
        RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
        TMNB_DIST_BACKEND="gloo",
    )
    import torch.distributed as dist

    import bench

    w, r, _ = bench.dist_setup()
    assert (w, r) == (world, rank)
    bench.barrier(w)
    t = bench.max_over_ranks(1.0 + rank, w)
    from timemachine_b200 import testsystems

    s = testsystems.build_system(30, 1.0, seed=bench.SEED + r)
    out[rank] = (t, float(s.x.sum()))
    bench.barrier(w)
    dist.destroy_process_group()


def test_two_ranks_max_over_ranks_and_own_replicas():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert res[0][0] == res[1][0] == pytest.approx(2.0)
    assert res[0][1] != res[1][1]  # each rank its own replica
