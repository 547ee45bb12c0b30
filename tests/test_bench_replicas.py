"""Multi-GPU runs of the bench are independent replicas (the path has no exchange step): every timed
quantity is the slowest rank's, reduced over the process group, and the whole-job rate is the units of
all ranks over that time.  Two gloo ranks on the CPU run the same reduction the bench runs over NCCL."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t = 1.0 + 0.5 * rank  # rank 1 is the slow one
    out[rank] = bench.reduce_max(t, dist)
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_and_sum_the_units():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert dict(out) == {0: 1.5, 1: 1.5}
    assert bench.replica_rate(world, 5, 1.5) == pytest.approx(10 / 1.5)
    assert bench.reduce_max(2.5) == 2.5  # no process group: the rank's own time
