"""Multi-GPU runs are replicas only: each rank solves its own copy of the
workload and nothing crosses ranks on the data path; the only collectives are
barriers and the max over ranks of the device time.  This checks that host
protocol with two gloo ranks on the CPU (127.0.0.1)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    try:
        dist.barrier()
        mine = 10.0 + 5.0 * rank          # rank 1 is the slowest replica
        slowest = bench.max_over_ranks(mine, dist)
        # value = world * units / slowest time, as bench.py reports it
        out[rank] = (slowest, world * 1000.0 / slowest)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replicas_take_the_slowest_rank():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    assert res[0][0] == 15.0 and abs(res[0][1] - 2000.0 / 15.0) < 1e-9


def test_single_process_needs_no_collective():
    import bench
    assert bench.max_over_ranks(12.5, None) == 12.5
