"""Multi-rank host logic of bench.py on the CPU (gloo, two ranks): the job's
time is the slowest rank's, and clip-parallel throughput is weak-scaled."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    r, w, l = bench.dist_env()
    assert (r, w, l) == (rank, world, rank)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        local = [10.0 + rank, 5.0 - rank]            # rank 1 is slower in the first timing
        got = bench.reduce_max(local, "cpu", world)
        out[rank] = got
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_reduce_max_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1] == [11.0, 5.0]


def test_weak_value_and_single_rank():
    import bench
    assert bench.reduce_max([3.0, 4.0], "cpu", 1) == [3.0, 4.0]
    # 4.096e7 voxels per rank, 2 ranks, 10 steps in 20 ms
    assert bench.weak_value(40960000, 2, 10, 20.0) == pytest.approx(40960000 * 2 * 10 / 0.02)
