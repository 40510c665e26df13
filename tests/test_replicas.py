"""bench.py --gpus N runs N independent replicas (no data-path collective):
each rank its own seeded stack, the step time the max over ranks, the job's
throughput every rank's pixel-frames over that time. The rank logic runs here
as two gloo processes on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 100.0 + 50.0 * rank  # rank 1 is the slower one
        ms = bench.max_over_ranks(local_ms, dist, "cpu")
        q.put((rank, bench.replica_seed(rank), ms, bench.job_throughput(world, 4543.0, ms)))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert len({r[1] for r in res}) == world  # each replica its own stack
    assert all(r[2] == 150.0 for r in res)  # every rank reports the slowest rank's time
    assert all(r[3] == pytest.approx(2 * 4543.0 / 0.150) for r in res)


def test_one_rank_needs_no_process_group():
    assert bench.max_over_ranks(12.5) == 12.5
    assert bench.job_throughput(1, 4543.0, 1000.0) == pytest.approx(4543.0)
