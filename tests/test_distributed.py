"""Multi-process host logic of the benchmark on CPU (gloo, world size 2).

The path does not shard: N GPUs run N replicas and the timed region is
reported as the slowest rank's.  These tests check that aggregation across
real process-group ranks (no GPU involved)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r "took" 1 + r seconds for its steps and 10 - r for e2e
        dev, e2e = bench.max_over_ranks([1.0 + rank, 10.0 - rank], dist)
        q.put((rank, dev, e2e, bench.aggregate_rate(50, dev, world)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_and_aggregate_with_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs)
    results = sorted(q.get(timeout=5) for _ in range(world))
    for rank, dev, e2e, rate in results:
        assert dev == 2.0 and e2e == 10.0      # slowest rank on every rank
        assert rate == pytest.approx(2 * 50 / 2.0)


def test_single_process_passthrough():
    assert bench.max_over_ranks([3.0, 4.0], None) == [3.0, 4.0]
    assert bench.aggregate_rate(10, 2.0, 1) == 5.0
