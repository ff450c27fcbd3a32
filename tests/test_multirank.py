"""Multi-rank host logic on CPU (gloo, world size 2): the instance partition
used when a batch is spread over several GPUs, and the max-over-ranks job
time the benchmark reports.  No GPU is touched."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, times, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from tests.conftest import load_package
        load_package()
        from ib_cu_b200 import sharding
        import bench
        mine = sharding.partition(costs, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        job = bench.max_over_ranks(times[rank], world, torch.device("cpu"))
        out.put((rank, gathered, job))
    finally:
        dist.destroy_process_group()


def test_partition_and_job_time_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    from tests.conftest import load_package
    load_package()
    from ib_cu_b200 import sharding
    world = 2
    costs = [((i * 7919) % 97 + 1) * 1000.0 for i in range(37)]
    times = [3.25, 4.5]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, costs, times, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = sharding.partition(costs, world)
    for rank, gathered, job in results:
        assert gathered == expect              # every rank derives the same partition
        assert job == max(times)               # the slowest rank's time
    ids = sorted(i for shard in expect for i in shard)
    assert ids == list(range(len(costs)))      # disjoint and complete
    loads = [sum(costs[i] for i in shard) for shard in expect]
    assert max(loads) - min(loads) <= max(costs)


def test_partition_edge_cases():
    from tests.conftest import load_package
    load_package()
    from ib_cu_b200 import sharding
    assert sharding.partition([], 3) == [[], [], []]
    assert sharding.partition([5.0], 2) == [[0], []]
    assert sharding.partition([1.0, 1.0, 1.0, 1.0], 4) == [[0], [1], [2], [3]]
    with pytest.raises(ValueError):
        sharding.partition([1.0], 0)
