"""The N > 1 path of bench.py on CPU: two gloo ranks (127.0.0.1), max-over-ranks timing and
the mesh sharding used when independent meshes are spread over GPUs (no data-path
collective: each rank fits its own meshes)."""
import datetime
import multiprocessing as mp
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        t = bench.max_over_ranks(10.0 + 3 * rank, dist, device="cpu")
        parts = bench.lpt_shard([5, 1, 4, 2, 8, 3, 7, 6], world)
        dist.barrier()
        q.put((rank, t, parts))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_timing_and_sharding():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[1] for r in res] == [13.0, 13.0]  # both ranks see the max
    parts = res[0][2]
    assert parts == res[1][2]
    assert sorted(parts[0] + parts[1]) == list(range(8)) and not set(parts[0]) & set(parts[1])
    loads = [sum([5, 1, 4, 2, 8, 3, 7, 6][i] for i in p) for p in parts]
    assert abs(loads[0] - loads[1]) <= 1


def test_lpt_shard_single_rank_and_empty():
    import bench
    assert bench.lpt_shard([3, 1, 2], 1) == [[0, 1, 2]]
    assert bench.lpt_shard([], 3) == [[], [], []]
