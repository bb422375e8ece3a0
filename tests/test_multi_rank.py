"""The N > 1 path of bench.py on CPU: two gloo ranks (127.0.0.1), max-over-ranks timing, the
mesh sharding of the batch leg (no data-path collective: each rank fits its own meshes) and
the batch report's whole-job totals, and the launcher that starts one process per GPU."""
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
        # the batch leg's path: the uneven 256-mesh mix's face counts sharded, this rank's share
        # "fitted" (unknowns stand-in: faces / 2), the report reduced over the ranks
        from its_b200 import meshes
        faces = meshes.batch_face_counts(256, 3)
        mine = bench.batch_shard(faces, world, rank)
        local = {"plain_ms": 100.0 + rank, "learned_ms": 2.0 - rank, "meshes": len(mine),
                 "unknowns": sum(faces[i] // 2 for i in mine), "max_rel_residual": 1e-15 * (rank + 1)}
        tot = bench.batch_totals(local, dist, device="cpu")
        dist.barrier()
        q.put((rank, t, parts, mine, tot))
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
    from its_b200 import meshes
    faces = meshes.batch_face_counts(256, 3)
    shards = [r[3] for r in res]
    assert sorted(shards[0] + shards[1]) == list(range(256)) and not set(shards[0]) & set(shards[1])
    lf = [sum(faces[i] for i in sh) for sh in shards]
    assert abs(lf[0] - lf[1]) <= max(faces)  # LPT: loads within one mesh of each other
    for r in res:  # every rank holds the same whole-job totals
        tot = r[4]
        assert tot["plain_ms"] == 101.0 and tot["learned_ms"] == 2.0 and tot["meshes"] == 256
        assert tot["unknowns"] == sum(f // 2 for f in faces) and tot["max_rel_residual"] == 2e-15


def test_launcher_starts_one_process_per_rank(tmp_path, monkeypatch):
    # bench.py --gpus N outside torchrun re-runs itself under torch.distributed.run with N
    # processes on 127.0.0.1; the command line is checked without starting anything
    import bench
    seen = {}

    class Done:
        returncode = 0

    def fake_run(cmd, *a, **k):
        seen["cmd"] = cmd
        return Done()

    monkeypatch.setattr(bench.subprocess, "run", fake_run)
    assert bench.launch_ranks(["--gpus", "4", "--steps", "2"], 4) == 0
    cmd = seen["cmd"]
    assert cmd[1:3] == ["-m", "torch.distributed.run"] and "--nproc-per-node=4" in cmd
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-3:] == ["--gpus", "4", "--steps", "2"][-3:] and cmd[-5].endswith("bench.py")


def test_lpt_shard_single_rank_and_empty():
    import bench
    assert bench.lpt_shard([3, 1, 2], 1) == [[0, 1, 2]]
    assert bench.lpt_shard([], 3) == [[], [], []]
