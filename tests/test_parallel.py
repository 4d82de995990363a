"""Multi-rank host logic on CPU (gloo, world_size 2): the ensemble sharding
(msg123_b200.parallel) and bench.py's cross-rank reductions.  The GPU work of each rank is
replaced by a deterministic stand-in; the assignment, the gather and the aggregate are
what is tested."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from msg123_b200 import parallel


def test_assign_every_member_once_and_balanced():
    work = parallel.member_work(range(64))
    for world in (1, 2, 3, 4, 8):
        parts, load = parallel.assign(work, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(64))
        assert max(load) - min(load) <= max(work) + 1e-9
        assert parallel.assign(work, world) == (parts, load)     # same answer on every rank
    with pytest.raises(ValueError):
        parallel.assign(work, 0)


def fake_runner(seeds, nsteps):
    stats = []
    for s in seeds:
        (nx, ny, nz), sigma = parallel.member_draw(s)
        stats.append({"seed": s, "accepted": nsteps, "newton_total": nsteps * (3 + s % 4), "cells": nx * ny * nz})
    return stats, 0.01 * len(seeds)


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out = parallel.run(12, 3, rank=rank, world_size=world, dist=dist, runner=fake_runner)
        import bench
        tmax = bench.reduce(dist, 1.5 + rank, "max")
        tsum = bench.reduce(dist, 1.5 + rank, "sum")
        q.put((rank, out, tmax, tsum))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_shard_and_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict()
    for _ in procs:
        rank, out, tmax, tsum = q.get(timeout=120)
        res[rank] = (out, tmax, tsum)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    o0, o1 = res[0][0], res[1][0]
    assert o0["parts"] == o1["parts"] and o0["stats"] == o1["stats"]
    assert [s["seed"] for s in o0["stats"]] == list(range(12))
    assert all(s["accepted"] == 3 for s in o0["stats"])
    expected = sum(s["cells"] * 3 for s in o0["stats"]) / max(0.01 * len(p) for p in o0["parts"])
    assert o0["throughput"] == pytest.approx(expected)
    assert res[0][1] == res[1][1] == 2.5 and res[0][2] == res[1][2] == 4.0


def _failing_runner(seeds, nsteps):
    import torch.distributed as dist
    if dist.get_rank() == 1:
        raise ValueError("member build failed")
    return fake_runner(seeds, nsteps)


def _failing_worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        parallel.run(8, 2, rank=rank, world_size=world, dist=dist, runner=_failing_runner)
        q.put((rank, None))
    except RuntimeError as e:
        q.put((rank, str(e)))
    finally:
        dist.destroy_process_group()


def test_gloo_rank_failure_reaches_every_rank():
    """Rank 1 raises while building its members: both ranks end with the same error, well
    inside the process group's timeout (no rank waits in the gather for the failed one)."""
    import time
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    t0 = time.time()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert time.time() - t0 < 50
    assert res[0] == res[1] and "rank 1: ValueError: member build failed" in res[0]
