"""Multi-GPU plumbing on the CPU: two gloo ranks (127.0.0.1) run the benchmark's replica logic --
barrier, max-over-ranks timing, whole-job throughput -- and partition a serving stream by mesh
with no exchange of data (every mesh served by exactly one rank)."""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    from ordito_b200.serving import mesh_for, mesh_key, serving_workload, shard_of

    dist = bench.Dist(backend="gloo")
    try:
        dist.barrier()
        # Each rank times its own replica; the job's time is the slowest rank's.
        ms = 10.0 + rank
        slowest = dist.max(ms)
        value = dist.world * 64 / (slowest / 1e3)
        # A serving stream split by mesh: this rank's share, keyed as the server keys meshes.
        stream = serving_workload(3, 300, rate=100.0, v_min=200, v_max=5000)
        keys = {r.mesh: mesh_key(*mesh_for(r.mesh)) for r in stream}
        mine = [i for i, r in enumerate(stream) if shard_of(keys[r.mesh], world) == rank]
        gathered = [None] * world
        dist.pg.all_gather_object(gathered, mine)
        out.put((rank, slowest, value, gathered, dist.world))
    finally:
        dist.close()


def test_two_gloo_replicas() -> None:
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = [out.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, value, gathered, w in results:
        assert w == world
        assert slowest == 11.0  # max over ranks
        assert value == pytest.approx(world * 64 / 0.011)
        shares = [set(g) for g in gathered]
        assert not (shares[0] & shares[1])  # disjoint
        assert shares[0] | shares[1] == set(range(300))  # complete
        assert shares[0] and shares[1]  # both ranks get work
