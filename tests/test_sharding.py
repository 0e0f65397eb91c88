"""Scene sharding across ranks (sph2o_b200/sharding.py) and bench.py's
multi-rank reductions, on the CPU: the partition itself, and world-size-2
gloo process groups that each take their shard of the 256-scene batched
workload, gather per-scene results to every rank, and combine per-rank
timings exactly as bench.py does under torchrun (bench.batch_shard,
bench.combine_batch_results, bench.replica_value, bench.max_over_ranks) --
with the backend's tensors on the host (no GPU, no particle data
exchanged)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from sph2o_b200 import scenes as S
from sph2o_b200.sharding import gather_scene_stats, partition_scenes, scene_cost, shard_for_rank


def workload_costs(count=256):
    params = S.batched_scene_params(count)
    return [scene_cost(p["dims"][0] * p["dims"][1] * p["dims"][2]) for p in params]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_partition_covers_every_scene_once_and_balances(world):
    costs = workload_costs()
    parts = partition_scenes(costs, world)
    flat = sorted(s for p in parts for s in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[s] for s in p) for p in parts]
    # greedy LPT: the heaviest rank exceeds the lightest by at most one scene
    assert max(loads) - min(loads) <= max(costs)
    assert max(loads) <= sum(costs) / world + max(costs)
    for r in range(world):
        assert shard_for_rank(costs, world, r) == parts[r]


def test_partition_is_deterministic_and_validates():
    costs = [5.0, 5.0, 3.0, 1.0]
    # 5 -> rank 0, 5 -> rank 1, 3 -> rank 0 (tie: lower rank), 1 -> rank 1
    assert partition_scenes(costs, 2) == partition_scenes(list(costs), 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        partition_scenes(costs, 0)
    with pytest.raises(ValueError):
        shard_for_rank(costs, 2, 2)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        costs = workload_costs()
        mine = shard_for_rank(costs, world, rank)
        # stand-in for a rank's batch run: per-scene numbers only
        local = {s: {"rank": rank, "fluid_particles": int(costs[s] / 4.0)} for s in mine}
        merged = gather_scene_stats(local, world)
        out.put((rank, sorted(merged), {k: v["rank"] for k, v in merged.items()}, len(mine)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_step_disjoint_shards_and_gather_all():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    costs = workload_costs()
    parts = partition_scenes(costs, world)
    for rank, scenes, owner, n in results:
        assert scenes == list(range(len(costs)))
        assert n == len(parts[rank])
        assert all(owner[s] == r for r in range(world) for s in parts[r])


def bench_rank_main(rank, world, port, out):
    """One rank of bench.py's multi-rank bookkeeping with a fake per-scene
    timing: the rank's shard of the batch, its batched result combined over
    ranks, the replica rate of the single-scene path and the max of e2e
    wall times."""
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        shard = bench.batch_shard(256, world, rank)
        params = S.batched_scene_params(256)
        particles = sum(p["dims"][0] * p["dims"][1] * p["dims"][2] for i, p in enumerate(params) if i in shard)
        ms = 1.0 + 0.01 * particles / 1000.0  # fake: step time grows with the shard's particles
        res = bench.combine_batch_results({"ms_per_step": ms, "fluid_particles": particles, "value": 0.0}, world)
        value, max_ms = bench.replica_value(1_000_000, 20, 30.0 + rank, world)
        wall = bench.max_over_ranks(2.0 + rank, world)
        out.put((rank, shard, particles, ms, res, value, max_ms, wall))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_run_bench_reductions():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=bench_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted((out.get(timeout=180) for _ in range(world)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = [r[1] for r in results]
    assert sorted(s for sh in shards for s in sh) == list(range(256))  # every scene on exactly one rank
    total = sum(r[2] for r in results)
    slowest = max(r[3] for r in results)
    for rank, shard, particles, ms, res, value, max_ms, wall in results:
        # whole-job rate: all ranks' particles over the slowest rank's step time
        assert res["fluid_particles_all_ranks"] == total
        assert res["ms_per_step_max_rank"] == slowest
        assert abs(res["value"] - total / (slowest / 1e3)) <= 1e-9 * res["value"]
        # replicas: world x particles x steps over the slowest rank's device time
        assert max_ms == 31.0
        assert abs(value - 2 * 1_000_000 * 20 / 0.031) <= 1e-6 * value
        assert wall == 3.0
