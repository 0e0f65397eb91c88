"""Independent scenes across ranks (one process per GPU).

SPH2O runs one scene per process and has no distributed path. A single
scene here does not shard (one GPU, no inter-GPU traffic); batches of
independent scenes do: each rank steps its own subset as one batch, and no
collective touches the particle data. The assignment is a greedy
longest-processing-time bin packing on a per-scene cost (fluid particles x
expected solver iterations), computed identically on every rank from the
same scene list, so it needs no communication; only the per-scene
statistics (a few numbers per scene) are gathered to rank 0 afterwards.
"""
from __future__ import annotations

import heapq


def scene_cost(fluid_particles: int, iterations: float = 1.0) -> float:
    """Work of one scene per step: its particle passes scale with the fluid
    particle count times the passes per step (solver iterations + fixed)."""
    return float(fluid_particles) * (2.0 + 2.0 * float(iterations))


def partition_scenes(costs, world: int):
    """Scenes (by index) per rank: heaviest first, each to the currently
    lightest rank (ties: lower scene index first, lower rank first). Every
    rank computes the same answer from the same costs."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda s: (-float(costs[s]), s))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for s in order:
        load, r = heapq.heappop(heap)
        parts[r].append(s)
        heapq.heappush(heap, (load + float(costs[s]), r))
    return [sorted(p) for p in parts]


def shard_for_rank(costs, world: int, rank: int):
    """The scene indices rank `rank` steps."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return partition_scenes(costs, world)[rank]


def gather_scene_stats(local: dict, world: int, group=None):
    """Merge {scene index: stats} from every rank on every rank (host
    objects through torch.distributed; gloo on CPU, nccl on GPUs)."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist

    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    merged = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError(f"scene {k} stepped by two ranks")
            merged[k] = v
    return merged
