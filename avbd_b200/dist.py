"""Multi-process plumbing for batched runs: one process per GPU.

Scenes are independent, so a multi-GPU run shards them across ranks with no
data-path collective.  The default split is strong scaling: one batch is
partitioned across the ranks, balanced by tetrahedra (`partition_scenes`);
weak scaling (every rank advances its own batch of the same size, drawn with
a rank-specific seed, `shard_seed`) remains an option.  torch.distributed is
used only for start/stop barriers and the max/sum reductions of timings and
counters.
"""
from __future__ import annotations

import datetime
import os


def env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def init(backend: str, timeout_s: int = 300):
    rank, world, local = env()
    if world <= 1:
        return rank, world, local
    import torch.distributed as dist
    if not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        kw = {}
        if backend == "nccl":
            import torch
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return rank, world, local


def active() -> bool:
    try:
        import torch.distributed as dist
        return dist.is_available() and dist.is_initialized()
    except ImportError:
        return False


def barrier(timeout_s: float | None = None):
    """Barrier over all ranks.  With `timeout_s` on a gloo group it is a
    monitored barrier: a rank that left (or never arrives) raises a
    RuntimeError naming it on rank 0 after `timeout_s`, instead of a hang."""
    if active():
        import torch.distributed as dist
        if timeout_s is not None and dist.get_backend() == "gloo":
            dist.monitored_barrier(timeout=datetime.timedelta(seconds=timeout_s))
        else:
            dist.barrier()


def reduce(values, op: str = "max", device=None):
    """Element-wise max (or sum) of a list of floats over all ranks."""
    if not active():
        return list(values)
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return t.cpu().tolist()


def partition_scenes(costs, world: int) -> list[list[int]]:
    """Splits scenes of the given costs (their tetrahedron counts: the solve
    streams one record per tet-vertex incidence per iteration) into `world`
    sets by longest-processing-time: scenes in descending cost (ties by id)
    each go to the set with the smallest total so far (ties to the lowest
    rank).  Deterministic, so every rank computes the same split alone.
    Returns each rank's scene ids in ascending order."""
    order = sorted(range(len(costs)), key=lambda s: (-costs[s], s))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for s in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(s)
        load[r] += costs[s]
    return [sorted(p) for p in parts]


def batch_partition(num_scenes: int, seed: int, world: int, n_min: int = 4, n_max: int = 24) -> list[list[int]]:
    """`partition_scenes` of the 1024-cube batch (avbd_b200.scenes.batched_cubes):
    each scene's cost is its 6 n^3 tetrahedra."""
    from .scenes import batched_cube_params
    costs = [6 * batched_cube_params(seed, s, n_min, n_max)[0] ** 3 for s in range(num_scenes)]
    return partition_scenes(costs, world)


def shard_seed(seed: int, rank: int) -> int:
    """Seed of the batch a rank advances (distinct scenes on every rank)."""
    return seed + 7919 * rank


def shutdown():
    if active():
        import torch.distributed as dist
        dist.destroy_process_group()
