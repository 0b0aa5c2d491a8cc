"""Multi-process plumbing for batched runs: one process per GPU.

Scenes are independent, so a multi-GPU run shards them across ranks with no
data-path collective (weak scaling: every rank advances its own batch of the
same size).  torch.distributed is used only for start/stop barriers and the
max-over-ranks reduction of timings and counters.
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


def shard_seed(seed: int, rank: int) -> int:
    """Seed of the batch a rank advances (distinct scenes on every rank)."""
    return seed + 7919 * rank


def shutdown():
    if active():
        import torch.distributed as dist
        dist.destroy_process_group()
