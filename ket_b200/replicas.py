"""Replica parallelism: one process per GPU, independent work units, no
data-path collective.

The state vector is not sharded (the backend targets one GPU per state).
What parallelises across GPUs without any exchange are independent units --
whole circuits (benchmark replicas), parameter sets of an adjoint batch,
circuits of the planner corpus.  Ranks take disjoint strided shards, work
alone, and meet only for a host-side gather and the max-over-ranks timing.
``torch.distributed`` is the plumbing (NCCL on GPUs, gloo on CPU tests).
"""
from __future__ import annotations

import datetime
import os
from typing import Any, List, Sequence


def env_rank_world():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def init(backend: str = "nccl", timeout_s: int = 300):
    """Join the process group named by the torchrun environment (127.0.0.1)."""
    import torch.distributed as dist
    rank, world, local = env_rank_world()
    if world > 1 and not dist.is_initialized():
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def shard(items: Sequence[Any], rank: int, world: int) -> List[Any]:
    """Disjoint strided shard: every item goes to exactly one rank."""
    return list(items[rank::world])


def unshard(shards: Sequence[Sequence[Any]]) -> List[Any]:
    """Inverse of `shard` given every rank's shard in rank order."""
    world = len(shards)
    out: List[Any] = []
    longest = max((len(s) for s in shards), default=0)
    for i in range(longest):
        for r in range(world):
            if i < len(shards[r]):
                out.append(shards[r][i])
    return out


def max_over_ranks(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather(obj: Any) -> List[Any]:
    """Every rank's object, in rank order (host-side, after the work)."""
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return [obj]
    out: List[Any] = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
