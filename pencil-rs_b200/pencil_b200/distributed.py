"""Multi-process plumbing for several GPUs (one process per GPU).

The virtual ranks of one plan live on one GPU, so a plan needs no inter-GPU
exchange.  Across GPUs, independent units (the grids of a ragged batch, or
whole-field replicas) are split with the reference's floor partition rule
(crates/pencil-array/src/geometry.rs:9-30) and run with no data-path
collective.  Timing is the maximum over ranks.
"""

from __future__ import annotations

from typing import List, Sequence


def shard(count: int, rank: int, world: int) -> range:
    """Units [floor(count*rank/world), floor(count*(rank+1)/world)) of `rank`."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank outside the process group")
    return range(count * rank // world, count * (rank + 1) // world)


def shard_list(items: Sequence, rank: int, world: int) -> List:
    return [items[i] for i in shard(len(items), rank, world)]


def max_over_ranks(value: float, group=None) -> float:
    """Maximum of a per-rank scalar (e.g. device time) over the process group."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_over_ranks(value: float, group=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())
