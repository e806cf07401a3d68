"""Multi-GPU plumbing for the batched KEM path: instance sharding and max-over-ranks timing.

KEM instances are independent, so N GPUs run N replicas, each on its own contiguous range
of instance indices (weak scaling: the per-GPU batch is fixed); there is no data-path
collective.  torch.distributed (NCCL on GPUs, gloo on CPU) carries only barriers and the
max-over-ranks reduction of the timed region.
"""
from __future__ import annotations

import datetime
import os


def env() -> tuple[int, int, int]:
    """(world_size, rank, local_rank) from the torchrun environment (1, 0, 0 when absent)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(per_rank: int, rank: int) -> tuple[int, int]:
    """Instance index range [first, first + per_rank) of `rank` under weak scaling."""
    return rank * per_rank, per_rank


def init(backend: str, timeout_s: float = 120.0, device=None):
    import torch.distributed as dist

    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return dist


def max_over_ranks(value: float, device="cpu") -> float:
    """The maximum of a per-rank value (e.g. elapsed milliseconds) over all ranks."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    x = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(x, op=dist.ReduceOp.MAX)
    return float(x.item())
