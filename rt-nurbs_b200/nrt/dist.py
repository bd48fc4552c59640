"""Multi-GPU plumbing of the benchmark: one process per GPU, torch.distributed
for the host-side barrier and the max-over-ranks time.

The intersection path shards by rays: every rank traces its own batch (its
own camera jitter seed) against its own copy of the read-only scene, with no
collective on the data path (weak scaling).  The only collectives are the
barrier around the timed region and the all-reduce (max) of the elapsed time.
"""
from __future__ import annotations

import os
from datetime import timedelta


def env_ranks():
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0):
    """Joins the process group when WORLD_SIZE > 1; returns (rank, world, local)."""
    import torch.distributed as dist

    rank, world, local = env_ranks()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return rank, world, local


def barrier():
    import torch.distributed as dist

    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def max_over_ranks(value: float, device="cpu") -> float:
    """The largest value over all ranks (every rank gets it)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_initialized() and dist.get_world_size() > 1):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seed(base: int, rank: int) -> int:
    """Jitter seed of a rank's ray batch: distinct per rank, reproducible."""
    return int(base) + int(rank)


def weak_scaling_rate(units_per_rank: float, world: int, max_seconds: float) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return units_per_rank * world / max_seconds


def finalize():
    import torch.distributed as dist

    if dist.is_initialized():
        dist.destroy_process_group()
