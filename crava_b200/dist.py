"""Rank plumbing for several GPUs of one node (one process per GPU).

The inversion hot path shards by independent units -- posterior units of
different cases or time-lapse vintages, and posterior realisations -- so
ranks running independent units exchange nothing on the data path: the
only collectives are the barrier around a timed region and the
max-over-ranks of its duration.  One grid too large for a GPU is split
over the ranks by dist_grid.py, whose exchange is the one data-path
communication.
"""
from __future__ import annotations

import datetime
import os


def rank_env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 300):
    """Initialises the default process group when world_size > 1; returns
    the torch.distributed module or None for a single process."""
    rank, world, local = rank_env()
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist

    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, x: float, device=None) -> float:
    """Maximum of x over all ranks (identity for a single process)."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(items, rank: int, world: int):
    """Round-robin share of independent work items for one rank."""
    return [it for i, it in enumerate(items) if i % world == rank]
