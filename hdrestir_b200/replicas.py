"""Replica bookkeeping for multi-GPU runs.

Frames and render jobs are independent (the reference renders one job per
delegate with no cross-frame exchange beyond its own persistent buffers), so N
GPUs run N independent replicas with no data-path collective. The only
collectives are the timing ones: a barrier around the timed region and a MAX
over ranks of each rank's device-timed duration. The whole-job rate is the
units all ranks processed divided by that maximum.
"""
from __future__ import annotations

import os


def dist_env() -> tuple[int, int, int]:
    """(rank, local_rank, world_size) from the torchrun environment (1 process when unset)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """MAX of a per-rank duration over all ranks (identity for one rank)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, max_ms: float) -> float:
    """Units per second of the whole job: every rank processed units_per_rank in at most max_ms."""
    if max_ms <= 0.0:
        raise ValueError("duration must be positive")
    return world * units_per_rank / (max_ms / 1000.0)


def barrier(world: int, cuda: bool = True) -> None:
    """Device idle on this rank, then all ranks, then device idle again."""
    if cuda:
        import torch
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if cuda:
        import torch
        torch.cuda.synchronize()
