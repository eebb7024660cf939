"""Independent replicas on several GPUs (one process per GPU, launched by torchrun).

Seed extensions do not exchange data: each rank extends its own shard of jobs and only
the timing crosses ranks -- a barrier around the timed region and the maximum of the
ranks' step times, so the whole-job rate is all ranks' jobs over the slowest rank.
"""
from __future__ import annotations

import os


def dist_env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_seed(base: int, rank: int) -> int:
    """Generator seed of a rank's shard: disjoint synthetic batches per rank."""
    return base + 1000 * rank


def max_over_ranks(value: float, device=None) -> float:
    """The largest of the ranks' values (identity on one rank)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(jobs_per_rank: int, step_ms: float, device=None) -> tuple[float, float]:
    """(all ranks' jobs per second over the slowest rank's step time, that step time)."""
    import torch.distributed as dist
    ws = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    slowest = max_over_ranks(step_ms, device)
    return jobs_per_rank * ws / (slowest * 1e-3), slowest
