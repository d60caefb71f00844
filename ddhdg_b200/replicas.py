"""Replicas across GPUs of one node (one process per GPU).

The hot path is per cell and per device, so N GPUs run N independent diodes:
there is no collective on the data path.  What crosses ranks is timing only:
a barrier before each timed region and the maximum of the ranks' times after
it, so that the whole-job throughput is the units of all ranks over the
slowest rank's time.  Works with any torch.distributed backend (NCCL on the
GPUs, gloo on the CPU)."""

from __future__ import annotations


def world_size() -> int:
    import torch.distributed as dist

    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def barrier() -> None:
    import torch.distributed as dist

    if world_size() > 1:
        dist.barrier()


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of a per-rank number over all ranks (every rank gets it).
    `device` must be a CUDA device under NCCL, the CPU under gloo."""
    import torch
    import torch.distributed as dist

    if world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, slowest_ms: float) -> float:
    """Units per second of the whole job: every rank did `units_per_rank`,
    the job took the slowest rank's time."""
    return world_size() * units_per_rank / (slowest_ms * 1e-3)
