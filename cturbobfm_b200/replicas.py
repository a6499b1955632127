"""Replica bookkeeping for runs on several GPUs of one node.

Operating points do not exchange data, so N GPUs run N independent
replicas ("replicas only"): no collective touches the data path. The only
collective is the reduction of each rank's device-timed duration to its
maximum, so that a whole-job rate is the work of all ranks over the slowest
rank's time."""

from __future__ import annotations


def max_over_ranks(ms: float, device=None) -> float:
    """The maximum of `ms` over all ranks of the default process group (the
    value itself without one). NCCL groups need `device` (a CUDA device)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(ms)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, ms_max: float) -> float:
    """Units per second of the whole job: every rank processed
    `units_per_rank` units in at most `ms_max` milliseconds."""
    if ms_max <= 0:
        raise ValueError("duration must be positive")
    return world * units_per_rank / (ms_max / 1e3)
