"""Replica bookkeeping for multi-GPU runs.

The SPH step has no exchange between independent scenes, so N GPUs run N
replicas (weak scaling) with no collective on the data path.  The only
collectives are the barriers around the timed region and one max-reduction
of the measured time, taken in the same order on every rank.
"""
from __future__ import annotations


def world_info():
    import os
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def barrier(dist):
    if dist is not None and dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def max_over_ranks(value: float, dist, device=None) -> float:
    """The max of `value` over all ranks (every rank gets it)."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_value(world: int, units_per_replica: int, steps: int, ms_max: float) -> float:
    """Whole-job units per second when every rank processes its own replica."""
    return world * units_per_replica * steps / (ms_max / 1000.0)
