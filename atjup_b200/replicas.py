"""Replica bookkeeping for `bench.py --gpus N`: the path does not shard (every GPU runs an
independent model), so ranks only agree on a barrier and on the slowest rank's time."""
from __future__ import annotations


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks of the default process group (the value itself
    when no group is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_seconds_per_step(max_seconds: float, steps: int, world: int) -> float:
    """Seconds per step of the whole job: world replicas each ran `steps` steps in max_seconds."""
    return max_seconds / (steps * world)
