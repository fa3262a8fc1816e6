"""Replica bookkeeping for runs with one process per GPU.

The batched search path does not shard: each rank holds a full replica of the
tree and searches its own query batch, as the reference's multi-GPU mode does
(open-harmonia/src/full-multi-prefix-sort-8thread.cu:333-371).  The only
cross-rank step is timing: the job's time is the slowest rank's, and the job
value is all ranks' queries over that time.
"""
from __future__ import annotations


def query_seed(base: int, rank: int) -> int:
    """Each replica searches its own batch."""
    return base + 1000 * rank


def max_over_ranks(value: float, device=None) -> float:
    """MAX of `value` over the default process group (identity when alone)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    if device is None and dist.get_backend() == "nccl":
        device = torch.device("cuda", torch.cuda.current_device())
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(queries_per_rank: int, world_size: int, ms_per_step_max: float) -> float:
    """Whole-job Mqueries/s: every rank's queries over the slowest rank's time."""
    return world_size * queries_per_rank / ms_per_step_max / 1e3
