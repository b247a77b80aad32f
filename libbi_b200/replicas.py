"""Multi-GPU use of the filter step: replicas.  A single filter does not
shard on this path (the Lorenz-96 workload fits one GPU many times over), so
N GPUs run N independent filters, one process per GPU, each with its own
seed; there is no exchange on the data path.  The only collective is the
reduction of the timings: a run's time is the slowest rank's, and the
whole-job rate counts every rank's particle-steps against it."""
from __future__ import annotations


def replica_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s filter: streams that never meet (the draws are
    counter-based functions of the seed)."""
    return int(base) + 1000 * int(rank)


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The largest `value` over all ranks (every rank receives it); the
    identity without a process group.  device: where the reduction tensor
    lives ("cuda" for NCCL, "cpu" for gloo)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, seconds: float) -> float:
    """Units of all ranks per second of the slowest rank."""
    return float(units_per_rank) * int(world) / float(seconds)
