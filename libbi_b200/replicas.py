"""Multi-GPU use of the filter step.

Replicas: a single filter does not shard on this path (the Lorenz-96
workload fits one GPU many times over), so N GPUs run N independent
filters, one process per GPU, each with its own seed; there is no exchange
on the data path.  The only collective is the reduction of the timings: a
run's time is the slowest rank's, and the whole-job rate counts every
rank's particle-steps against it.

Sharded batches: the filters of a batch (PMMH chains, SMC^2 parameter
particles, the batched workload) are independent, so they are partitioned
over the ranks by cost (particles x steps), each rank runs its share as one
local batch, and a single all-gather assembles every filter's results in
filter order.  Every filter is seeded by itself, so the assembled results
equal those of one batch holding all filters, bit for bit."""
from __future__ import annotations

import numpy as np


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


def partition_by_cost(costs, world: int):
    """Filter indices per rank: longest first onto the least-loaded rank
    (ties to the lower rank, then the lower index), so that every rank
    computes the same partition.  Each rank's list is in ascending order."""
    world = int(world)
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def gather_by_filter(parts, rank: int, rows, nfilters: int, dist=None, device: str = "cpu"):
    """The (nfilters, width) array of per-filter rows on every rank, where
    `rows` holds this rank's rows for the filters parts[rank] in that order.
    One all-gather of equally sized (padded) FP64 blocks; without a process
    group the rank's own rows placed in filter order."""
    mine = list(parts[rank])
    rows = np.asarray(rows, np.float64).reshape(len(mine), -1) if mine else np.zeros((0, 0))
    width = rows.shape[1] if mine else None
    if dist is None:
        if len(parts) != 1:
            raise ValueError("several parts need a process group")
        out = np.zeros((nfilters, width if width is not None else 0))
        out[mine] = rows
        return out
    import torch

    # the row width, agreed over all ranks (a rank may hold no filter)
    w = torch.tensor([width if width is not None else -1], dtype=torch.int64, device=device)
    dist.all_reduce(w, op=dist.ReduceOp.MAX)
    width = int(w.item())
    m = max(len(p) for p in parts)
    buf = torch.zeros((max(m, 1), width), dtype=torch.float64, device=device)
    if mine:
        buf[: len(mine)] = torch.from_numpy(rows).to(device)
    outs = [torch.empty_like(buf) for _ in range(len(parts))]
    dist.all_gather(outs, buf)
    out = np.zeros((nfilters, width))
    for r, p in enumerate(parts):
        if p:
            out[p] = outs[r][: len(p)].cpu().numpy()
    return out


def sharded_batch_filter(models, nparticles, resamplers, seeds, y, t0: float = 0.0, dt: float = 1.0,
                         ess_rel: float = 0.5, dist=None, device: str = "cuda"):
    """Filter<BootstrapPF>::filter for every filter of a batch, the filters
    partitioned over the ranks of `dist` (none: this process runs them all).
    y: (T, nfilters, nobs) host observations.  Returns, on every rank,
    (logLikelihood[F], logIncrements[T, F], status[F], parts), parts[r]
    being the filters rank r ran."""
    from .filter import BatchedBootstrapPF

    F = len(models)
    y = np.asarray(y)
    T = y.shape[0]
    rank = dist.get_rank() if dist is not None else 0
    world = dist.get_world_size() if dist is not None else 1
    parts = partition_by_cost([int(n) * T for n in nparticles], world)
    mine = parts[rank]
    rows = np.zeros((0, 2 + T))
    if mine:
        b = BatchedBootstrapPF([models[i] for i in mine], [int(nparticles[i]) for i in mine],
                               [resamplers[i] for i in mine], [int(seeds[i]) for i in mine], ess_rel=ess_rel)
        try:
            ll, inc, _, st = b.filter(np.ascontiguousarray(y[:, mine, :]), t0, dt)
        finally:
            b.close()
        rows = np.column_stack([ll, st.astype(np.float64), inc.T])
    out = gather_by_filter(parts, rank, rows, F, dist, device)
    return out[:, 0], np.ascontiguousarray(out[:, 2:].T), out[:, 1].astype(np.int32), parts
