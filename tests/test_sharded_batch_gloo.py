"""Batched filters shard over ranks: the cost partition, and the all-gather
that gives every rank every filter's results in filter order.  Ranks are
gloo processes on the CPU; each runs the oracle's FP64 filter for the
filters of its share, and the assembled table must equal the serial run of
every filter."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from libbi_b200.replicas import gather_by_filter, partition_by_cost

NS = [64, 512, 128, 256, 96, 320]
SEEDS = [11, 12, 13, 14, 15, 16]
T = 6


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_rows(idx):
    from libbi_b200 import ModelPZ
    from libbi_b200 import _native as N
    from oracle.oracle import Oracle

    orc = Oracle()
    desc = ModelPZ().desc()
    y, _ = orc.simulate(desc, 3, T, 0.0, 1.0)
    rows = []
    for i in idx:
        cfg = N.Config()
        cfg.nparticles = NS[i]
        cfg.resampler = N.BPF_RESAMPLER_SYSTEMATIC
        cfg.ess_rel = 1.0
        cfg.seed = SEEDS[i]
        r = orc.filter(desc, cfg, y, T, 0.0, 1.0)
        rows.append(np.concatenate([[r["ll"], float(r["rc"])], r["inc"]]))
    return np.array(rows).reshape(len(idx), 2 + T)


def _rank(rank, world, port, nf, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        parts = partition_by_cost([NS[i] * T for i in range(nf)], world)
        rows = _oracle_rows(parts[rank]) if parts[rank] else np.zeros((0, 2 + T))
        out[rank] = (parts, gather_by_filter(parts, rank, rows, nf, dist, "cpu"))
    finally:
        dist.destroy_process_group()


def test_partition_by_cost():
    costs = [5, 3, 8, 1, 1, 9, 2]
    for world in (1, 2, 3, 8):
        parts = partition_by_cost(costs, world)
        assert len(parts) == world
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        assert all(p == sorted(p) for p in parts)
        assert parts == partition_by_cost(costs, world)  # every rank computes the same
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
    assert partition_by_cost([1, 2, 3], 4)[3] == []
    with pytest.raises(ValueError):
        partition_by_cost([1], 0)


def test_gather_without_process_group():
    rows = np.arange(6.0).reshape(3, 2)
    out = gather_by_filter([[0, 1, 2]], 0, rows[[0, 1, 2]], 3)
    np.testing.assert_array_equal(out, rows)
    with pytest.raises(ValueError):
        gather_by_filter([[0], [1]], 0, rows[:1], 2)


@pytest.mark.parametrize("world,nf", [(2, 6), (3, 2)])
def test_gloo_ranks_assemble_every_filter(world, nf):
    """Two ranks sharing six filters; three ranks sharing two (one rank
    holds none and still takes part in the gather)."""
    pytest.importorskip("torch.distributed")
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, nf, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    want = _oracle_rows(list(range(nf)))
    parts0 = out[0][0]
    assert sum(len(p) for p in parts0) == nf
    if world > nf:
        assert any(len(p) == 0 for p in parts0)
    for r in range(world):
        parts, table = out[r]
        assert parts == parts0
        np.testing.assert_array_equal(table, want)
