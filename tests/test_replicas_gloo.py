"""The multi-GPU path is replicas (one filter per rank, no exchange on the
data path): two gloo ranks on the CPU check the host side of it: distinct
per-rank seeds whose filters differ, the slowest rank's time reaching every
rank, and the whole-job rate over all ranks' work.  Each rank runs the
oracle's CPU filter as its stand-in replica."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    from libbi_b200 import ModelPZ
    from libbi_b200.replicas import max_over_ranks, replica_seed, whole_job_rate
    from libbi_b200 import _native as N
    from oracle.oracle import Oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        orc = Oracle()
        model = ModelPZ()
        desc = model.desc()
        y, _ = orc.simulate(desc, 1, 8, 0.0, 1.0)
        cfg = N.Config()
        cfg.nparticles = 256
        cfg.resampler = N.BPF_RESAMPLER_SYSTEMATIC
        cfg.ess_rel = 1.0
        cfg.seed = replica_seed(7, rank)
        ll = orc.filter(desc, cfg, y, 8, 0.0, 1.0)["ll"]
        # every rank learns every rank's log-likelihood and seed
        got = [None] * world
        dist.all_gather_object(got, (cfg.seed, ll))
        elapsed = 10.0 + 5.0 * rank  # a stand-in per-rank time in ms
        slowest = max_over_ranks(elapsed, dist, "cpu")
        rate = whole_job_rate(256 * 8, world, slowest / 1e3)
        out[rank] = (got, slowest, rate)
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas():
    pytest.importorskip("torch.distributed")
    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    (g0, s0, r0), (g1, s1, r1) = out[0], out[1]
    assert g0 == g1  # both ranks see both replicas
    seeds = [s for s, _ in g0]
    lls = [v for _, v in g0]
    assert seeds[0] != seeds[1] and lls[0] != lls[1]  # independent replicas
    assert s0 == s1 == 15.0  # the slowest rank's time on every rank
    assert r0 == r1 == pytest.approx(256 * 8 * 2 / 0.015)
