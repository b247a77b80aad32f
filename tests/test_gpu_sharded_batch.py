"""A batch of filters sharded over ranks gives, on every rank, exactly the
results of one batch holding all filters: two gloo ranks on one GPU (their
kernels are independent; only the all-gather of the results crosses
processes, on the CPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

NS = [512, 4096, 1024, 2048, 768, 1536, 3072]
RES = ["systematic", "multinomial", "systematic", "multinomial", "systematic", "multinomial", "systematic"]
T = 10


def _workload():
    from libbi_b200 import ModelL96

    rng = np.random.default_rng(8)
    models = [ModelL96(dim=40, F=float(f)) for f in rng.uniform(6.0, 10.0, len(NS))]
    y = rng.standard_normal((T, len(NS), 40)).astype(np.float32) * 3.0
    seeds = [300 + i for i in range(len(NS))]
    return models, seeds, y


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    from libbi_b200.replicas import sharded_batch_filter

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        models, seeds, y = _workload()
        ll, inc, st, parts = sharded_batch_filter(models, NS, RES, seeds, y, 0.0, 0.05, ess_rel=0.5, dist=dist,
                                                  device="cpu")
        out[rank] = (ll, inc, st, parts)
    finally:
        dist.destroy_process_group()


def test_two_ranks_equal_one_batch(cuda):
    from libbi_b200 import BatchedBootstrapPF
    from libbi_b200.replicas import sharded_batch_filter

    models, seeds, y = _workload()
    b = BatchedBootstrapPF(models, NS, RES, seeds, ess_rel=0.5)
    ll_ref, inc_ref, _, st_ref = b.filter(y, 0.0, 0.05)
    b.close()
    assert (st_ref == 0).all()

    # one process, no process group: the same batch
    ll1, inc1, st1, parts1 = sharded_batch_filter(models, NS, RES, seeds, y, 0.0, 0.05, ess_rel=0.5)
    assert parts1 == [list(range(len(NS)))]
    np.testing.assert_array_equal(ll1, ll_ref)
    np.testing.assert_array_equal(inc1, inc_ref)

    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    parts = out[0][3]
    assert all(len(p) > 0 for p in parts) and sorted(sum(parts, [])) == list(range(len(NS)))
    for r in range(world):
        ll, inc, st, pr = out[r]
        assert pr == parts
        np.testing.assert_array_equal(ll, ll_ref)
        np.testing.assert_array_equal(inc, inc_ref)
        np.testing.assert_array_equal(st, st_ref)
