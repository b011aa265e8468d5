"""The N>1 path of bench.py without GPUs: two gloo ranks each score their own
query shard (replicas, no data-path collective) and agree on the step time as
the max over ranks; whole-job throughput is the sum of the shards over that
time.  The scoring itself is the oracle's here (the CPU stands in for each
rank's GPU)."""

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import time

    import torch

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import gkmsvm_lite_b200.synthetic as syn
    from oracle import oracle as orc

    rng = np.random.default_rng(3)
    sv = syn.random_codes(rng, 30, 60)
    coef = rng.normal(size=30)
    kd = orc.KernelDef.from_params("gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0})
    m = orc.OracleModel(sv, None, coef, 0.0, kd)
    # each rank its own shard of the query stream (seed + rank), as bench.py
    xq = syn.random_codes(np.random.default_rng(100 + rank), 6, 50)
    dist.barrier()
    t0 = time.perf_counter()
    s = orc.scores(m, xq)
    dt = torch.tensor([time.perf_counter() - t0 + 0.01 * rank])
    dist.all_reduce(dt, op=dist.ReduceOp.MAX)
    got = torch.from_numpy(s[:, 0].copy())
    parts = [torch.zeros_like(got) for _ in range(world)]
    dist.all_gather(parts, got)
    if rank == 0:
        out.put((float(dt), [p.numpy() for p in parts]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas_max_time():
    import gkmsvm_lite_b200.synthetic as syn
    from oracle import oracle as orc

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    t, parts = q.get(timeout=120)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    # rank 1 added 10 ms: the job time is the slower rank's
    assert t >= 0.01
    rng = np.random.default_rng(3)
    sv = syn.random_codes(rng, 30, 60)
    coef = rng.normal(size=30)
    kd = orc.KernelDef.from_params("gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0})
    m = orc.OracleModel(sv, None, coef, 0.0, kd)
    for r in range(2):
        xq = syn.random_codes(np.random.default_rng(100 + r), 6, 50)
        np.testing.assert_allclose(parts[r], orc.scores(m, xq)[:, 0], rtol=1e-12)
