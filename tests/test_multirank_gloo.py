"""The N>1 path of bench.py without GPUs: two gloo ranks run bench.py's own
shard choice (shard_seed), timed region (timed_region: warm-up, barrier, timed
steps) and job aggregation (job_throughput: max seconds over ranks, units
summed) around a CPU step that scores each rank's shard with the oracle (the
CPU stands in for each rank's GPU; replicas, no data-path collective).  The
launcher (launch_command) starts N ranks itself when no torchrun world exists
and refuses a world that disagrees with --gpus."""

import argparse
import os
import socket
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _model():
    import gkmsvm_lite_b200.synthetic as syn
    from oracle import oracle as orc

    rng = np.random.default_rng(3)
    sv = syn.random_codes(rng, 30, 60)
    coef = rng.normal(size=30)
    kd = orc.KernelDef.from_params("gkmrbf", {"L": 11, "k": 7, "d": 3, "gamma": 2.0})
    return orc.OracleModel(sv, None, coef, 0.0, kd)


def _shard(rank):
    import bench
    import gkmsvm_lite_b200.synthetic as syn

    return syn.random_codes(np.random.default_rng(bench.shard_seed(rank, base=100)), 6 + 2 * rank, 50)


def _rank(rank, world, port, out):
    import datetime
    import time

    import torch

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    from oracle import oracle as orc

    m = _model()
    xq = _shard(rank)
    last = {}

    def step():
        last["scores"] = orc.scores(m, xq)[:, 0]
        if rank == 1:
            time.sleep(0.02)  # the slower rank sets the job's time

    steps = 3
    sec = bench.timed_region(step, steps, 1, dist=dist)
    tmax, units, value = bench.job_throughput(sec, steps * len(xq), dist=dist)
    # shards differ in size: gather them padded to the largest
    got = torch.full((16,), float("nan"), dtype=torch.float64)
    got[:len(xq)] = torch.from_numpy(last["scores"].copy())
    parts = [torch.zeros_like(got) for _ in range(world)]
    dist.all_gather(parts, got)
    if rank == 0:
        out.put((sec, tmax, units, value, [p.numpy()[:6 + 2 * r] for r, p in enumerate(parts)]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas_through_bench_functions():
    from oracle import oracle as orc

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    sec0, tmax, units, value, parts = q.get(timeout=180)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    # rank 1 slept 20 ms per timed step: the job time is the slower rank's
    assert tmax >= 0.06 and tmax >= sec0
    assert units == 3 * (6 + 8)
    assert value == pytest.approx(units / tmax)
    m = _model()
    for r in range(2):
        np.testing.assert_allclose(parts[r], orc.scores(m, _shard(r))[:, 0], rtol=1e-12)


def test_launcher_starts_ranks_or_refuses_mismatch():
    sys.path.insert(0, ROOT)
    import bench

    a = argparse.Namespace(gpus=4)
    cmd = bench.launch_command(a, {})
    assert cmd[1:4] == ["-m", "torch.distributed.run", "--nnodes=1"]
    assert "--nproc-per-node=4" in cmd and "127.0.0.1" in cmd
    assert bench.launch_command(a, {"WORLD_SIZE": "4"}) is None
    assert bench.launch_command(argparse.Namespace(gpus=1), {}) is None
    with pytest.raises(SystemExit, match="WORLD_SIZE=2"):
        bench.launch_command(a, {"WORLD_SIZE": "2"})
