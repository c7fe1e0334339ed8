"""Multi-rank host logic of the replica path on CPU: two gloo ranks (spawned
processes, rendezvous on 127.0.0.1) shard an ensemble, aggregate units and
timings, and gather per-job results, exactly as the GPU ranks do over NCCL."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from picsar_b200.ensemble import ensemble_jobs
from picsar_b200.replicas import job_cost, shard_jobs


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from picsar_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        specs = ensemble_jobs(count=64, seed=9, steps=100)
        mine = replicas.shard_jobs(specs, world, rank)
        units = sum(s.particles * s.steps for s in mine)
        ms = 100.0 + 50.0 * rank                      # this rank's timed region
        tot_units, max_ms = replicas.aggregate(units, ms)
        recs = replicas.gather([(s.seed, rank) for s in mine])
        q.put((rank, [s.seed for s in mine], tot_units, max_ms, recs))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_aggregate_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    specs = ensemble_jobs(count=64, seed=9, steps=100)
    seeds = [s.seed for s in specs]
    r0, r1 = out[0][1], out[1][1]
    assert sorted(r0 + r1) == sorted(seeds) and not set(r0) & set(r1)
    total = sum(s.particles * s.steps for s in specs)
    for _, _, tot_units, max_ms, recs in out:
        assert tot_units == total
        assert max_ms == 150.0
        assert sorted(r[0] for r in recs) == sorted(seeds)
        assert [r[1] for r in recs] == [0] * len(r0) + [1] * len(r1)


def test_shard_balance_and_single_rank():
    specs = ensemble_jobs(count=256, seed=2024, steps=100)
    assert shard_jobs(specs, 1, 0) == specs
    loads = [sum(job_cost(s) for s in shard_jobs(specs, 4, r)) for r in range(4)]
    assert max(loads) / min(loads) < 1.1
    parts = [shard_jobs(specs, 3, r) for r in range(3)]
    assert sum(len(p) for p in parts) == len(specs)
