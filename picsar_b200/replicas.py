"""Replicas across GPUs of one node: one process per GPU, each stepping its
own independent simulations; the data path has no collective.

The reference scales one simulation over MPI ranks by domain decomposition
(src/parallelization/mpi/mpi_routines.F90); here the units that shard are
whole simulations (ensemble jobs, served requests), so ranks only agree on
who runs what and combine timings and results at the end:

  * ``shard_jobs``: longest-processing-time-first assignment of jobs to
    ranks by their predicted cost (particle-steps weighted by shape order);
  * ``aggregate``: whole-job units summed and the timed region's duration
    maximised over ranks (the benchmark's reporting rule);
  * ``gather``: every rank's result records collected on all ranks.

All three work with any torch.distributed backend (NCCL on GPUs, gloo on
CPU for tests).
"""
from __future__ import annotations

import heapq

import torch
import torch.distributed as dist

# relative cost of one particle-step by shape order (fused particle kernel,
# FP32, measured on B200 proxies: ~10.6 / 7.4 / 3.9 G particle-steps/s)
ORDER_COST = {1: 1.0, 2: 1.45, 3: 2.7}


def job_cost(spec) -> float:
    return spec.particles * spec.steps * ORDER_COST.get(spec.order, 1.0)


def shard_jobs(specs, world: int, rank: int):
    """The jobs of `specs` this rank runs (greedy LPT over predicted cost;
    deterministic, every job on exactly one rank)."""
    order = sorted(range(len(specs)), key=lambda i: (-job_cost(specs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    mine = []
    for i in order:
        load, r = heapq.heappop(heap)
        if r == rank:
            mine.append(i)
        heapq.heappush(heap, (load + job_cost(specs[i]), r))
    return [specs[i] for i in sorted(mine)]


def _device():
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def aggregate(units: float, ms: float):
    """(units summed over ranks, ms maximised over ranks)."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(units), float(ms)
    dev = _device()
    u = torch.tensor([float(units)], dtype=torch.float64, device=dev)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=dev)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(u.item()), float(t.item())


def gather(records):
    """Concatenation of every rank's list of picklable records, in rank
    order, on every rank."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return list(records)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(records))
    return [r for part in out for r in part]
