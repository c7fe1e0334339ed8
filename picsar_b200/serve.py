"""Serving loop: simulation jobs arriving over time, continuously batched.

A request is a ``JobSpec`` with an arrival time.  The server keeps every
admitted job's particles and fields resident on the device and steps all of
them together, one batched step (``Ensemble``) per iteration:

  * arrived requests wait in a FIFO queue and are admitted, in order, while
    the predicted device bytes of the resident jobs plus the next one stay
    within the HBM budget (``ensemble.job_bytes``);
  * membership changes only between iterations: newly admitted jobs join the
    next batched step, finished jobs (their step count reached) leave after
    their last step and free their memory for the queue;
  * every job gets FP64 diagnostics: the Gauss-law residual at admission and
    at completion, the total energy after its first step (the kinetic part is
    summed by the particle kernel) and at completion, so its energy drift and
    charge-conservation drift are reported beside its latency.

Latency = completion time - arrival time, measured on the host wall clock
after the device finished the job's last step.  ``clock="iterations"``
replays arrivals in units of batched iterations instead of seconds, which
makes the mix of jobs on the device reproducible (used by the tests).

The reference has no serving mode (one simulation per MPI job).
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .ensemble import Ensemble, JobSpec, job_bytes


@dataclass
class Request:
    rid: int
    spec: JobSpec
    arrival: float                 # seconds (wall clock) or iterations


@dataclass
class JobResult:
    rid: int
    spec: JobSpec
    arrival: float
    admitted: float = 0.0
    finished: float = 0.0
    energy0: float = 0.0
    energy1: float = 0.0
    gauss0: float = 0.0
    gauss1: float = 0.0
    bytes: int = 0

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def energy_drift(self) -> float:
        return (self.energy1 - self.energy0) / self.energy0 if self.energy0 else 0.0

    @property
    def gauss_drift(self) -> float:
        return abs(self.gauss1 - self.gauss0) / self.gauss0 if self.gauss0 else 0.0


def poisson_requests(specs, rate, seed=0, start_id=0):
    """Requests for ``specs`` with exponential inter-arrival times of mean
    1/rate seconds (a Poisson stream), first arrival at 0."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=len(specs))
    gaps[0] = 0.0
    t = np.cumsum(gaps)
    return [Request(start_id + i, s, float(a)) for i, (s, a) in enumerate(zip(specs, t))]


def percentile(values, q):
    return float(np.percentile(np.asarray(values, dtype=np.float64), q)) if values else 0.0


@dataclass
class ServeReport:
    results: list
    makespan: float
    particle_steps: int
    iterations: int
    peak_bytes: int
    peak_resident_jobs: int
    launches: int
    extra: dict = field(default_factory=dict)

    def summary(self):
        lat = [r.latency for r in self.results]
        return {
            "jobs": len(self.results),
            "p50_latency_s": percentile(lat, 50),
            "p99_latency_s": percentile(lat, 99),
            "mean_latency_s": float(np.mean(lat)) if lat else 0.0,
            "particle_steps_per_s": self.particle_steps / self.makespan if self.makespan else 0.0,
            "makespan_s": self.makespan,
            "iterations": self.iterations,
            "peak_resident_jobs": self.peak_resident_jobs,
            "peak_device_bytes": self.peak_bytes,
            "max_abs_energy_drift": max((abs(r.energy_drift) for r in self.results), default=0.0),
            "max_gauss_drift": max((r.gauss_drift for r in self.results), default=0.0),
            **self.extra,
        }


class Server:
    """Continuous-batching server of periodic PIC jobs on one GPU.

    precision: "fp32" (mixed) or "fp64"; hbm_budget: bytes of job state the
    server may keep resident; configs: {order: TiledConfig} (autotuned by
    the caller, or defaults); on_finish(request, sim): optional callback
    that sees a job's TiledSim after its last step, before it is freed."""

    def __init__(self, precision="fp32", hbm_budget=150 * 10 ** 9, configs=None,
                 device="cuda", track_ids=False, on_finish=None):
        self.precision = precision
        self.budget = int(hbm_budget)
        self.configs = configs or {}
        self.device = torch.device(device)
        self.track_ids = track_ids
        self.on_finish = on_finish

    def run(self, requests, clock="wall", idle_sleep=2e-4):
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        pending = collections.deque(reqs)
        queue = collections.deque()
        ens = Ensemble([], precision=self.precision, configs=self.configs, device=self.device,
                       track_ids=self.track_ids, use_graph=False)
        state = {}                 # id(member) -> [request, result, steps_left]
        results = []
        used = 0
        peak_bytes = peak_jobs = 0
        psteps = 0
        it = 0
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        now = lambda: (time.perf_counter() - t0) if clock == "wall" else float(it)
        while pending or queue or ens.members:
            t = now()
            while pending and pending[0].arrival <= t:
                queue.append(pending.popleft())
            changed = False
            while queue:
                r = queue[0]
                b = job_bytes(r.spec, self.precision, self.configs.get(r.spec.order))
                if used + b > self.budget and ens.members:
                    break
                if b > self.budget:
                    raise ValueError(f"job {r.rid} needs {b} B, above the HBM budget")
                queue.popleft()
                m = ens.add(r.spec)
                d = m[1].diagnostics(gauss=True)
                res = JobResult(r.rid, r.spec, r.arrival, admitted=now(),
                                gauss0=d["gauss_norm"], bytes=b)
                state[id(m)] = [r, res, r.spec.steps]
                used += b
                changed = True
            if changed:
                ens.rebuild()
                peak_bytes = max(peak_bytes, used)
                peak_jobs = max(peak_jobs, ens.njobs)
            if ens.njobs == 0:
                if pending and clock == "wall":
                    time.sleep(min(idle_sleep, max(0.0, pending[0].arrival - now())))
                elif pending:
                    it = max(it, int(np.ceil(pending[0].arrival)))
                continue
            ens.step(1)
            # one batched step in flight at a time: admission decisions follow
            # the device timeline, not a host that ran ahead
            torch.cuda.current_stream(self.device).synchronize()
            it += 1
            psteps += ens.particles_total
            done = []
            for m in ens.members:
                st = state[id(m)]
                st[2] -= 1
                if st[2] == m[0].steps - 1:
                    # the particle kernel sums the kinetic energy per tile:
                    # the reference energy is taken after the job's first step
                    st[1].energy0 = m[1].diagnostics(gauss=False)["total"]
                if st[2] == 0:
                    done.append(m)
            if done:
                tf = now()
                for m in done:
                    r, res, _ = state.pop(id(m))
                    d = m[1].diagnostics(gauss=True)
                    res.finished = tf
                    res.energy1, res.gauss1 = d["total"], d["gauss_norm"]
                    if self.on_finish is not None:
                        self.on_finish(r, m[1])
                    results.append(res)
                    used -= res.bytes
                ens.remove(done)
                ens.rebuild()
        torch.cuda.synchronize(self.device)
        makespan = now()
        results.sort(key=lambda r: r.rid)
        return ServeReport(results, makespan, psteps, it, peak_bytes, peak_jobs, ens.launches)


def fifo_latencies(requests, service_s):
    """Completion latencies of the same request stream served one job at a
    time, first come first served, each taking service_s[rid] seconds."""
    reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
    t = 0.0
    out = {}
    for r in reqs:
        t = max(t, r.arrival) + service_s[r.rid]
        out[r.rid] = t - r.arrival
    return out
