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
    charge-conservation drift are reported beside its latency;
  * the HBM budget is reserved in the admission stream's allocator pool
    before the first request (no device allocation while serving);
  * admission builds the job on a side stream while the batch steps; the
    host runs at most four batched steps ahead of the device and no host
    synchronisation happens per step or per membership change;
  * once the membership has been stable for a few iterations the batched
    step is captured in a CUDA graph (without a device synchronisation) and
    replayed until the membership changes again.

``serve_fifo_plain`` serves the same stream one job at a time on the plain
FP64 path, the comparison baseline.

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
    # per batched step: (device completion time, resident particles)
    timeline: list = field(default_factory=list)

    def tail(self, frac=0.25):
        """The stream's tail: the time from the last batched step that held at
        least `frac` of the peak resident particles to the end, and the
        share of all particle-steps done in it.  Throughput over the whole
        makespan counts the tail, in which the few jobs left cannot fill the
        GPU."""
        if not self.timeline:
            return 0.0, 0.0
        peak = max(p for _, p in self.timeline)
        last = max(i for i, (_, p) in enumerate(self.timeline) if p >= frac * peak)
        t_last = self.timeline[last][0]
        ps_tail = sum(p for _, p in self.timeline[last + 1:])
        tot = sum(p for _, p in self.timeline)
        return max(0.0, self.makespan - t_last), (ps_tail / tot if tot else 0.0)

    def summary(self):
        lat = [r.latency for r in self.results]
        tail_s, tail_share = self.tail()
        # offered load: the stream's particle-steps over its arrival span (at
        # rates where this is below the server's capacity the throughput is
        # set by the arrivals, not by the server)
        span = max((r.arrival for r in self.results), default=0.0)
        return {
            "jobs": len(self.results),
            "p50_latency_s": percentile(lat, 50),
            "p99_latency_s": percentile(lat, 99),
            "mean_latency_s": float(np.mean(lat)) if lat else 0.0,
            "particle_steps_per_s": self.particle_steps / self.makespan if self.makespan else 0.0,
            "offered_particle_steps_per_s": self.particle_steps / span if span > 0 else None,
            "makespan_s": self.makespan,
            "iterations": self.iterations,
            "peak_resident_jobs": self.peak_resident_jobs,
            "peak_device_bytes": self.peak_bytes,
            "max_abs_energy_drift": max((abs(r.energy_drift) for r in self.results), default=0.0),
            "max_gauss_drift": max((r.gauss_drift for r in self.results), default=0.0),
            "tail_s": tail_s,
            "tail_particle_steps_share": tail_share,
            "particle_steps_per_s_before_tail":
                (self.particle_steps * (1.0 - tail_share) / (self.makespan - tail_s)
                 if self.makespan > tail_s else 0.0),
            **self.extra,
        }


_ADMISSION_STREAMS = {}
_ALLOC_KEYS = ("num_device_alloc", "num_device_free", "num_alloc_retries", "num_sync_all_streams")


def _admission_stream(dev):
    """One admission stream per device for the life of the process: the
    caching allocator pools blocks per allocating stream, so the memory of
    retired jobs (built on this stream) is reused by later builds, in this
    run and the next."""
    s = _ADMISSION_STREAMS.get(dev.index)
    if s is None:
        s = _ADMISSION_STREAMS[dev.index] = torch.cuda.Stream(device=dev)
    return s


def _reserve(dev, stream, nbytes, small_segments=512):
    """Fill the caching allocator's pools of `stream` with `nbytes` of device
    memory (one segment, split later for the jobs' large arrays) and
    `small_segments` 2 MiB segments (for their small arrays), then release
    the tensors: the blocks stay cached for that stream.  A device allocation
    made while the persistent particle kernel holds the GPU can stall the
    host for tens of milliseconds; with the budget reserved up front the
    builds allocate nothing from the device."""
    free, _ = torch.cuda.mem_get_info(dev)
    nbytes = int(min(nbytes, free - (4 << 30)))
    with torch.cuda.stream(stream):
        if nbytes > 0:
            big = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            del big
        small = [torch.empty(1 << 20, dtype=torch.uint8, device=dev)
                 for _ in range(2 * small_segments)]
        del small


def _readout_stream(dev):
    """The stream of finished jobs' read-outs (one per device)."""
    key = ("readout", dev.index)
    s = _ADMISSION_STREAMS.get(key)
    if s is None:
        s = _ADMISSION_STREAMS[key] = torch.cuda.Stream(device=dev)
    return s


def _pinned(n, dtype):
    return torch.empty(n, dtype=dtype, pin_memory=True)


class _Readout:
    """A finished job's read-out, staged so that the host never waits for
    the device: (1) its device descriptor and its admission and first-step
    diagnostics are copied to pinned host memory on the read-out stream;
    (2) once they have landed, the completion diagnostics (energies and the
    Gauss residual, whose charge deposition reads the particle arrays the
    descriptor points at) run on that stream and are copied back; (3) the
    result is then complete.  The job has left the batch, so nothing else
    writes its state."""

    def __init__(self, request, res, sim, d0, d1, stream, last_step):
        self.request, self.res, self.sim = request, res, sim
        self.d0, self.d1, self.stream = d0, d1, stream
        self.stage = 0
        stream.wait_event(last_step)
        with torch.cuda.stream(stream):
            self.raw = _pinned(sim.job_dev.numel(), torch.uint8)
            self.raw.copy_(sim.job_dev, non_blocking=True)
            self.h0 = _pinned(9, torch.float64)
            self.h0.copy_(d0, non_blocking=True)
            self.h1 = _pinned(9, torch.float64)
            self.h1.copy_(d1, non_blocking=True)
            self.ev = torch.cuda.Event()
            self.ev.record(stream)

    def advance(self, block):
        """Move on as far as the device allows (block: wait for it); True
        once the result is complete."""
        if self.stage == 0:
            if block:
                self.ev.synchronize()
            elif not self.ev.query():
                return False
            self.sim.set_job_bytes(self.raw)
            with torch.cuda.stream(self.stream):
                d = self.sim.diagnostics(gauss=True, to_host=False, pull=False)
                self.h2 = _pinned(9, torch.float64)
                self.h2.copy_(d, non_blocking=True)
                self.ev = torch.cuda.Event()
                self.ev.record(self.stream)
            self.stage = 1
        if self.stage == 1:
            if block:
                self.ev.synchronize()
            elif not self.ev.query():
                return False
            g0, e1, d = self.h0.tolist(), self.h1.tolist(), self.h2.tolist()
            res = self.res
            res.gauss0 = g0[7]
            res.energy0 = e1[0] + sum(e1[1:7])
            res.energy1, res.gauss1 = d[0] + sum(d[1:7]), d[7]
            self.stage = 2
        return True


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

    def run(self, requests, clock="wall", idle_sleep=2e-4, lag=4, graph_after=3,
            builds_per_step=2):
        """Serve `requests`; returns a ServeReport.

        Admission builds a job (allocation, initial state, load, Gauss
        residual, sort) on a side stream while the resident batch keeps
        stepping; the job joins the batch at the first iteration boundary
        after its build completed; while a batch is resident at most
        `builds_per_step` builds are issued between two of its steps, so
        that a burst of arrivals does not leave the device without queued
        steps.  Membership changes repack the device descriptors without
        host synchronisation.  Up to `lag` batched steps are in flight ahead
        of the host; a job completes when the device finishes its last step
        (CUDA event time); its read-out (completion diagnostics) runs on a
        third stream without blocking the host, and its memory goes back to
        the budget when the read-out is done.  After `graph_after`
        iterations without a membership change the step is replayed from a
        CUDA graph (0: never).  clock="iterations": arrivals and latencies
        in iterations, admission and retirement synchronous, so the mix on
        the device is reproducible."""
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        pending = collections.deque(reqs)
        queue = collections.deque()
        dev = self.device
        wall = clock == "wall"
        main = torch.cuda.current_stream(dev)
        side = _admission_stream(dev)
        rstream = _readout_stream(dev)
        ens = Ensemble([], precision=self.precision, configs=self.configs, device=dev,
                       track_ids=self.track_ids, use_graph=False)
        preparing = collections.deque()  # [request, result, member, event, Gauss diagnostics]
        state = {}                       # id(member) -> [request, result, steps left, diag0, diag1]
        inflight = collections.deque()   # (event, iteration, members that finished there, particles)
        finishing = collections.deque()  # _Readout of finished jobs
        timeline = []
        stable = 0                       # iterations since the last membership change
        results = []
        used = 0
        peak_bytes = peak_jobs = 0
        psteps = 0
        it = 0
        torch.cuda.synchronize(dev)
        # blocks cached in other streams' pools go back to the device first, so
        # that admission allocations do not run the device out of memory and
        # make the allocator free its cache with a device synchronisation;
        # then the budget is reserved in the admission stream's pool
        torch.cuda.empty_cache()
        _reserve(dev, side, self.budget + (256 << 20))
        torch.cuda.synchronize(dev)
        alloc0 = torch.cuda.memory_stats(dev)
        t0 = time.perf_counter()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev0.record(main)
        now = lambda: (time.perf_counter() - t0) if wall else float(it)
        # host seconds per phase of the loop (reported with the results)
        phase = collections.defaultdict(float)
        tick = time.perf_counter

        def retire(ev, k, done, parts):
            tw = tick()
            ev.synchronize()
            phase["wait_for_device"] += tick() - tw
            timeline.append((ev0.elapsed_time(ev) / 1e3 if wall else float(k), parts))
            for m in done:
                r, res, _, d0, d1 = state.pop(id(m))
                res.finished = ev0.elapsed_time(ev) / 1e3 if wall else float(k)
                finishing.append(_Readout(r, res, m[1], d0, d1, rstream, ev))

        def finish(block):
            nonlocal used
            tf = tick()
            while finishing and finishing[0].advance(block):
                f = finishing.popleft()
                if self.on_finish is not None:
                    self.on_finish(f.request, f.sim)
                results.append(f.res)
                used -= f.res.bytes
            # later read-outs may already be past their first stage
            for f in list(finishing)[1:]:
                f.advance(False)
            phase["readout"] += tick() - tf

        while pending or queue or preparing or ens.members or inflight or finishing:
            t = now()
            while pending and pending[0].arrival <= t:
                queue.append(pending.popleft())
            # admission: reserve the job's bytes and build it on the side stream
            built = 0
            while queue and (built < builds_per_step or not ens.members):
                r = queue[0]
                b = job_bytes(r.spec, self.precision, self.configs.get(r.spec.order))
                if b > self.budget:
                    raise ValueError(f"job {r.rid} needs {b} B, above the HBM budget")
                if used + b > self.budget and (ens.members or preparing or inflight or
                                               finishing):
                    break
                queue.popleft()
                used += b
                peak_bytes = max(peak_bytes, used)
                res = JobResult(r.rid, r.spec, r.arrival, admitted=now(), bytes=b)
                ta = tick()
                # Everything the build writes is allocated on the side stream
                # (its own pool): a block freed on the main stream may still be
                # read by the steps queued there, so the side stream must never
                # write one.  The build runs concurrently with the batch's steps.
                with torch.cuda.stream(side):
                    d0 = torch.empty(9, dtype=torch.float64, device=dev)
                    m = ens.prepare(r.spec, diag_out=d0)
                    ev = torch.cuda.Event()
                    ev.record(side)
                preparing.append([r, res, m, ev, d0])
                built += 1
                phase["admission_build"] += tick() - ta
            # jobs whose build finished join at this iteration boundary
            join = []
            while preparing and (not wall or preparing[0][3].query()):
                r, res, m, ev, d0 = preparing.popleft()
                main.wait_event(ev)
                for tsr in m[1].tensors() + [d0]:
                    tsr.record_stream(main)
                state[id(m)] = [r, res, r.spec.steps, d0, None]
                join.append(m)
            if join:
                stable = 0
                tj = tick()
                ens.join(join)
                phase["join_repack"] += tick() - tj
                peak_jobs = max(peak_jobs, ens.njobs)
            if ens.members:
                ts = tick()
                ens.use_graph = graph_after > 0 and stable >= graph_after
                ens.step(1)
                stable += 1
                it += 1
                parts = ens.particles_total
                psteps += parts
                done = []
                for m in ens.members:
                    st = state[id(m)]
                    st[2] -= 1
                    if st[2] == m[0].steps - 1:
                        # the particle kernel sums the kinetic energy: the
                        # reference energy is the one after the job's first step
                        st[4] = m[1].diagnostics(gauss=False, to_host=False).clone()
                    if st[2] == 0:
                        done.append(m)
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(main)
                if done:
                    ens.leave(done)
                    stable = 0
                inflight.append((ev, it, done, parts))
                phase["step_launch"] += tick() - ts
            # retire: at most `lag` steps ahead of the host (all of them with
            # the iterations clock or an idle batch)
            while inflight and (not wall or not ens.members or len(inflight) > lag or
                                inflight[0][0].query()):
                retire(*inflight.popleft())
            if finishing:
                finish(block=not wall)
            if not ens.members and not inflight:
                if preparing or finishing:
                    time.sleep(idle_sleep)
                elif not queue and pending:
                    if wall:
                        time.sleep(min(idle_sleep, max(0.0, pending[0].arrival - now())))
                    else:
                        it = max(it, int(np.ceil(pending[0].arrival)))
        torch.cuda.synchronize(dev)
        makespan = now()
        results.sort(key=lambda r: r.rid)
        rep = ServeReport(results, makespan, psteps, it, peak_bytes, peak_jobs, ens.launches,
                          timeline=timeline)
        rep.extra["host_seconds_by_phase"] = dict(phase)
        alloc1 = torch.cuda.memory_stats(dev)
        rep.extra["allocator"] = {k: alloc1.get(k, 0) - alloc0.get(k, 0) for k in _ALLOC_KEYS}
        return rep


def serve_fifo_plain(requests, device="cuda", idle_sleep=2e-4):
    """The same request stream served the way one simulation per process runs
    it: one job at a time, first come first served, each on the plain FP64
    path (PicsarModule, PICSAR arrays).  Latency = completion (host wall
    clock, after the device finished the job) - arrival.  Returns a
    ServeReport."""
    from .picsar import PicsarModule
    reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
    dev = torch.device(device)
    results, psteps = [], 0
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0
    for r in reqs:
        while now() < r.arrival:
            time.sleep(min(idle_sleep, r.arrival - now()))
        res = JobResult(r.rid, r.spec, r.arrival, admitted=now())
        sp = r.spec
        st = sp.initial_state(device=dev)
        m = PicsarModule(*sp.n, nguards=3, nox=sp.order, particle_pusher=sp.pusher, device=dev)
        m.add_species("electron", -1.0, 1.0, st.x, st.y, st.z, st.ux, st.uy, st.uz, st.w)
        del st
        m.step(sp.steps)
        torch.cuda.synchronize(dev)
        res.finished = now()
        psteps += sp.particles * sp.steps
        results.append(res)
        del m
    makespan = now()
    results.sort(key=lambda r: r.rid)
    return ServeReport(results, makespan, psteps, 0, 0, 1, 0)


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
