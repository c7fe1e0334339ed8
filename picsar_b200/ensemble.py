"""Batched ensembles: many independent periodic simulations stepped together.

Each simulation ("job") keeps its own grids and particle arrays in the tiled
layout of ``TiledSim``; the ensemble packs all job descriptors into one
device array and steps every job in a fixed set of launches:

  * one fused particle kernel per shape order (persistent CTAs pull
    (job, tile) items from a work list that covers every tile of every job
    of that order, the most loaded tiles first);
  * one B half push, one E push and one B half push over the cells of all
    jobs (``pxrb_tiled_push_b`` / ``pxrb_tiled_push_e`` with per-job cell
    offsets);
  * a batched counting sort per order group every ``sort_interval`` steps
    (``pxrb_tiled_sort_batch``).

The per-step launches are captured once in a CUDA graph and replayed; the
sorts and re-layouts have graphs of their own.  Jobs of one order share one tile shape,
thread count and accumulator (template parameters of the particle kernel),
chosen per order by ``picsar_b200.autotune``.

This is the batched form of the reference's per-species, per-tile loops
(src/submain.F90:104-195 driven once per simulation); the reference itself
runs one simulation per process.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .init import thermal_plasma
from .tiled import TiledConfig, TiledJob, TiledSim, _stream, h2d, launch_threads

_lib.register({"pxrb_tiled_sort_batch": "p I I I i s", "pxrb_tiled_relayout": "p I I I i s"})


@dataclass
class JobSpec:
    """One periodic thermal-plasma simulation of an ensemble or a served
    stream: grid cells, particles per cell, thermal momentum spread, shape
    order, pusher (0 Boris, 1 Vay), steps to run and the seed of its initial
    state."""
    n: tuple
    ppc: int
    sigma: float
    order: int
    pusher: int = 0
    steps: int = 100
    seed: int = 0

    def __post_init__(self):
        if int(self.steps) < 1:
            raise ValueError(f"a job runs at least one step (steps = {self.steps})")
        if int(self.ppc) < 0 or min(int(v) for v in self.n) < 1:
            raise ValueError(f"invalid job size: n = {self.n}, ppc = {self.ppc}")

    @property
    def cells(self) -> int:
        return int(self.n[0]) * int(self.n[1]) * int(self.n[2])

    @property
    def particles(self) -> int:
        return self.cells * int(self.ppc)

    def initial_state(self, device="cuda"):
        return thermal_plasma(self.n, self.ppc, self.sigma, seed=self.seed, device=device)


def ensemble_jobs(count=256, seed=2024, steps=100, cells=(16, 96), ppcs=(1, 2, 4, 8, 16),
                  orders=(1, 2, 3), sigma=(1e-3, 5e-2), steps_range=None, pusher=0):
    """Job specs of the uneven ensemble: per-axis cell counts uniform over
    ``cells`` (inclusive), ppc drawn from ``ppcs``, shape order from
    ``orders``, u_th log-uniform over ``sigma``; every job ``steps`` steps (or
    uniform over ``steps_range``, inclusive).  One master seed gives every
    job its own seed."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = tuple(int(v) for v in rng.integers(cells[0], cells[1] + 1, size=3))
        ppc = int(rng.choice(ppcs))
        order = int(rng.choice(orders))
        sg = float(math.exp(rng.uniform(math.log(sigma[0]), math.log(sigma[1]))))
        st = int(rng.integers(steps_range[0], steps_range[1] + 1)) if steps_range else int(steps)
        out.append(JobSpec(n=n, ppc=ppc, sigma=sg, order=order, pusher=pusher, steps=st,
                           seed=int(rng.integers(0, 2 ** 31 - 1))))
    return out


def job_bytes(spec: JobSpec, precision="fp32", config: TiledConfig | None = None) -> int:
    """Device bytes a job holds once loaded (grids, particles with their sort
    buffers, per-tile arrays): the admission cost of the serving loop."""
    cfg = config or TiledConfig()
    t = cfg.tile[0]
    g = max(3, cfg.drift + 2)
    r = 4 if precision == "fp32" else 8
    nt = [-(-v // t) for v in spec.n]
    al = 4 if r == 4 else 2
    pitch = -(-(nt[0] * t + 2 * g) // al) * al
    fcells = pitch * (nt[1] * t + 2 * g) * (nt[2] * t + 2 * g)
    ntiles = nt[0] * nt[1] * nt[2]
    grid = 6 * fcells * r + 4 * spec.cells * 8 + ntiles * (t ** 3 * 4 + 32)
    parts = spec.particles * (2 * (7 * r + 4) + 8)
    return int(grid + parts + (1 << 16))


_CAPTURE_STREAMS = {}


def _capture_stream(dev):
    """The stream graphs are captured on (one per device, from torch's
    high-priority pool, so that it is not one of the low-priority pool
    streams other code keeps for its own work)."""
    s = _CAPTURE_STREAMS.get(dev.index)
    if s is None:
        s = _CAPTURE_STREAMS[dev.index] = torch.cuda.Stream(device=dev, priority=-1)
    return s


class _Group:
    """Jobs of one shape order: one particle-kernel launch and one batched
    sort per step / sort interval."""

    def __init__(self, order, cfg, first, count):
        self.order, self.cfg, self.first, self.count = order, cfg, first, count
        self.work = None
        self.nwork = 0
        self.max_tiles = 0
        self.max_np = 0
        self.smem = 0
        self.acc = 2
        self.ctr = None


class Ensemble:
    """Independent periodic simulations stepped in one set of launches.

    specs: JobSpec list (any mix of grid sizes, ppc, orders, pushers).
    configs: {order: TiledConfig} (defaults: TiledConfig()); all jobs of an
    order share it.  states: optional list of PlasmaState (default: each
    spec's seeded thermal plasma).  use_graph: replay the per-step launches
    from a CUDA graph (captured on the first step)."""

    def __init__(self, specs, precision="fp32", configs=None, device="cuda", track_ids=False,
                 states=None, use_graph=True):
        self.device = torch.device(device)
        self.precision = precision
        self.prec = 0 if precision in ("fp32", "mixed") else 1
        self.configs = {o: (configs or {}).get(o, TiledConfig()) for o in (1, 2, 3)}
        self.track_ids = track_ids
        self.use_graph = use_graph
        self.num_sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        self.members = []          # [spec, sim] in packed (order-grouped) order
        self.launches = 0
        self.it = 0
        self._graph = None
        self._sort_graphs = {}
        specs = list(specs)
        for i, sp in enumerate(specs):
            st = states[i] if states is not None else None
            self.members.append(self._make_member(sp, st))
        self.rebuild()

    # ----------------------------------------------------------------- setup
    def _make_member(self, spec, state=None, diag_out=None):
        """A job's simulation, loaded and sorted on the current stream.
        diag_out: optional DEVICE float64[9] that receives the FP64
        diagnostics (with the Gauss residual) of the loaded state, taken
        before the sort so that no descriptor is read back."""
        sim = TiledSim(spec.n, order=spec.order, pusher=spec.pusher, precision=self.precision,
                       config=self.configs[spec.order], track_ids=self.track_ids,
                       device=self.device)
        st = state if state is not None else spec.initial_state(device=self.device)
        sim.load_particles(st.x, st.y, st.z, st.ux, st.uy, st.uz, st.w, sort=False)
        del st
        if diag_out is not None:
            diag_out.copy_(sim.diagnostics(gauss=True, to_host=False, pull=False))
        sim.sort()
        self.launches += sim.launches
        return [spec, sim]

    def prepare(self, spec, state=None, diag_out=None):
        """Build a job's member on the current stream without adding it (see
        join)."""
        return self._make_member(spec, state, diag_out)

    def join(self, members):
        """Add prepared members (their preparation must be complete on, or
        ordered before, the current stream) and repack on the device."""
        self.members.extend(members)
        self.rebuild(pull=False)

    def leave(self, members):
        """Retire members and repack on the device; the retired simulations
        keep their state (and descriptors) for reading."""
        self.remove(members)
        self.rebuild(pull=False)

    def add(self, spec, state=None):
        """Admit one more job (the caller rebuilds before the next step)."""
        m = self._make_member(spec, state)
        self.members.append(m)
        return m

    def remove(self, members):
        """Retire jobs (their device memory is released when the last
        reference to the returned simulations goes)."""
        ids = {id(m) for m in members}
        self.members = [m for m in self.members if id(m) not in ids]

    def rebuild(self, pull=True):
        """Pack descriptors, group by order, build work lists and per-job
        cell offsets for the current membership.  pull=True packs the host
        descriptors after reading each back from the device (one host
        synchronisation per member); pull=False packs on the device by
        copying each member's current device descriptor (no host
        synchronisation: the serving loop's path)."""
        self.members.sort(key=lambda m: m[0].order)
        self._graph = None
        self._sort_graphs = {}
        nj = len(self.members)
        self.njobs = nj
        if nj == 0:
            self.groups = []
            return
        sz = C.sizeof(TiledJob)
        if pull:
            host = bytearray(sz * nj)
            for k, (sp, sim) in enumerate(self.members):
                sim._pull_job()      # re-layouts may have exchanged its particle buffers
                host[k * sz:(k + 1) * sz] = bytes(sim.job)
            self.jobs_dev = torch.frombuffer(host, dtype=torch.uint8).to(self.device)
        else:
            # (a retired member keeps its old slot: its job_dev view holds
            # the previous packed array)
            self.jobs_dev = torch.cat([sim.job_dev for _, sim in self.members])
        # each member's device descriptor is its slot of the packed array, so
        # the member sees what the batched launches change there
        for k, (sp, sim) in enumerate(self.members):
            sim.job_dev = self.jobs_dev[k * sz:(k + 1) * sz]
        self.groups = []
        k = 0
        while k < nj:
            o = self.members[k][0].order
            e = k
            while e < nj and self.members[e][0].order == o:
                e += 1
            grp = _Group(o, self.configs[o], k, e - k)
            items = []
            for jj in range(k, e):
                sp, sim = self.members[jj]
                grp.max_tiles = max(grp.max_tiles, sim.ntiles)
                grp.max_np = max(grp.max_np, sim.np)
                grp.smem = max(grp.smem, sim.smem)
                grp.acc = sim.acc
                items.append((-sp.ppc, jj, sim.ntiles))
            items.sort()                    # densest jobs' tiles first
            w = np.concatenate([np.stack([np.full(nt, jj, np.int32),
                                          np.arange(nt, dtype=np.int32)], 1)
                                for _, jj, nt in items])
            grp.work = h2d(torch.from_numpy(np.ascontiguousarray(w)), self.device)
            grp.nwork = int(w.shape[0])
            grp.ctr = torch.zeros(1, dtype=torch.int32, device=self.device)
            self.groups.append(grp)
            k = e
        offs = [0]
        for sp, sim in self.members:
            offs.append(offs[-1] + -(-sp.cells // 1024) * 1024)
        self.total_cells = offs[-1]
        self.cell_off = h2d(torch.tensor(offs, dtype=torch.int64), self.device)
        self.particles_total = sum(sim.np for _, sim in self.members)

    # -------------------------------------------------------------- stepping
    def _launch_step(self):
        s = _stream()
        jd = self.jobs_dev.data_ptr()
        for grp in self.groups:
            cfg = grp.cfg
            ctas = min(grp.nwork, self.num_sms * cfg.ctas_per_sm)
            _lib.call("pxrb_tiled_particle_step", jd, grp.order, self.prec, cfg.tile[0],
                      cfg.drift, grp.acc, grp.work.data_ptr(), grp.nwork, None,
                      grp.ctr.data_ptr(), launch_threads(cfg, grp.acc), ctas, grp.smem, s)
        co = self.cell_off.data_ptr()
        _lib.call("pxrb_tiled_push_b", jd, self.njobs, self.prec, co, self.total_cells, 0.5, s)
        _lib.call("pxrb_tiled_push_e", jd, self.njobs, self.prec, co, self.total_cells, 1, s)
        _lib.call("pxrb_tiled_push_b", jd, self.njobs, self.prec, co, self.total_cells, 0.5, s)

    def _launch_sort(self, grp):
        sz = C.sizeof(TiledJob)
        _lib.call("pxrb_tiled_sort_batch", self.jobs_dev.data_ptr() + grp.first * sz,
                  grp.count, self.prec, grp.max_tiles, grp.max_np, _stream())

    def _launch_relayout(self, grp):
        sz = C.sizeof(TiledJob)
        _lib.call("pxrb_tiled_relayout", self.jobs_dev.data_ptr() + grp.first * sz,
                  grp.count, self.prec, grp.max_tiles, grp.max_np, _stream())

    def _capture(self, fn):
        """fn's launches captured in a CUDA graph on a side stream.  fn has
        run eagerly once before (kernel attributes are set), and nothing is
        allocated inside it, so the capture needs no device synchronisation
        (torch.cuda.graph would synchronise the device and empty the cache):
        the device keeps running queued steps while the host captures, and a
        replay orders after whatever precedes it on the replaying stream."""
        side = _capture_stream(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            g.capture_begin(capture_error_mode="thread_local")
            try:
                fn()
            finally:
                g.capture_end()
        return g

    def _run(self, key, fn):
        """Run fn eagerly the first time, from its captured graph after."""
        if not self.use_graph:
            fn()
            return
        g = self._sort_graphs.get(key)
        if g is None:
            fn()
            self._sort_graphs[key] = self._capture(fn)
        else:
            g.replay()

    def step(self, nsteps=1):
        """nsteps PIC steps of every job."""
        if self.njobs == 0:
            return
        for _ in range(nsteps):
            if self.use_graph:
                if self._graph is None:
                    self._launch_step()              # first step runs eagerly
                    self._graph = self._capture(self._launch_step)
                else:
                    self._graph.replay()
            else:
                self._launch_step()
            self.launches += len(self.groups) + 3
            self.it += 1
            for grp in self.groups:
                K, R = grp.cfg.sort_interval, grp.cfg.relayout_interval
                if K > 0 and self.it % K == 0:
                    self._run(("sort", grp.order), lambda grp=grp: self._launch_sort(grp))
                    self.launches += 7
                elif R > 0 and self.it % R == 0 and grp.max_np > 0 and grp.acc != 4:
                    self._run(("relayout", grp.order), lambda grp=grp: self._launch_relayout(grp))
                    self.launches += 3

    # ------------------------------------------------------------ results
    def sims(self):
        """(spec, TiledSim) pairs in the packed order."""
        return [(sp, sim) for sp, sim in self.members]

    def diagnostics(self, gauss=False):
        """FP64 energies (and Gauss residuals) of every job, packed order."""
        return [sim.diagnostics(gauss=gauss) for _, sim in self.members]

    def slow_path_count(self):
        return sum(sim.slow_path_count() for _, sim in self.members)

    def error_flags(self):
        return [sim.error_flag() for _, sim in self.members]

    def state_bytes(self):
        return sum(sim.state_bytes() for _, sim in self.members)

    def profile_steps(self, nsteps=3):
        """Eager steps with CUDA events around each step's particle kernels
        and around its Yee launches: (particle-kernel ms, Yee ms) per step,
        averaged."""
        s = torch.cuda.current_stream()
        pk = yee = 0.0
        for _ in range(nsteps):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[0].record(s)
            jd = self.jobs_dev.data_ptr()
            for grp in self.groups:
                cfg = grp.cfg
                ctas = min(grp.nwork, self.num_sms * cfg.ctas_per_sm)
                _lib.call("pxrb_tiled_particle_step", jd, grp.order, self.prec, cfg.tile[0],
                          cfg.drift, grp.acc, grp.work.data_ptr(), grp.nwork, None,
                          grp.ctr.data_ptr(), launch_threads(cfg, grp.acc), ctas, grp.smem, _stream())
            ev[1].record(s)
            co = self.cell_off.data_ptr()
            _lib.call("pxrb_tiled_push_b", jd, self.njobs, self.prec, co, self.total_cells, 0.5,
                      _stream())
            _lib.call("pxrb_tiled_push_e", jd, self.njobs, self.prec, co, self.total_cells, 1,
                      _stream())
            _lib.call("pxrb_tiled_push_b", jd, self.njobs, self.prec, co, self.total_cells, 0.5,
                      _stream())
            ev[2].record(s)
            self.launches += len(self.groups) + 3
            self.it += 1
            for grp in self.groups:
                K = grp.cfg.sort_interval
                if K > 0 and self.it % K == 0:
                    self._launch_sort(grp)
                    self.launches += 7
            torch.cuda.synchronize()
            pk += ev[0].elapsed_time(ev[1])
            yee += ev[1].elapsed_time(ev[2])
        return pk / nsteps, yee / nsteps

    def algorithmic_bytes(self):
        """Algorithmic HBM bytes of one step's particle kernels: each
        particle's state read and written once (FP32: 32 + 28 B; FP64:
        60 + 52 B) plus E/B read and the FP64 J read-modify-write once per
        cell (FP32: 24 + 48 B; FP64: 48 + 48 B)."""
        pb, cb = (60, 72) if self.prec == 0 else (112, 96)
        return sum(pb * sim.np + cb * sp.cells for sp, sim in self.members)
