#!/usr/bin/env python
"""Benchmark of the PIC step (particle-steps/s) on one B200 per rank.

Workload ("large"): periodic homogeneous thermal electron plasma, 256^3
cells, 8 particles per cell (134,217,728 electrons), u ~ N(0, 0.01^2) per
component, order-3 shapes, Boris pusher, 8^3 cell tiles, re-sort every 20
steps, 2nd-order Yee at 0.95 CFL, normalized units (c = mu0 = eps0 = 1,
dx = 1), FP32 mixed precision (FP64 J flush and energy sums).  Synthetic
seeded input stands in for the reference's decks.  A step is one full PIC
step: fused gather/push/deposit kernel, B/E/B Yee pushes, the periodic
counting sort every 20 steps, and between sorts a bank-order re-layout of
each tile every 4 steps.

Arms:
  (default)          this framework; also reports the plain FP64 GPU path,
                     the end-to-end host-buffer run, the CPU oracle
                     baseline, a roofline of the fused particle kernel and
                     the SM clocks sampled during the timed region.
  --impl reference   the reference algorithm on the host CPU cores: the
                     C++ restatement of PICSAR's Fortran routines (the
                     Fortran itself cannot be compiled here), OpenMP over
                     the reference's tile loops, on a bounded sample.

Multi-GPU: independent replicas, one per rank (no data-path collective);
value = particle-steps of all ranks / max over ranks of the timed region.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "large": dict(n=(256, 256, 256), ppc=8, order=3, tile=(8, 8, 8), sort_interval=20,
                  sigma=0.01, pusher=0,
                  desc="256^3 cells, 8 ppc (134,217,728 electrons), order 3, tiles 8^3, "
                       "re-sort every 20 steps (bank re-layout every 4 between), Boris, "
                       "u_th 0.01, periodic"),
    "medium": dict(n=(128, 128, 64), ppc=8, order=3, tile=(8, 8, 8), sort_interval=20,
                   sigma=0.01, pusher=0,
                   desc="128x128x64 cells, 8 ppc (8,388,608 electrons), order 3, tiles 8^3, "
                        "re-sort every 20 steps (bank re-layout every 4 between), Boris, "
                        "u_th 0.01, periodic (profiling size)"),
    "uneven": dict(n=(512, 128, 128), ppc=16, order=2, tile=(8, 8, 8), sort_interval=20,
                   sigma=0.005, u_drift=0.2, pusher=0, init="two_stream", autotune=True,
                   desc="512x128x128 cells, density ramp 0->1 over x in [0,256) then flat, "
                        "16 ppc at n0 (~100.7 M electrons), two beams u_x=+-0.2 with u_th "
                        "0.005, order 2, Boris, periodic, autotuned tiles and sort interval"),
    "plain-small": dict(n=(32, 32, 32), ppc=8, order=1, tile=(8, 8, 8), sort_interval=20,
                        sigma=0.01, pusher=0,
                        desc="32^3 cells, 8 ppc (262,144 electrons), order 1, Boris, u_th 0.01"),
}
BYTES_PER_PARTICLE = {0: (32 + 28), 1: (60 + 52)}        # particle kernel, per particle
# Shared-memory work of the fused particle kernel per particle (FP32 engine):
# energy-conserving gather points (E: 3*S*N*N, B: 3*N*S*S; N = order+1,
# S = order) and fast-path Esirkepov accumulator updates (3*(N-1)*N*N, per
# fixed-point word).  Conflict-free shared-memory rates of the B200,
# warp-instructions per clock per SM, measured with a 32-bit load / 32-bit
# atomic-add probe at 8-64 resident warps: LDS.32 0.88, ATOMS.32 0.61.
GATHER_POINTS = {1: 18, 2: 90, 3: 252}
DEPOSIT_UPDATES = {1: 12, 2: 54, 3: 144}
SMEM_RATE = {"lds": 0.88, "atoms": 0.61}


def smem_per_particle(order, acc):
    """(window loads, accumulator atomics) per particle of the fused particle
    kernel.  The cell-grouped kernel (acc 4) loads each window value once per
    group (pair) of particles of a cell and updates a J node once per pair."""
    if acc == 4:
        return GATHER_POINTS[order] / 2.0, DEPOSIT_UPDATES[order] / 2.0
    return GATHER_POINTS[order], DEPOSIT_UPDATES[order] * (2 if acc == 2 else 1)


def smem_floor_ms(order, acc, particles, sms, clock_mhz):
    """Lower bound of the fused particle kernel's time set by shared-memory
    instruction throughput (loads and accumulator atomics, conflict-free)."""
    lds, atoms = smem_per_particle(order, acc)
    clk_per_warp = lds / SMEM_RATE["lds"] + atoms / SMEM_RATE["atoms"]
    return particles / 32.0 * clk_per_warp / sms / (clock_mhz * 1e6) * 1e3
GRID_BYTES_PER_CELL = {0: (24 + 48), 1: (48 + 48)}        # E,B read + J FP64 read-modify-write

def particle_flops(order):
    """Algorithmic floating-point operations of one particle-step of the
    particle kernel at a shape order (mul / add / sub / sqrt / divide count
    one, an FMA two), counted from the loops of the oracle's restatement of
    the reference with the tensor-product gather factored (x, then y, then z):
      gather shapes  node and staggered shape per axis (orders 1/2/3: 1/10/24);
      gather         per component a*b*c + b*c + c FMAs over its stencil
                     (a, b, c = node or staggered extents of the component);
      push           Boris (68) + set_gamma (8);
      position       5 per axis;
      deposit shapes new and old node shapes per axis (1/8/15 each);
      deposit        per component of the no-node-change Esirkepov box of
                     N = order+1 nodes per axis: prefix 2N-3, ds N, A and B
                     5N, weights 4N^2, node updates 2 N^2 (N-1);
      energy         11."""
    n, s = order + 1, order
    shape = {1: (1, 0), 2: (8, 2), 3: (15, 9)}[order]
    comps = [(s, n, n), (n, s, n), (n, n, s), (n, s, s), (s, n, s), (s, s, n)]
    gather = sum(2 * (a * b * c + b * c + c) for a, b, c in comps)
    deposit = 3 * ((2 * n - 3) + n + 5 * n + 4 * n * n + 2 * n * n * (n - 1))
    return (3 * sum(shape) + gather + 76 + 15 + 6 * shape[0] + deposit + 11)


def _initial_state(wl, seed, n=None, device="cuda"):
    """Seeded synthetic initial plasma of a workload (optionally on a
    smaller grid `n` with the same profile, for CPU samples)."""
    from picsar_b200.init import thermal_plasma, two_stream_ramp
    n = n or wl["n"]
    if wl.get("init") == "two_stream":
        ramp = max(1, round(256 * n[0] / wl["n"][0]))
        return two_stream_ramp(n, wl["ppc"], wl["u_drift"], wl["sigma"], seed=seed,
                               ramp_cells=ramp, device=device)
    return thermal_plasma(n, wl["ppc"], wl["sigma"], seed=seed, device=device)


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling (every 100 ms) of the SM clock and the throttle
    reasons of this rank's GPU while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, dev_index):
        import torch
        import tempfile
        self.proc = None
        self.index = None
        fd, self.out = tempfile.mkstemp(prefix=f"pxrb_clocks_rank{dev_index}_", suffix=".csv")
        os.close(fd)
        try:
            pr = torch.cuda.get_device_properties(dev_index)
            want = (int(pr.pci_domain_id), int(pr.pci_bus_id), int(pr.pci_device_id))
            r = subprocess.run(["nvidia-smi", "--query-gpu=index,pci.bus_id",
                                "--format=csv,noheader"], capture_output=True, text=True,
                               timeout=20)
            for line in r.stdout.splitlines():
                idx, pb = (p.strip() for p in line.split(",", 1))
                dom, bus, devfn = pb.split(":")
                if (int(dom, 16), int(bus, 16), int(devfn.split(".")[0], 16)) == want:
                    self.index = idx
        except Exception as e:
            print(f"clock sampler: {e!r}", file=sys.stderr)
            self.index = None
        if self.index is None:
            print(f"clock sampler: no nvidia-smi index for this GPU", file=sys.stderr)

    def start(self):
        if self.index is None:
            return
        self.fh = open(self.out, "w")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", self.index,
                                      f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "100"],
                                     stdout=self.fh, stderr=subprocess.DEVNULL)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        with open(self.out) as f:
            for line in f:
                p = [v.strip() for v in line.split(",")]
                if len(p) < 7:
                    continue
                try:
                    sm.append(float(p[0]))
                    mx.append(float(p[1]))
                except ValueError:
                    continue
                for name, v in zip(self.NAMES, p[3:7]):
                    if v == "Active":
                        reasons.add(name)
        try:
            os.unlink(self.out)
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    import torch
    import torch.distributed as dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1 and not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def _max_over_ranks(x, ws):
    import torch
    import torch.distributed as dist
    if ws == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(ws):
    import torch
    import torch.distributed as dist
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()


# ---------------------------------------------------------------------------
def cpu_oracle_rate(wl, steps, warmup, threads=None):
    """Oracle (C++ restatement of the reference routines, OpenMP over tiles)
    on a 32^3-cell sample of the workload: returns particle-steps/s."""
    from oracle import oracle as O
    from picsar_b200.init import thermal_plasma
    n = (32, 32, 32)
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    if wl.get("init") == "two_stream":
        n = (64, 16, 16)
    st = _initial_state(wl, 11, n=n, device="cpu").numpy()
    sim = O.OracleSim(n, 3, order=wl["order"], pusher=wl["pusher"], tiles=(4, 4, 4),
                      sorting_period=wl["sort_interval"])
    sim.add_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    np_ = len(st["x"])
    sim.step(warmup)
    t0 = time.perf_counter()
    sim.step(steps)
    el = time.perf_counter() - t0
    return np_ * steps / el, el, np_, O.num_threads()


def run_reference(args):
    """Reference arm: the oracle (PICSAR's routines restated, OpenMP over
    16^3-cell tiles, all host cores) on the full workload configuration --
    the same grid, particle count, shape order and pusher as this
    framework's line.  The metric is a rate, so each timed step is one full
    PIC step of the whole state; the step counts are capped (warm-up 1,
    timed 2) to keep the run within minutes."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload in ("ensemble", "serve"):
        return run_reference_jobs(args)
    from oracle import oracle as O
    wl = WORKLOADS[args.workload]
    os.environ["OMP_NUM_THREADS"] = str(os.cpu_count())
    n = wl["n"]
    st = _initial_state(wl, 1234, device="cpu").numpy()
    N = len(st["x"])
    o = O.OracleSim(n, 3, order=wl["order"], pusher=wl["pusher"],
                    tiles=tuple(max(1, v // 16) for v in n),
                    sorting_period=wl["sort_interval"])
    t0 = time.perf_counter()
    o.add_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    t_load = time.perf_counter() - t0
    del st
    warm, steps = min(args.warmup, 1), max(1, min(args.steps, 2))
    o.step(warm)
    t0 = time.perf_counter()
    o.step(steps)
    el = time.perf_counter() - t0
    rate = N * steps / el
    nth = O.num_threads()
    ncell = n[0] * n[1] * n[2]
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": rate,
        "unit": "particle-steps/s", "n_gpus": ws, "steps": steps, "warmup": warm,
        "ms_per_step": 1e3 * el / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["desc"], "particles": N, "cells": ncell,
                   "sample": f"the full workload: {steps} timed PIC steps after {warm} "
                             f"warm-up (steps capped from --steps {args.steps} / --warmup "
                             f"{args.warmup}; the metric is a rate)"},
        "cpu_baseline": {"value": rate, "unit": "particle-steps/s", "cores": nth,
                         "kind": "port",
                         "sample": f"{steps} PIC steps of the full {N}-particle, {ncell}-cell "
                                   f"workload, OpenMP over 16^3-cell tiles "
                                   f"(load {t_load:.1f} s untimed)"},
        "e2e": {"value": rate, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "PICSAR's Fortran cannot be compiled in this image (no Fortran compiler); "
                "the reference arm runs the line-by-line C++ restatement of its routines, "
                "whose kernels are pinned bit for bit to the reference's own routines",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_jobs(args):
    """Reference arm of the ensemble / served workloads: the oracle (OpenMP
    over tiles, all host cores) on a bounded sample of jobs of the same
    distribution, each job its own simulation as the reference runs them."""
    from oracle import oracle as O
    from picsar_b200.ensemble import ensemble_jobs
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    os.environ["OMP_NUM_THREADS"] = str(os.cpu_count())
    specs = ensemble_jobs(count=args.jobs, seed=2024, steps=100)
    sample = sorted(specs[:16], key=lambda sp: sp.particles)[:4]
    steps = max(1, min(args.steps, 3))
    ps, el_tot = 0, 0.0
    for sp in sample:
        st = sp.initial_state(device="cpu").numpy()
        sim = O.OracleSim(sp.n, 3, order=sp.order, pusher=sp.pusher, tiles=(2, 2, 2),
                          sorting_period=20)
        sim.add_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
        sim.step(1)
        t0 = time.perf_counter()
        sim.step(steps)
        el_tot += time.perf_counter() - t0
        ps += sp.particles * steps
    rate = ps / el_tot
    nth = O.num_threads()
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": rate,
        "unit": "particle-steps/s", "n_gpus": ws, "steps": steps, "warmup": 1,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload,
                   "sample": f"{len(sample)} smallest of the first 16 jobs, {steps} steps each"},
        "cpu_baseline": {"value": rate, "unit": "particle-steps/s", "cores": nth, "kind": "port",
                         "sample": f"{len(sample)} jobs x {steps} steps, OpenMP over tiles"},
        "e2e": {"value": rate, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def run_ours(args, emit=True):
    """The default arm on a fixed workload; prints the JSON line (emit) and
    returns it (rank 0; None on the other ranks)."""
    import torch
    from picsar_b200.init import thermal_plasma
    from picsar_b200.tiled import TiledConfig, TiledSim

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    wl = WORKLOADS[args.workload]
    prec = 0 if args.precision == "fp32" else 1
    cfg = TiledConfig(tile=wl["tile"], sort_interval=wl["sort_interval"], drift=1,
                      threads=args.threads, ctas_per_sm=args.ctas_per_sm, acc=args.acc,
                      relayout_interval=args.relayout, select_lanes=bool(args.select_lanes))
    tuned = None
    if wl.get("autotune"):
        from picsar_b200 import autotune
        r = autotune.tune(wl["order"], args.precision, ppc=wl["ppc"], sigma=wl["sigma"],
                          u_drift=wl.get("u_drift", 0.0),
                          pusher=wl["pusher"], acc=args.acc)
        cfg = _with_acc({wl["order"]: r.config}, args.acc)[wl["order"]]
        tuned = {"proxy_rate": r.rate, "cached": r.cached}
    st = _initial_state(wl, 1234 + rank)
    N = st.np
    sim = TiledSim(wl["n"], order=wl["order"], pusher=wl["pusher"], precision=args.precision,
                   config=cfg)
    sim.load_state(st)
    cnt = (sim.tile_off[1:] - sim.tile_off[:-1]).double()
    q = torch.quantile(cnt, torch.tensor([0.0, 0.1, 0.5, 0.9, 0.99, 1.0], dtype=torch.float64,
                                         device=cnt.device)).tolist()
    occupancy = {"particles_per_tile_p0_p10_p50_p90_p99_p100": q,
                 "empty_tile_fraction": float((cnt == 0).double().mean()),
                 "max_over_mean": float(cnt.max() / cnt.mean())}
    del cnt
    for _ in range(args.warmup):
        sim.step(1)
    torch.cuda.synchronize()
    e0 = sim.diagnostics(gauss=False)
    stream = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    launches0 = sim.launches
    deferred0 = sim.deferred_count()
    _barrier(ws)
    clocks.start()
    t_start.record(stream)
    for s in range(args.steps):
        sim.step(1, events=ev[s])
    t_end.record(stream)
    _barrier(ws)
    clk = clocks.stop()
    ms_total = t_start.elapsed_time(t_end)
    ms_total = _max_over_ranks(ms_total, ws)
    kern_ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    launches = sim.launches - launches0
    deferred = (sim.deferred_count() - deferred0) / (N * args.steps)
    e1 = sim.diagnostics(gauss=False)
    slow = sim.slow_path_count()
    value = N * ws * args.steps / (ms_total * 1e-3)

    # roofline of the fused particle kernel
    peak, peak_kind = _peaks()
    ncell = wl["n"][0] * wl["n"][1] * wl["n"][2]
    alg_bytes = BYTES_PER_PARTICLE[prec] * N + GRID_BYTES_PER_CELL[prec] * ncell
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "particle_kernel_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            tj = json.load(f)
        key = f"{args.workload}_{args.precision}"
        if key in tj:
            traffic = tj[key]["dram_bytes_per_launch"]

    # end-to-end through the public API with host buffers
    e2e = None
    if not args.skip_e2e:
        del sim
        torch.cuda.empty_cache()
        e2e = run_e2e(st, wl, args, ws, cfg)
    else:
        del sim
    del st
    torch.cuda.empty_cache()
    # plain FP64 GPU path on the same workload (the comparison baseline)
    fp64 = None
    if not args.skip_fp64:
        fp64 = run_plain_fp64(wl, args, ws, rank)

    # the tiled engine in FP64 on the same workload (the same engine, 1e-12
    # of the oracle), with its roofline
    fp64_tiled = None
    if not args.skip_fp64 and not getattr(args, "skip_fp64_tiled", False) and prec == 0:
        fp64_tiled = run_tiled_fp64(wl, args, ws, rank, cfg)

    # FP32 mixed vs FP64 vs the oracle from one developed state: one-step
    # error, energy and Gauss-law drift and field spectra over the run, for
    # each pusher (rank 0: the oracle runs on the host cores)
    accuracy = None
    if rank == 0 and not args.skip_accuracy and args.precision == "fp32":
        accuracy = [run_accuracy(wl, args, p, cfg, with_oracle=not args.skip_cpu)
                    for p in (0, 1)]

    cpu = None
    if rank == 0 and not args.skip_cpu:
        orc = accuracy[0].get("oracle") if accuracy else None
        if orc:
            cpu = {"value": orc["particle_steps_per_s"], "unit": "particle-steps/s",
                   "cores": orc["threads"], "kind": "port",
                   "sample": f"1 PIC step of the full workload ({orc['particles']} particles, "
                             f"{ncell} cells) from its developed state (oracle, OpenMP over "
                             f"16^3-cell tiles), {orc['step_seconds']:.1f} s"}
        else:
            rate, el, np_, nth = cpu_oracle_rate(wl, args.cpu_steps, 1, os.cpu_count())
            cpu = {"value": rate, "unit": "particle-steps/s", "cores": nth, "kind": "port",
                   "sample": f"{args.cpu_steps} PIC steps of a 32^3-cell, {np_}-particle "
                             f"sample of the workload (oracle, OpenMP over 4^3 tiles), "
                             f"{el:.1f} s"}
    if rank == 0:
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_total / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if prec == 0 else "f64", "data": "synthetic",
            "config": {"workload": wl["desc"],
                       "precision": "FP32 mixed (FP64 J flush and energy sums)" if prec == 0
                       else "FP64", "particles_per_gpu": N, "cells": ncell,
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "l2": "inputs larger than L2 (particle SoA "
                             f"{N * 32 / 1e9:.1f} GB per GPU), no flush",
                       "tuning": {"tile": list(cfg.tile), "drift": cfg.drift,
                                  "threads": cfg.threads, "ctas_per_sm": cfg.ctas_per_sm,
                                  "sort_interval": cfg.sort_interval,
                                  "relayout_interval": cfg.relayout_interval, "acc": cfg.acc,
                                  "select_lanes": cfg.select_lanes,
                                  "autotuned": tuned},
                       "tile_occupancy": occupancy},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": (f"k_cell_step<{wl['order']}>" if cfg.acc == 4 else
                                    f"k_tile_step<{'float' if prec == 0 else 'double'},"
                                    f"{wl['order']}>"),
                         "kernel_ms": kern_ms, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes},
            "smem_roofline": _smem_roofline(wl, prec, cfg, N, kern_ms, clk),
            "compute_roofline": _compute_roofline(wl, prec, N, kern_ms),
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
            "fp64_plain": fp64,
            "fp64_tiled": fp64_tiled,
            "energy": {"start": e0["total"], "end": e1["total"],
                       "rel_change": (e1["total"] - e0["total"]) / e0["total"]},
            "slow_path_particle_steps": slow,
            "deferred_fraction": deferred,
            "accuracy": accuracy,
        }
        if ws == 1 and args.workload == "large" and not getattr(args, "skip_workloads", False):
            line["workloads"] = _workload_legs(args)
        if emit:
            print(json.dumps(line), flush=True)
    if ws > 1 and emit:
        import torch.distributed as dist
        dist.destroy_process_group()
    return line if rank == 0 else None


def _compute_roofline(wl, prec, N, kern_ms):
    """The particle kernel against the measured FMA throughput of this GPU's
    CUDA cores (the tensor cores have no part in the particle step): FP32
    engine against the faster of scalar FP32 and packed f32x2 FMA, FP64
    engine against FP64 FMA (picsar_b200.peaks, about 3 s of probes; packed
    f32x2 FMAs measured no faster than scalar ones on B200)."""
    from picsar_b200 import peaks
    p = peaks.fma_peaks(iters=4096, repeats=2)
    peak = max(p["fp32"], p["fp32x2"]) if prec == 0 else p["fp64"]
    fl = particle_flops(wl["order"])
    achieved = fl * N / (kern_ms * 1e-3) / 1e12
    return {"bound": "fp32" if prec == 0 else "fp64", "flop_per_particle_step": fl,
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peaks_measured": p, "peak_kind": "measured (pxrb_fma_probe)"}


def _smem_roofline(wl, prec, cfg, N, kern_ms, clk):
    if prec != 0:
        return None
    import torch
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = (clk or {}).get("sm_mhz") or 1965.0
    floor = smem_floor_ms(wl["order"], cfg.acc, N, sms, mhz)
    return {"bound": "shared-memory instructions", "floor_ms": floor, "kernel_ms": kern_ms,
            "frac": floor / kern_ms,
            "window_loads_per_particle": smem_per_particle(wl["order"], cfg.acc)[0],
            "accumulator_atomics_per_particle": smem_per_particle(wl["order"], cfg.acc)[1],
            "rates_warp_inst_per_clk_sm": SMEM_RATE, "sm_mhz": mhz}


DEV_STEPS = 10            # FP64 steps that develop the fields before the comparisons
B0 = (0.0, 0.0, 0.5)      # uniform magnetic field of the accuracy legs (omega_c = omega_p / 2)
SPECTRUM_SHELLS = (1, 2, 4, 8, 16, 32, 64, 128)


def _developed_state(wl, pusher, cfg64):
    """The workload's seeded plasma in a uniform field B0, stepped DEV_STEPS
    times by the FP64 tiled engine: E and B grown from the particles' own
    currents plus B0, so both pushers' rotation terms are exercised.
    Returns the state as PICSAR FP64 arrays: fields (3 guards) and particles
    in id order."""
    import torch
    from picsar_b200.picsar import grid_zeros
    from picsar_b200.tiled import TiledSim
    st = _initial_state(wl, 4321)
    t = TiledSim(wl["n"], order=wl["order"], pusher=pusher, precision="fp64", config=cfg64,
                 track_ids=True)
    for name, v in zip(("bx", "by", "bz"), B0):
        if v:
            t.import_field(name, grid_zeros(*wl["n"], 3).fill_(v), 3)
    t.load_state(st)
    del st
    t.step(DEV_STEPS)
    f = {n: t.export_field(n, 3) for n in ("ex", "ey", "ez", "bx", "by", "bz")}
    p = t.particles()
    del t
    torch.cuda.empty_cache()
    return f, p


def _sim_from_state(wl, prec, pusher, cfg, f, p):
    from picsar_b200.tiled import TiledSim
    t = TiledSim(wl["n"], order=wl["order"], pusher=pusher, precision=prec, config=cfg,
                 track_ids=True)
    for name, a in f.items():
        t.import_field(name, a, 3)
    t.load_particles(p["x"], p["y"], p["z"], p["ux"], p["uy"], p["uz"], p["w"], ids=p["id"])
    return t


def _field_spectrum(sim, names):
    """Shell-averaged power sum_c |FFT(F_c)|^2 over the periodic nodes,
    shells of integer |k| (k in grid wave numbers)."""
    import torch
    nx, ny, nz = sim.n
    tot = None
    for name in names:
        a = sim.export_field(name, 3)[3:3 + nx, 3:3 + ny, 3:3 + nz]
        F = torch.fft.fftn(a)
        pw = F.real ** 2 + F.imag ** 2
        del F
        tot = pw if tot is None else tot + pw
    dev = tot.device
    k = [torch.fft.fftfreq(n, d=1.0 / n, device=dev, dtype=torch.float64) for n in (nx, ny, nz)]
    kk = torch.sqrt(k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 +
                    k[2][None, None, :] ** 2)
    shell = torch.round(kk).long().flatten()
    spec = torch.bincount(shell, weights=tot.flatten()) / torch.bincount(shell).clamp(min=1)
    return spec.cpu().numpy()


def _spectra_ratio(s32, s64, kmax):
    import numpy as np
    r = s32[1:kmax + 1] / np.maximum(s64[1:kmax + 1], 1e-300)
    return {"ratio_fp32_over_fp64_median": float(np.median(r)),
            "ratio_min": float(r.min()), "ratio_max": float(r.max()),
            "shells": {str(k): {"fp64": float(s64[k]), "ratio": float(s32[k] / s64[k])}
                       for k in SPECTRUM_SHELLS if k <= kmax}}


def _rel_l2_t(a, b):
    import torch
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b).clamp(min=1e-300))


def _oracle_one_step(wl, pusher, f, p):
    """The oracle (all host cores, OpenMP over 16^3-cell tiles) one step from
    the exported state.  Returns its fields E, B, J (GPU tensors, PICSAR
    layout), particle columns in id order (GPU) and the step's seconds."""
    import numpy as np
    import torch
    from oracle import oracle as O
    n = wl["n"]
    os.environ["OMP_NUM_THREADS"] = str(os.cpu_count())
    o = O.OracleSim(n, 3, order=wl["order"], pusher=pusher,
                    tiles=tuple(max(1, v // 16) for v in n))
    for name, a in f.items():
        o.set_field(name, a.cpu().numpy())
    host = {c: p[c].cpu().numpy() for c in ("x", "y", "z", "ux", "uy", "uz", "w")}
    ids = p["id"].to(torch.float64).cpu().numpy()
    t0 = time.perf_counter()
    o.add_particles(host["x"], host["y"], host["z"], host["ux"], host["uy"], host["uz"],
                    host["w"], pid=ids)
    t_load = time.perf_counter() - t0
    del host, ids
    t0 = time.perf_counter()
    o.step(1)
    el = time.perf_counter() - t0
    fields = {}
    for name in ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz"):
        a = np.asfortranarray(o.get_field(name))
        fields[name] = torch.from_numpy(a).cuda()
    cols = o.columns(["x", "y", "z", "ux", "uy", "uz", "id"])
    nth = O.num_threads()
    del o
    idx = torch.from_numpy(cols.pop("id").astype(np.int64)).cuda()
    parts = {}
    for c, v in cols.items():
        t = torch.empty(len(v), dtype=torch.float64, device="cuda")
        t[idx] = torch.from_numpy(v).cuda()
        parts[c] = t
    return fields, parts, el, t_load, nth


def run_accuracy(wl, args, pusher, cfg, with_oracle=True):
    """FP32 mixed against FP64 and both against the oracle, from a developed
    state of the full workload (uniform B0 plus DEV_STEPS FP64 steps; the
    same exported PICSAR-layout state loaded into each):
      * one step: relative L2 of E, B, J and of the particle momenta and
        positions, FP32 tiled and FP64 tiled against the oracle (the
        reference's routines restated, all host cores) and FP32 against FP64;
      * `accuracy_steps` steps: total-energy drift (from step 1, the first
        step with a kinetic energy sum), Gauss-law residual drift, and the
        shell-averaged E and B power spectra at steps 0, steps/2 and steps."""
    import torch
    from picsar_b200.tiled import SUPPORTED_SHAPES_FP64, TiledConfig
    t0 = time.perf_counter()
    cfg = TiledConfig(tile=cfg.tile, sort_interval=cfg.sort_interval, drift=cfg.drift,
                      threads=cfg.threads, acc=cfg.acc, relayout_interval=cfg.relayout_interval,
                      select_lanes=cfg.select_lanes)
    cfg64 = cfg
    if (cfg.tile[0], cfg.drift) not in SUPPORTED_SHAPES_FP64:
        cfg64 = TiledConfig(tile=cfg.tile, sort_interval=cfg.sort_interval,
                            drift=min(cfg.drift, 1), threads=cfg.threads,
                            relayout_interval=cfg.relayout_interval)
    f, p = _developed_state(wl, pusher, cfg64)
    steps = args.accuracy_steps
    sims = {"fp64": _sim_from_state(wl, "fp64", pusher, cfg64, f, p),
            "fp32": _sim_from_state(wl, "fp32", pusher, cfg, f, p)}
    kmax = min(wl["n"]) // 2
    spectra = {"E": {}, "B": {}}
    spec0 = {prec: {"E": _field_spectrum(t, ("ex", "ey", "ez")),
                    "B": _field_spectrum(t, ("bx", "by", "bz"))} for prec, t in sims.items()}
    for fl in ("E", "B"):
        spectra[fl]["0"] = _spectra_ratio(spec0["fp32"][fl], spec0["fp64"][fl], kmax)
    g0, d1, one = {}, {}, {}
    for prec, t in sims.items():
        g0[prec] = t.diagnostics(gauss=True)["gauss_norm"]
        t.step(1, keep_j=True)
        d1[prec] = t.diagnostics(gauss=False)
        fl = {n: t.export_field(n, 3) for n in ("ex", "ey", "ez", "bx", "by", "bz",
                                                   "jx", "jy", "jz")}
        pp = t.particles()
        fl.update({c: pp[c] for c in ("x", "y", "z", "ux", "uy", "uz")})
        del pp
        one[prec] = fl
    res = {"pusher": "Vay" if pusher else "Boris", "steps": steps,
           "state": f"seeded plasma in a uniform B = {list(B0)}, then {DEV_STEPS} FP64 steps",
           "one_step_rel_l2": {}}

    def errs(a, b):
        out = {}
        for k in b:
            if k in ("x", "y", "z"):
                L = float(wl["n"]["xyz".index(k)])
                d = torch.remainder(a[k] - b[k] + L / 2, L) - L / 2
                out[k] = float(torch.linalg.norm(d) / torch.linalg.norm(b[k]))
            else:
                out[k] = _rel_l2_t(a[k], b[k])
        return out
    res["one_step_rel_l2"]["fp32_vs_fp64"] = errs(one["fp32"], one["fp64"])
    if with_oracle:
        of, op, el, t_load, nth = _oracle_one_step(wl, pusher, f, p)
        ref = dict(of)
        ref.update(op)
        res["one_step_rel_l2"]["fp64_vs_oracle"] = errs(one["fp64"], ref)
        res["one_step_rel_l2"]["fp32_vs_oracle"] = errs(one["fp32"], ref)
        res["oracle"] = {"step_seconds": el, "load_seconds": t_load, "threads": nth,
                         "particles": int(p["x"].numel()),
                         "particle_steps_per_s": p["x"].numel() / el}
        del of, op, ref
    del one, f, p
    torch.cuda.empty_cache()
    half = max(1, steps // 2)
    for prec, t in sims.items():
        t.step(half - 1)
        spec0[prec]["E_half"] = _field_spectrum(t, ("ex", "ey", "ez"))
        spec0[prec]["B_half"] = _field_spectrum(t, ("bx", "by", "bz"))
        t.step(steps - half)
        d = t.diagnostics(gauss=True)
        spec0[prec]["E_end"] = _field_spectrum(t, ("ex", "ey", "ez"))
        spec0[prec]["B_end"] = _field_spectrum(t, ("bx", "by", "bz"))
        res[prec] = {"energy_drift": (d["total"] - d1[prec]["total"]) / d1[prec]["total"],
                     "gauss_residual_start": g0[prec], "gauss_residual_end": d["gauss_norm"],
                     "gauss_residual_drift": abs(d["gauss_norm"] - g0[prec]) / g0[prec],
                     "error_flag": t.error_flag()}
    for fl in ("E", "B"):
        spectra[fl][str(half)] = _spectra_ratio(spec0["fp32"][fl + "_half"],
                                                spec0["fp64"][fl + "_half"], kmax)
        spectra[fl][str(steps)] = _spectra_ratio(spec0["fp32"][fl + "_end"],
                                                 spec0["fp64"][fl + "_end"], kmax)
    res["field_spectra"] = spectra
    e32, e64 = abs(res["fp32"]["energy_drift"]), abs(res["fp64"]["energy_drift"])
    g32, g64 = res["fp32"]["gauss_residual_drift"], res["fp64"]["gauss_residual_drift"]
    res["energy_drift_ratio_fp32_over_fp64"] = e32 / e64 if e64 else None
    res["gauss_drift_fp32_minus_fp64"] = g32 - g64
    res["gauss_residual_ratio_fp32_over_fp64"] = (res["fp32"]["gauss_residual_end"] /
                                                  res["fp64"]["gauss_residual_end"])
    res["seconds"] = time.perf_counter() - t0
    del sims
    torch.cuda.empty_cache()
    return res


def run_e2e(st, wl, args, ws, cfg):
    """The same job end to end through the reference-facing module surface
    (picsar_b200.picsar.PicsarModule on the tiled engine): the PICSAR FP64
    particle arrays handed over from pinned host memory (add_species: upload,
    conversion, sort), the steps with the FP64 energies copied back to the
    host every step, and the particle arrays the steps change (x, y, z, u,
    gamma^-1, in the order they were added) copied back at the end.  The
    module is built before the timed region (field allocation)."""
    import torch
    from picsar_b200.picsar import PicsarModule
    N = st.np
    host = {c: getattr(st, c).to("cpu").pin_memory() for c in ("x", "y", "z", "ux", "uy", "uz", "w")}
    out_cols = ("part_x", "part_y", "part_z", "part_ux", "part_uy", "part_uz", "part_gaminv")
    out_host = {c: torch.empty(N, dtype=torch.float64).pin_memory() for c in out_cols}
    diag_host = torch.empty((args.steps, 9), dtype=torch.float64).pin_memory()
    m = PicsarModule(*wl["n"], nguards=3, nox=wl["order"], particle_pusher=wl["pusher"],
                     engine="tiled", precision=args.precision, tiled_config=cfg)
    stream = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    _barrier(ws)
    w0 = time.perf_counter()
    ev[0].record(stream)
    m.add_species("electron", -1.0, 1.0, host["x"], host["y"], host["z"], host["ux"],
                  host["uy"], host["uz"], host["w"])
    ev[1].record(stream)
    for s_ in range(args.steps):
        m.step(1)
        diag_host[s_].copy_(m.diagnostics(gauss=False, to_host=False), non_blocking=True)
    ev[2].record(stream)
    sp = m.species[0]
    for c in out_cols:
        out_host[c].copy_(getattr(sp, c), non_blocking=True)
    ev[3].record(stream)
    _barrier(ws)
    wall = time.perf_counter() - w0
    ms = _max_over_ranks(ev[0].elapsed_time(ev[3]), ws)
    phases = {"add_species_ms": ev[0].elapsed_time(ev[1]),
              "steps_ms": ev[1].elapsed_time(ev[2]),
              "download_ms": ev[2].elapsed_time(ev[3])}
    del m
    torch.cuda.empty_cache()
    h2d = 7 * 8 * N
    d2h = len(out_cols) * 8 * N + args.steps * 9 * 8
    # the host link: pinned copies of 1 GiB each way; the end-to-end bound is
    # the steps plus both transfers at that bandwidth, with nothing overlapped
    bw = _pcie_gbs()
    bound_s = phases["steps_ms"] * 1e-3 + h2d / (bw["h2d_gbs"] * 1e9) + d2h / (bw["d2h_gbs"] * 1e9)
    bound = N * ws * args.steps / bound_s
    value = N * ws * args.steps / (ms * 1e-3)
    return {"value": value, "unit": "particle-steps/s",
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
            "ms": ms, "wall_s": wall, "phases": phases, "host_link": bw,
            "transfer_bound_value": bound, "frac_of_transfer_bound": value / bound,
            "what": "job through PicsarModule(engine='tiled'): PICSAR FP64 particle arrays "
                    "from pinned host memory (add_species), every step with its FP64 energies "
                    "copied to the host, final x, y, z, u, gamma^-1 arrays copied to the host"}


def _pcie_gbs(nbytes=1 << 30, reps=3):
    """Pinned host <-> device copy bandwidth (GB/s) of this GPU's host link,
    best of `reps` copies of `nbytes` each way (CUDA events)."""
    import torch
    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream()
    out = {}
    for name, dst, src in (("h2d_gbs", d, h), ("d2h_gbs", h, d)):
        best = None
        for _ in range(reps + 1):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            dst.copy_(src, non_blocking=True)
            b.record(s)
            b.synchronize()
            t = a.elapsed_time(b)
            best = t if best is None else min(best, t)
        out[name] = nbytes / (best * 1e-3) / 1e9
    del h, d
    return out


def run_plain_fp64(wl, args, ws, rank):
    """The plain FP64 GPU path (PICSAR arrays, FP64 atomics) on the workload."""
    import torch
    from picsar_b200.init import thermal_plasma
    from picsar_b200.picsar import PicsarModule
    st = _initial_state(wl, 1234 + rank)
    m = PicsarModule(*wl["n"], nguards=3, nox=wl["order"], particle_pusher=wl["pusher"])
    m.add_species("electron", -1.0, 1.0, st.x, st.y, st.z, st.ux, st.uy, st.uz, st.w)
    N = st.np
    del st
    m.step(1)
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    _barrier(ws)
    a.record(stream)
    m.step(args.fp64_steps)
    b.record(stream)
    _barrier(ws)
    ms = _max_over_ranks(a.elapsed_time(b), ws)
    del m
    torch.cuda.empty_cache()
    return {"value": N * ws * args.fp64_steps / (ms * 1e-3), "unit": "particle-steps/s",
            "steps": args.fp64_steps, "ms_per_step": ms / args.fp64_steps,
            "what": "plain FP64 GPU path: PICSAR guarded FP64 arrays, one thread per "
                    "particle, global FP64 atomics, separate bc kernels"}


def run_tiled_fp64(wl, args, ws, rank, cfg):
    """The tiled engine in FP64 on the workload: steps and particle-kernel
    time (CUDA events), with the kernel's HBM roofline (FP64 layout: 60 B
    read + 52 B written per particle, 96 B per cell)."""
    import torch
    from picsar_b200.tiled import SUPPORTED_SHAPES_FP64, TiledConfig, TiledSim
    c64 = TiledConfig(tile=cfg.tile, drift=min(cfg.drift, 1), threads=cfg.threads,
                      sort_interval=cfg.sort_interval, relayout_interval=0)
    if (c64.tile[0], c64.drift) not in SUPPORTED_SHAPES_FP64:
        return None
    st = _initial_state(wl, 1234 + rank)
    N = st.np
    t = TiledSim(wl["n"], order=wl["order"], pusher=wl["pusher"], precision="fp64", config=c64)
    t.load_state(st)
    del st
    t.step(2)
    steps = max(args.fp64_steps, 4)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    _barrier(ws)
    a.record(stream)
    for s_ in range(steps):
        t.step(1, events=ev[s_])
    b.record(stream)
    _barrier(ws)
    ms = _max_over_ranks(a.elapsed_time(b), ws)
    kern = sum(x.elapsed_time(y) for x, y in ev) / steps
    del t
    torch.cuda.empty_cache()
    peak, peak_kind = _peaks()
    ncell = wl["n"][0] * wl["n"][1] * wl["n"][2]
    alg = BYTES_PER_PARTICLE[1] * N + GRID_BYTES_PER_CELL[1] * ncell
    return {"value": N * ws * steps / (ms * 1e-3), "unit": "particle-steps/s", "steps": steps,
            "ms_per_step": ms / steps, "kernel_ms": kern,
            "roofline": {"bound": "hbm", "achieved": alg / (kern * 1e-3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": alg / (kern * 1e-3) / 1e9 / peak,
                         "peak_kind": peak_kind, "algorithmic_bytes_per_launch": alg},
            "threads": c64.fp64_threads,
            "what": "tiled engine in FP64 (within 1e-12 of the oracle), same tiles and sort "
                    "interval, no re-layout (the FP64 kernel makes one pass), one CTA per SM"}


def _plain_fp64_jobs(specs, steps=2):
    """Plain FP64 GPU path, one job at a time (PICSAR arrays, FP64 atomics):
    per job its setup (initial state, module, add_species; host wall clock
    between device synchronisations), its first step and then `steps` more
    steps (CUDA events).  Returns (particle-steps/s of the timed steps over
    all jobs, {index: ms per step}, {index: seconds of setup and first step
    beyond one step})."""
    import torch
    from picsar_b200.picsar import PicsarModule
    per, extra, tot_ps, tot_ms = {}, {}, 0, 0.0
    s = torch.cuda.current_stream()
    for i, sp in enumerate(specs):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = sp.initial_state(device="cuda")
        m = PicsarModule(*sp.n, nguards=3, nox=sp.order, particle_pusher=sp.pusher)
        m.add_species("electron", -1.0, 1.0, st.x, st.y, st.z, st.ux, st.uy, st.uz, st.w)
        del st
        torch.cuda.synchronize()
        setup_s = time.perf_counter() - t0
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record(s)
        m.step(1)
        ev[1].record(s)
        m.step(steps)
        ev[2].record(s)
        torch.cuda.synchronize()
        ms = ev[1].elapsed_time(ev[2])
        per[i] = ms / steps
        extra[i] = setup_s + max(0.0, ev[0].elapsed_time(ev[1]) - per[i]) * 1e-3
        tot_ps += sp.particles * steps
        tot_ms += ms
        del m
    torch.cuda.empty_cache()
    return tot_ps / (tot_ms * 1e-3), per, extra


def _tuned_configs(specs, precision="fp32", acc=2):
    from picsar_b200 import autotune
    t0 = time.perf_counter()
    tuned = autotune.tune_ensemble(specs, precision, acc=acc)
    dt = time.perf_counter() - t0
    info = {str(o): {"tile": r.config.tile[0], "drift": r.config.drift,
                     "threads": r.config.threads, "sort_interval": r.config.sort_interval,
                     "relayout_interval": r.config.relayout_interval,
                     "select_lanes": r.config.select_lanes,
                     "proxy_rate": r.rate, "ppc": r.ppc, "sigma": r.sigma, "cached": r.cached}
            for o, r in tuned.items()}
    return {o: r.config for o, r in tuned.items()}, info, dt


def _with_acc(configs, acc):
    """Configs with the requested FP32 accumulator mode where their shape
    has it compiled (autotune.acc_for)."""
    from picsar_b200.autotune import acc_for
    from picsar_b200.tiled import TiledConfig
    out = {}
    for o, c in configs.items():
        a = acc_for(c.tile[0], c.drift, acc, o)
        out[o] = TiledConfig(tile=c.tile, drift=c.drift, threads=c.threads,
                             ctas_per_sm=c.ctas_per_sm, sort_interval=c.sort_interval, acc=a,
                             relayout_interval=c.relayout_interval,
                             select_lanes=c.select_lanes)
    return out


def _ensemble_accuracy(specs, configs, steps):
    """The same jobs as an FP32 mixed and as an FP64 ensemble: per job the
    total-energy drift from step 1 to the last step and the Gauss-law
    residual at the end, FP32 against FP64."""
    import torch
    from picsar_b200.ensemble import Ensemble
    out = {}
    for prec, cfg in (("fp32", configs), ("fp64", None)):
        ens = Ensemble(specs, prec, cfg)
        g0 = [d["gauss_norm"] for d in ens.diagnostics(gauss=True)]
        ens.step(1)
        d1 = ens.diagnostics()
        ens.step(steps - 1)
        d2 = ens.diagnostics(gauss=True)
        order = [id(sp) for sp, _ in ens.sims()]
        out[prec] = {k: (abs((b["total"] - a["total"]) / a["total"]), b["gauss_norm"], g)
                     for k, a, b, g in zip(order, d1, d2, g0)}
        del ens
        torch.cuda.empty_cache()
    keys = list(out["fp64"])
    er = [out["fp32"][k][0] / max(out["fp64"][k][0], 1e-300) for k in keys]
    gr = [out["fp32"][k][1] / out["fp64"][k][1] for k in keys]
    return {"jobs": len(keys), "steps": steps,
            "energy_drift_fp32_median": float(statistics.median(out["fp32"][k][0] for k in keys)),
            "energy_drift_fp64_median": float(statistics.median(out["fp64"][k][0] for k in keys)),
            "energy_drift_ratio_median": float(statistics.median(er)),
            "energy_drift_ratio_max": float(max(er)),
            "jobs_within_2x_fp64_energy_drift": int(sum(
                out["fp32"][k][0] <= 2 * out["fp64"][k][0] + 1e-7 for k in keys)),
            "gauss_residual_ratio_max": float(max(gr)),
            "gauss_residual_ratio_min": float(min(gr))}


def _ensemble_measure(specs, configs, steps, warmup, ws, fp64_jobs, accuracy=True):
    """The batched ensemble of `specs`: `warmup` untimed steps, `steps` timed
    steps (CUDA events, max over ranks), the particle kernels' roofline, the
    energy drift over the timed steps and the plain FP64 path on a sample of
    `fp64_jobs` jobs run one at a time.  Returns a dict."""
    import torch
    from picsar_b200.ensemble import Ensemble
    local = torch.cuda.current_device()
    ens = Ensemble(specs, "fp32", configs)
    N = ens.particles_total
    ens.step(warmup)
    # kinetic energy is summed per tile by the particle kernel: read it after a step
    d0 = ens.diagnostics()
    pk_ms, yee_ms = ens.profile_steps(2)
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    l0 = ens.launches
    _barrier(ws)
    clocks.start()
    a.record(stream)
    ens.step(steps)
    b.record(stream)
    _barrier(ws)
    clk = clocks.stop()
    ms = _max_over_ranks(a.elapsed_time(b), ws)
    launches = ens.launches - l0
    d1 = ens.diagnostics()
    drift = [(y["total"] - x["total"]) / x["total"] for x, y in zip(d0, d1)]
    value = N * ws * steps / (ms * 1e-3)
    peak, peak_kind = _peaks()
    alg = ens.algorithmic_bytes()
    achieved = alg / (pk_ms * 1e-3) / 1e9
    flags = ens.error_flags()
    slow = ens.slow_path_count()
    del ens
    torch.cuda.empty_cache()
    acc = None
    if accuracy:
        acc = _ensemble_accuracy(specs[::8][:32], configs, steps + warmup)
    fp64 = None
    if fp64_jobs > 0:
        sample = specs[::max(1, len(specs) // fp64_jobs)][:fp64_jobs]
        rate64, _, _ = _plain_fp64_jobs(sample, steps=2)
        fp64 = {"value": rate64 * ws, "unit": "particle-steps/s", "jobs_sampled": len(sample),
                "what": "plain FP64 GPU path, jobs launched one at a time (sampled jobs, "
                        "2 timed steps each after 1 untimed)"}
    return {
        "value": value, "unit": "particle-steps/s", "steps": steps, "warmup": warmup,
        "ms_per_step": ms / steps, "particles": N, "jobs": len(specs),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None,
                     "kernel": "k_tile_step (one launch per order group)",
                     "kernel_ms": pk_ms, "yee_ms": yee_ms, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": alg},
        "gpu_launches": launches, "clocks": clk, "fp64_plain": fp64,
        "speedup_vs_fp64_plain": value / fp64["value"] if fp64 else None,
        "energy_drift": {"median_abs": float(statistics.median(abs(x) for x in drift)),
                         "max_abs": float(max(abs(x) for x in drift))},
        "error_flags": int(sum(flags)), "slow_path_particle_steps": slow,
        "accuracy": acc,
    }


ENSEMBLE_DESC = ("uneven periodic thermal-plasma jobs (cells/axis U{16..96}, ppc {1,2,4,8,16}, "
                 "order {1,2,3}, u_th log-U[0.001,0.05]), one batched step per iteration "
                 "replayed from CUDA graphs")


def run_ensemble(args):
    """Batched ensemble of uneven jobs (256 periodic thermal plasmas, cells
    per axis U{16..96}, ppc in {1,2,4,8,16}, order in {1,2,3}, u_th
    log-uniform 0.001-0.05, 100 steps each) in one persistent kernel set
    replayed from CUDA graphs; autotuned per order; compared with the plain
    FP64 path run job by job."""
    import torch
    from picsar_b200.ensemble import ensemble_jobs
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    specs = ensemble_jobs(count=args.jobs, seed=2024 + rank, steps=args.steps + args.warmup)
    configs, tune_info, tune_s = _tuned_configs(specs, acc=args.acc)
    configs = _with_acc(configs, args.acc)
    for o, c in configs.items():
        tune_info[str(o)]["acc"] = c.acc
    r = _ensemble_measure(specs, configs, args.steps, args.warmup, ws,
                          0 if args.skip_fp64 else args.fp64_jobs,
                          accuracy=not args.skip_accuracy)
    if rank == 0:
        line = {
            "metric": "particle-steps/s", "value": r["value"], "unit": "particle-steps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"ensemble: {len(specs)} {ENSEMBLE_DESC}",
                       "particles_per_gpu": r["particles"], "jobs": len(specs),
                       "precision": "FP32 mixed (FP64 J flush and energy sums)",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "l2": "inputs larger than L2 (particle SoA "
                             f"{r['particles'] * 32 / 1e9:.1f} GB), no flush",
                       "autotuned": tune_info, "autotune_seconds": tune_s},
            "cpu_baseline": None, "e2e": None,
            **{k: r[k] for k in ("roofline", "gpu_launches", "clocks", "fp64_plain",
                                 "speedup_vs_fp64_plain", "energy_drift", "error_flags",
                                 "slow_path_particle_steps", "accuracy")},
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def _serve_measure(specs, configs, rates, hbm_budget_gb, fifo_rate):
    """The served stream of `specs` at each Poisson rate (jobs/s, arrivals
    seeded by the rate), continuously batched, against the one-at-a-time
    plain FP64 FIFO model built from each job's measured service time, and
    the FIFO stream actually served at `fifo_rate` (None: not served).
    Returns a dict."""
    import torch
    from picsar_b200.ensemble import ensemble_jobs
    from picsar_b200.serve import (Server, fifo_latencies, percentile, poisson_requests,
                                   serve_fifo_plain)
    local = torch.cuda.current_device()
    # warm-up: a few short jobs through the server (kernel attributes, pools)
    # and the initial states of the stream's largest jobs (the generator's
    # kernels for those sizes load on first use)
    warm = ensemble_jobs(count=6, seed=5, steps=3, cells=(16, 24))
    Server("fp32", configs=configs).run(poisson_requests(warm, 1e6), clock="wall")
    for sp in sorted(specs, key=lambda x: -x.particles)[:4]:
        sp.initial_state(device="cuda")
    # per job the plain FP64 service time: setup and first step, then its
    # remaining steps at the measured time per step
    _, per_ms, extra_s = _plain_fp64_jobs(specs, steps=2)
    service = {i: extra_s[i] + per_ms[i] * specs[i].steps / 1e3 for i in range(len(specs))}
    work = sum(sp.particles * sp.steps for sp in specs)
    sweep = []
    clocks = ClockSampler(local)
    clocks.start()
    for lam in rates:
        reqs = poisson_requests(specs, lam, seed=1000 + int(round(lam)))
        rep = Server("fp32", hbm_budget=int(hbm_budget_gb * 1e9), configs=configs).run(reqs)
        s = rep.summary()
        fifo = fifo_latencies(reqs, service)
        fl = list(fifo.values())
        fifo_span = max(r.arrival + fifo[r.rid] for r in reqs)
        sweep.append({"rate_jobs_per_s": lam, **s,
                      "fp64_fifo": {"p50_latency_s": percentile(fl, 50),
                                    "p99_latency_s": percentile(fl, 99),
                                    "particle_steps_per_s": work / fifo_span}})
    clk = clocks.stop()
    fifo_served = None
    if fifo_rate:
        # the one-at-a-time FP64 stream actually served at one rate, against
        # the model built from the separately measured service times
        reqs = poisson_requests(specs, fifo_rate, seed=2000)
        srep = serve_fifo_plain(reqs).summary()
        fifo = fifo_latencies(reqs, service)
        fl = list(fifo.values())
        fifo_served = {"rate_jobs_per_s": fifo_rate, "served": srep,
                       "model": {"p50_latency_s": percentile(fl, 50),
                                 "p99_latency_s": percentile(fl, 99)},
                       "p50_served_over_model": srep["p50_latency_s"] / percentile(fl, 50)}
    return {"sweep": sweep, "clocks": clk, "fp64_service_s_total": sum(service.values()),
            "fp64_fifo_served": fifo_served}


SERVE_DESC = ("jobs per rate from the ensemble distribution, steps U{50..500}, Poisson "
              "arrivals, continuous batching")


def run_serve(args):
    """Served stream: Poisson arrivals at each rate of --rates (jobs/s) of
    jobs from the ensemble distribution with steps U{50..500}, admitted by
    an HBM budget, continuously batched; p50/p99 latency and throughput,
    against one-job-at-a-time plain FP64 execution (FIFO) of the same
    stream, each job's service time measured on the plain FP64 path."""
    import torch
    from picsar_b200.ensemble import ensemble_jobs
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    rates = [float(x) for x in args.rates.split(",")]
    specs = ensemble_jobs(count=args.jobs, seed=77 + rank, steps_range=(50, 500))
    configs, tune_info, tune_s = _tuned_configs(specs, acc=args.acc)
    configs = _with_acc(configs, args.acc)
    for o, c in configs.items():
        tune_info[str(o)]["acc"] = c.acc
    r = _serve_measure(specs, configs, rates, args.hbm_budget, args.fifo_rate)
    if rank == 0:
        top = max(r["sweep"], key=lambda x: x["particle_steps_per_s"])
        line = {
            "metric": "particle-steps/s", "value": top["particle_steps_per_s"] * ws,
            "unit": "particle-steps/s", "n_gpus": ws, "steps": None, "warmup": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"served stream: {len(specs)} {SERVE_DESC}, HBM budget "
                                   f"{args.hbm_budget:g} GB",
                       "rates_jobs_per_s": rates, "autotuned": tune_info,
                       "autotune_seconds": tune_s},
            **r,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def _workload_legs(args):
    """Compact single-GPU measurements of the other workloads, reported in
    the default line: the ensemble (256 jobs, 20 timed steps, plain FP64 on
    24 sampled jobs), the served stream (48 jobs at 50 and 200 jobs/s, the
    FIFO FP64 stream served at 50 jobs/s) and the uneven-density workload
    (20 timed steps, plain FP64 on the same state).  A leg that raises
    reports its error instead of a number."""
    import copy
    import torch
    from picsar_b200.ensemble import ensemble_jobs
    out = {}

    def leg(name, fn):
        t0 = time.perf_counter()
        try:
            out[name] = fn()
        except Exception as e:                      # report, keep the headline
            out[name] = {"error": repr(e)[:400]}
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        out[name]["leg_seconds"] = time.perf_counter() - t0

    state = {}

    def ensemble():
        specs = ensemble_jobs(count=256, seed=2024, steps=23)
        configs, tune_info, tune_s = _tuned_configs(specs, acc=args.acc)
        configs = _with_acc(configs, args.acc)
        state["configs"] = configs
        r = _ensemble_measure(specs, configs, 20, 3, 1, 24, accuracy=False)
        r["workload"] = f"ensemble: 256 {ENSEMBLE_DESC}"
        r["autotune_seconds"] = tune_s
        return r

    def serve():
        specs = ensemble_jobs(count=48, seed=77, steps_range=(50, 500))
        configs = state.get("configs")
        if configs is None:
            configs = _with_acc(_tuned_configs(specs, acc=args.acc)[0], args.acc)
        r = _serve_measure(specs, configs, [50.0, 200.0], args.hbm_budget, 50.0)
        r["workload"] = f"served stream: 48 {SERVE_DESC}, HBM budget {args.hbm_budget:g} GB"
        return r

    def uneven():
        a = copy.copy(args)
        a.workload, a.steps, a.warmup = "uneven", 20, 3
        a.skip_e2e = a.skip_cpu = a.skip_accuracy = a.skip_fp64_tiled = True
        a.skip_workloads = True
        r = run_ours(a, emit=False)
        keep = ("value", "unit", "ms_per_step", "steps", "warmup", "roofline", "fp64_plain",
                "gpu_launches", "clocks", "slow_path_particle_steps", "deferred_fraction")
        d = {k: r[k] for k in keep}
        d["workload"] = r["config"]["workload"]
        d["tuning"] = r["config"]["tuning"]
        d["tile_occupancy"] = r["config"]["tile_occupancy"]
        d["speedup_vs_fp64_plain"] = (r["value"] / r["fp64_plain"]["value"]
                                      if r.get("fp64_plain") else None)
        return d

    leg("ensemble", ensemble)
    leg("serve", serve)
    leg("uneven", uneven)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large",
                    choices=sorted(WORKLOADS) + ["ensemble", "serve"])
    ap.add_argument("--jobs", type=int, default=None, help="ensemble / served jobs")
    ap.add_argument("--fp64-jobs", type=int, default=24)
    ap.add_argument("--rates", default="10,20,50,100,200")
    ap.add_argument("--hbm-budget", type=float, default=150.0, help="GB")
    ap.add_argument("--fifo-rate", type=float, default=50.0,
                    help="rate (jobs/s) of the served one-at-a-time FP64 baseline")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--threads", type=int, default=256)
    ap.add_argument("--ctas-per-sm", type=int, default=2)
    ap.add_argument("--relayout", type=int, default=4,
                    help="bank re-layout interval between sorts (0: none), fixed workloads")
    ap.add_argument("--acc", type=int, default=1,
                    help="FP32 current accumulator: 1 int32 fixed point (default: energy drift "
                         "and Gauss residual within 1e-3 of FP64's, one-step field error "
                         "~1e-4), 2 two-word 64-bit fixed point (~1e-5, slower), 0 FP32")
    ap.add_argument("--select-lanes", type=int, default=1, choices=[0, 1],
                    help="FP32 particle kernel: lanes of distinct bank classes per warp with a "
                         "second pass for the others (1) or one pass (0), fixed workloads")
    ap.add_argument("--fp64-steps", type=int, default=3)
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-accuracy", action="store_true")
    ap.add_argument("--skip-workloads", action="store_true",
                    help="leave out the compact ensemble / serve / uneven legs of the "
                         "default line")
    ap.add_argument("--accuracy-steps", type=int, default=200)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.steps is None:
        args.steps = {"ensemble": 95, "uneven": 500}.get(args.workload, 200)
    if args.jobs is None:
        args.jobs = 256 if args.workload == "ensemble" else 48
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "ensemble":
        return run_ensemble(args)
    if args.workload == "serve":
        return run_serve(args)
    run_ours(args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
