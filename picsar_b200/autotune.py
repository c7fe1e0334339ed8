"""Autotuner of the tiled engine: cell-tile shape (edge and window margin),
threads per tile CTA, sort interval and bank re-layout interval, chosen by
timing.

For a (shape order, precision, particles per cell, thermal spread, beam
drift) class of jobs, a proxy simulation large enough to occupy every SM (at least two tiles
per resident CTA) is stepped under each candidate and timed with CUDA events
on the launching stream.  Stage 1 times every compiled (tile edge, margin)
pair at both thread counts (FP64: 256 and 512 threads, one CTA per SM)
over 20 steps with a sort every 5 steps; stage 2
times the two best at each pair of sort interval and bank re-layout interval
over 40 steps (the slow path for particles that drifted out of their tile
window, the bank conflicts of particles that changed cell, and the sorts
and re-layouts themselves all count); stage 3 (FP32) times the winner
without the bank-class lane selection.  Results are cached per GPU model in
a JSON file (``$PICSAR_B200_CACHE`` or ``~/.cache/picsar_b200/autotune.json``).

The reference has no autotuner: its tile counts, vector lengths and
sorting period are deck parameters (src/parallelization/tiling/tiling.F90,
src/housekeeping/sorting.F90).
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import asdict, dataclass, field, replace

import torch

from .init import thermal_plasma
from ._lib import PicsarB200Error
from .tiled import SUPPORTED_ACC, SUPPORTED_SHAPES, TiledConfig, TiledSim

THREADS = (128, 256)
THREADS_FP64 = (256, 512)     # the FP64 engine runs one CTA per SM
SORT_INTERVALS = (5, 10, 20, 40)
RELAYOUT_INTERVALS = (0, 2, 4)


@dataclass
class TuneResult:
    order: int
    precision: str
    ppc: int
    sigma: float
    config: TiledConfig
    rate: float                     # particle-steps/s of the winner on the proxy
    table: list = field(default_factory=list)   # (tile, drift, threads, sort, relayout, rate)
    cached: bool = False


def _cache_path():
    p = os.environ.get("PICSAR_B200_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "picsar_b200", "autotune.json")


def _key(order, precision, ppc, sigma, pusher, u_drift=0.0, device_name=None, acc=2):
    """Cache key of a job class: GPU model, order, precision, ppc, thermal
    spread in half-decades, beam drift (2 decimals), pusher, FP32 current
    accumulator."""
    name = device_name or torch.cuda.get_device_name()
    sb = round(math.log10(max(sigma, 1e-6)) * 2) / 2
    db = f"|d{round(u_drift, 2)}" if u_drift else ""
    ab = f"|a{acc}" if precision == "fp32" else ""
    return f"{name}|o{order}|{precision}|ppc{ppc}|s{sb}{db}|p{pusher}{ab}|v7"


def acc_for(edge, drift, acc, order=3):
    """The FP32 accumulator a (tile edge, margin) shape runs with when `acc`
    is asked for: `acc` where that shape has it compiled, else the two-word
    mode every shape has.  Mode 4 (the cell-grouped kernel, shape orders 1
    and 3) falls back to mode 1, the same int32 accumulator with one
    particle per thread."""
    if acc == 4 and order == 2:
        acc = 1
    ok = SUPPORTED_ACC.get((edge, drift), (2,))
    if acc in ok:
        return acc
    return 1 if acc == 4 and 1 in ok else 2


def proxy_grid(ppc, num_sms, tile=8, ctas_per_sm=2):
    """Smallest grid of whole 8^3 tiles with at least two tiles per resident
    CTA, x and y equal, at most ~12 M particles."""
    need = 2 * num_sms * ctas_per_sm
    nz_t = 8
    nxy_t = max(4, math.ceil(math.sqrt(need / nz_t)))
    n = (nxy_t * tile, nxy_t * tile, nz_t * tile)
    while n[0] * n[1] * n[2] * ppc > 12_000_000 and n[2] > 16:
        n = (n[0], n[1], n[2] // 2)
    return n


def _time(cfg, order, precision, st, n, steps, pusher):
    sim = TiledSim(n, order=order, pusher=pusher, precision=precision, config=cfg)
    sim.load_state(st)
    sim.step(2)                                    # warm-up (kernel attributes)
    s = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(s)
    sim.step(steps)
    b.record(s)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    rate = sim.np * steps / (ms * 1e-3)
    del sim
    return rate


def tune(order, precision="fp32", ppc=8, sigma=0.01, pusher=0, use_cache=True,
         shapes=None, threads=THREADS, sort_intervals=SORT_INTERVALS,
         relayout_intervals=RELAYOUT_INTERVALS, seed=7, u_drift=0.0, acc=2):
    """Best TiledConfig for jobs of this class, timed on a proxy simulation
    (thermal spread sigma; u_drift > 0: two counter-streaming beams u_x =
    +-u_drift, as in a two-stream plasma).  acc: the FP32 current
    accumulator the jobs will run with; every candidate is timed with it
    (acc_for) and the returned config carries it."""
    path = _cache_path()
    key = _key(order, precision, ppc, sigma, pusher, u_drift, acc=acc)
    if use_cache and os.path.exists(path):
        try:
            with open(path) as f:
                c = json.load(f).get(key)
            if c:
                cfg = TiledConfig(**{**c["config"], "tile": tuple(c["config"]["tile"])})
                return TuneResult(order, precision, ppc, sigma, cfg, c["rate"], c["table"],
                                  cached=True)
        except (OSError, ValueError, TypeError, KeyError):
            pass
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    n = proxy_grid(ppc, props.multi_processor_count)
    st = thermal_plasma(n, ppc, sigma, seed=seed, device="cuda")
    if u_drift:
        st.ux[0::2] += u_drift
        st.ux[1::2] -= u_drift
    if shapes is None:
        shapes = sorted(SUPPORTED_SHAPES)
    table = []
    ranked = []
    fp64 = precision == "fp64"
    for edge, drift in shapes:
        for th in (THREADS_FP64 if fp64 and threads == THREADS else threads):
            # a short sort interval, so that shapes are ranked by the kernel
            # rather than by the slow path of particles that left their window
            cfg = TiledConfig(tile=(edge, edge, edge), drift=drift, sort_interval=5,
                              relayout_interval=0, acc=acc_for(edge, drift, acc, order),
                              **({"fp64_threads": th} if fp64 else {"threads": th}))
            try:
                r = _time(cfg, order, precision, st, n, 20, pusher)
            except (ValueError, RuntimeError, PicsarB200Error) as e:   # not compiled here
                table.append((edge, drift, th, 5, 0, None, str(e)[:80]))
                continue
            table.append((edge, drift, th, 5, 0, r))
            ranked.append((r, cfg))
    # stage 2 for the two best (shape, threads) pairs of stage 1: a shape that
    # loses at the stage-1 sort interval can win at another
    ranked.sort(key=lambda rc: -rc[0])
    best = None
    for _, cfg0 in ranked[:2]:
        for K in sort_intervals:
            for R in relayout_intervals:
                if R >= K:
                    continue
                cfg = replace(cfg0, sort_interval=K, relayout_interval=R)
                r = _time(cfg, order, precision, st, n, 40, pusher)
                th = cfg0.fp64_threads if fp64 else cfg0.threads
                table.append((cfg0.tile[0], cfg0.drift, th, K, R, r))
                if best is None or r > best[1]:
                    best = (cfg, r)
    # stage 3 (FP32): the winner in one pass, without the bank-class lane
    # selection (it costs a second pass, which loses where many particles
    # change cell every step)
    if precision == "fp32":
        c1 = best[0]
        cfg = replace(c1, select_lanes=False)
        r = _time(cfg, order, precision, st, n, 40, pusher)
        table.append((c1.tile[0], c1.drift, c1.threads, c1.sort_interval, c1.relayout_interval,
                      r, "one pass"))
        if r > best[1]:
            best = (cfg, r)
    res = TuneResult(order, precision, ppc, sigma, best[0], best[1], table)
    if use_cache:
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            data = {}
            if os.path.exists(path):
                with open(path) as f:
                    data = json.load(f)
            data[key] = {"config": asdict(res.config), "rate": res.rate, "table": table}
            with open(path, "w") as f:
                json.dump(data, f, indent=1)
        except (OSError, ValueError):
            pass
    return res


def representative(specs):
    """Per shape order: the particle-weighted median ppc and the 90th
    percentile thermal spread of the jobs (the drift out of tile windows is
    set by the fast tail)."""
    out = {}
    for o in (1, 2, 3):
        js = [s for s in specs if s.order == o]
        if not js:
            continue
        js_ppc = sorted(js, key=lambda s: s.ppc)
        tot = sum(s.particles for s in js)
        acc, ppc = 0, js_ppc[-1].ppc
        for s in js_ppc:
            acc += s.particles
            if acc >= tot / 2:
                ppc = s.ppc
                break
        sig = sorted(s.sigma for s in js)
        out[o] = (ppc, sig[min(len(sig) - 1, int(0.9 * len(sig)))], js[0].pusher)
    return out


def tune_ensemble(specs, precision="fp32", use_cache=True, acc=2):
    """{order: TiledConfig} for an ensemble, one tuning per order present."""
    res = {}
    for o, (ppc, sig, pusher) in representative(specs).items():
        res[o] = tune(o, precision, ppc=ppc, sigma=sig, pusher=pusher, use_cache=use_cache,
                      acc=acc)
    return res
