"""Batched ensembles (many simulations in one set of launches, CUDA graphs)
against the same jobs run one at a time, through the C ABI.

FP64: every job of the ensemble equals the same job stepped alone (and the
oracle) to 1e-12 relative L2 in E, B, J and particle momenta.  FP32 mixed:
within 1e-5 of the job stepped alone (the only difference is the order of
the FP64 flush atomics of overlapping tile windows).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from picsar_b200.ensemble import Ensemble, JobSpec, ensemble_jobs
from picsar_b200.tiled import TiledConfig, TiledSim
from tests._cases import rel_l2

pytestmark = pytest.mark.gpu

SPECS = [
    JobSpec(n=(16, 24, 16), ppc=2, sigma=0.05, order=1, pusher=0, steps=6, seed=11),
    JobSpec(n=(24, 16, 20), ppc=4, sigma=0.02, order=2, pusher=1, steps=6, seed=12),
    JobSpec(n=(16, 16, 16), ppc=1, sigma=0.05, order=3, pusher=0, steps=6, seed=13),
    JobSpec(n=(20, 16, 24), ppc=3, sigma=0.01, order=1, pusher=1, steps=6, seed=14),
    JobSpec(n=(16, 20, 16), ppc=2, sigma=0.03, order=3, pusher=1, steps=6, seed=15),
]


def _alone(spec, prec, cfg):
    t = TiledSim(spec.n, order=spec.order, pusher=spec.pusher, precision=prec, config=cfg,
                 track_ids=True)
    t.load_state(spec.initial_state())
    t.step(spec.steps, keep_j=False)
    return t


def _cmp(a, b, tol):
    for name in ("ex", "ey", "ez", "bx", "by", "bz"):
        e = rel_l2(a.export_field(name, 3).cpu().numpy(), b.export_field(name, 3).cpu().numpy())
        assert e <= tol, (name, e)
    pa = {k: v.cpu().numpy() for k, v in a.particles().items()}
    pb = {k: v.cpu().numpy() for k, v in b.particles().items()}
    assert np.array_equal(pa["id"], pb["id"])
    for c in ("ux", "uy", "uz", "gaminv"):
        e = rel_l2(pa[c], pb[c])
        assert e <= tol, (c, e)


@pytest.mark.parametrize("use_graph", [True, False])
def test_ensemble_fp64_matches_jobs_alone(cuda, use_graph):
    cfg = TiledConfig(tile=(8, 8, 8), sort_interval=2)
    ens = Ensemble(SPECS, precision="fp64", configs={1: cfg, 2: cfg, 3: cfg}, track_ids=True,
                   use_graph=use_graph)
    ens.step(6)
    torch.cuda.synchronize()
    assert all(f == 0 for f in ens.error_flags())
    for spec, sim in ens.sims():
        _cmp(sim, _alone(spec, "fp64", cfg), 1e-12)


def test_ensemble_fp64_matches_oracle(cuda):
    spec = SPECS[1]
    cfg = TiledConfig(tile=(8, 8, 8), sort_interval=3)
    ens = Ensemble(SPECS[:3], precision="fp64", configs={1: cfg, 2: cfg, 3: cfg},
                   track_ids=True)
    ens.step(3)
    st = spec.initial_state(device="cuda").numpy()     # the ensemble draws it on the device
    o = O.OracleSim(spec.n, 3, order=spec.order, pusher=spec.pusher)
    o.add_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    o.step(3)
    sim = [s for sp, s in ens.sims() if sp is spec][0]
    for name in ("ex", "ey", "ez", "bx", "by", "bz"):
        e = rel_l2(sim.export_field(name, 3).cpu().numpy(), o.get_field(name))
        assert e <= 1e-12, (name, e)
    got = {k: v.cpu().numpy() for k, v in sim.particles().items()}
    ref = o.particles()
    for c in ("ux", "uy", "uz"):
        assert rel_l2(got[c], ref[c]) <= 1e-12, c


def test_ensemble_fp32_matches_jobs_alone(cuda):
    cfgs = {1: TiledConfig(tile=(8, 8, 8), sort_interval=2),
            2: TiledConfig(tile=(8, 8, 8), drift=2, threads=128, sort_interval=3),
            3: TiledConfig(tile=(4, 4, 4), drift=1, sort_interval=2)}
    ens = Ensemble(SPECS, precision="fp32", configs=cfgs, track_ids=True)
    ens.step(6)
    for spec, sim in ens.sims():
        _cmp(sim, _alone(spec, "fp32", cfgs[spec.order]), 1e-5)


@pytest.mark.parametrize("use_graph", [True, False])
def test_ensemble_cell_groups_match_jobs_alone(cuda, use_graph):
    """Orders 1 and 3 on the cell-grouped kernel (accumulator mode 4) in a
    batch: the batched sort keeps each job's cell order, the batched step
    launches the kernel's CTA size and skips the bank re-layout, and every
    job ends where it does alone (to the order of the FP64 flush atomics)."""
    cell = TiledConfig(tile=(8, 8, 8), drift=1, acc=4, sort_interval=2, relayout_interval=1)
    cfgs = {1: cell, 2: TiledConfig(tile=(8, 8, 8), sort_interval=3), 3: cell}
    ens = Ensemble(SPECS, precision="fp32", configs=cfgs, track_ids=True, use_graph=use_graph)
    ens.step(6)
    torch.cuda.synchronize()
    assert all(f == 0 for f in ens.error_flags())
    for spec, sim in ens.sims():
        _cmp(sim, _alone(spec, "fp32", cfgs[spec.order]), 1e-5)


def test_batched_sort_layout_matches_single_job_sort(cuda):
    """After one batched sort every job has the same tile offsets and the
    same set of particles per tile as after its own single-job sort."""
    cfg = TiledConfig(tile=(8, 8, 8), sort_interval=1)
    ens = Ensemble(SPECS, precision="fp32", configs={1: cfg, 2: cfg, 3: cfg}, track_ids=True,
                   use_graph=False)
    ens.step(1)                          # one step, then the batched sort
    for spec, sim in ens.sims():
        off_b = sim.tile_off.cpu().numpy().copy()
        pid_b = sim.arrays()["pid"].cpu().numpy().copy()
        sim.sort()                       # single-job path on the same state
        off_s = sim.tile_off.cpu().numpy()
        pid_s = sim.arrays()["pid"].cpu().numpy()
        assert np.array_equal(off_b, off_s)
        for t in range(sim.ntiles):
            a, b = off_s[t], off_s[t + 1]
            assert np.array_equal(np.sort(pid_b[a:b]), np.sort(pid_s[a:b])), t


def test_uneven_ensemble_runs(cuda):
    """A slice of the uneven ensemble distribution (sizes 16-32 per axis,
    ppc 1-16, orders 1-3): runs under CUDA graphs with no error flag and
    finite energies, and keeps every particle."""
    specs = ensemble_jobs(count=12, seed=5, steps=10, cells=(16, 32))
    ens = Ensemble(specs, precision="fp32")
    d0 = ens.diagnostics()
    ens.step(10)
    d1 = ens.diagnostics()
    assert all(f == 0 for f in ens.error_flags())
    for a, b in zip(d0, d1):
        assert np.isfinite(b["total"]) and b["kinetic"] > 0, (a, b)
    assert ens.particles_total == sum(s.particles for s in specs)
