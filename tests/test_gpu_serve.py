"""Serving loop on the GPU: each job's result is the same alone and in the
mix (continuous batching with jobs joining and leaving while it runs), and
admission keeps the resident state within the HBM budget.

Tolerance: FP64 1e-12 relative L2 (fields and momenta); FP32 mixed 1e-5
(the mix changes only the order of the FP64 current-flush atomics and the
phase of the periodic sort).
"""
import numpy as np
import pytest
import torch

from picsar_b200.ensemble import JobSpec, job_bytes
from picsar_b200.serve import Request, Server
from picsar_b200.tiled import TiledConfig
from tests._cases import rel_l2

pytestmark = pytest.mark.gpu

TARGET = JobSpec(n=(16, 24, 16), ppc=4, sigma=0.03, order=2, pusher=0, steps=8, seed=77)
OTHERS = [
    JobSpec(n=(24, 16, 16), ppc=2, sigma=0.02, order=2, pusher=1, steps=12, seed=1),
    JobSpec(n=(16, 16, 16), ppc=1, sigma=0.05, order=1, pusher=0, steps=4, seed=2),
    JobSpec(n=(16, 16, 20), ppc=2, sigma=0.01, order=3, pusher=0, steps=10, seed=3),
    JobSpec(n=(20, 16, 16), ppc=3, sigma=0.02, order=2, pusher=0, steps=6, seed=4),
]


def _capture(store):
    def cb(req, sim):
        torch.cuda.synchronize()
        out = {n: sim.export_field(n, 3).cpu().numpy() for n in ("ex", "ey", "ez", "bx", "by", "bz")}
        p = sim.particles()
        for c in ("ux", "uy", "uz", "gaminv", "id"):
            out["p_" + c] = p[c].cpu().numpy()
        store[req.rid] = out
    return cb


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_result_same_alone_and_in_mix(cuda, precision, tol):
    cfg = {o: TiledConfig(tile=(8, 8, 8), sort_interval=3) for o in (1, 2, 3)}
    alone, mixed = {}, {}
    Server(precision, configs=cfg, track_ids=True, on_finish=_capture(alone)).run(
        [Request(100, TARGET, 0)], clock="iterations")
    reqs = [Request(0, OTHERS[0], 0), Request(1, OTHERS[1], 0), Request(100, TARGET, 2),
            Request(2, OTHERS[2], 5), Request(3, OTHERS[3], 6)]
    rep = Server(precision, configs=cfg, track_ids=True, on_finish=_capture(mixed)).run(
        reqs, clock="iterations")
    assert rep.peak_resident_jobs >= 4            # the target really ran in a mix
    a, b = alone[100], mixed[100]
    assert np.array_equal(a["p_id"], b["p_id"])
    for k in a:
        if k != "p_id":
            assert rel_l2(b[k], a[k]) <= tol, (k, rel_l2(b[k], a[k]))
    lat = {r.rid: r.latency for r in rep.results}
    assert lat[100] == TARGET.steps               # admitted at arrival, no queueing


def test_admission_respects_hbm_budget(cuda):
    specs = [JobSpec(n=(16, 16, 16), ppc=4, sigma=0.02, order=1, steps=5, seed=i)
             for i in range(6)]
    b = job_bytes(specs[0], "fp32")
    srv = Server("fp32", hbm_budget=2 * b + b // 2)
    rep = srv.run([Request(i, s, 0) for i, s in enumerate(specs)], clock="iterations")
    assert len(rep.results) == 6
    assert rep.peak_resident_jobs == 2
    assert rep.peak_bytes <= 2 * b + b // 2
    lat = sorted(r.latency for r in rep.results)
    assert lat == [5, 5, 10, 10, 15, 15]          # FIFO admission in pairs
    s = rep.summary()
    assert s["max_gauss_drift"] < 1e-5


def test_job_bytes_matches_allocation(cuda):
    from picsar_b200.tiled import TiledSim
    spec = JobSpec(n=(24, 16, 20), ppc=3, sigma=0.02, order=3, steps=1, seed=9)
    t = TiledSim(spec.n, order=3, precision="fp32")
    t.load_state(spec.initial_state())
    pred = job_bytes(spec, "fp32")
    assert t.state_bytes() <= pred <= t.state_bytes() * 1.2 + (1 << 20)


def test_fifo_plain_baseline_serves_every_job(cuda):
    from picsar_b200.serve import serve_fifo_plain
    specs = [JobSpec(n=(16, 16, 16), ppc=1, sigma=0.02, order=1, steps=3, seed=i)
             for i in range(3)]
    rep = serve_fifo_plain([Request(i, s, 0.0) for i, s in enumerate(specs)])
    s = rep.summary()
    assert s["jobs"] == 3
    lat = [r.latency for r in rep.results]
    assert all(v > 0 for v in lat) and lat == sorted(lat)      # one at a time, in order


def test_wall_clock_server_runs_a_stream(cuda):
    from picsar_b200.ensemble import ensemble_jobs
    from picsar_b200.serve import poisson_requests
    specs = ensemble_jobs(count=8, seed=3, steps_range=(3, 12), cells=(16, 24))
    rep = Server("fp32").run(poisson_requests(specs, 200.0, seed=1), clock="wall")
    s = rep.summary()
    assert s["jobs"] == 8 and s["max_gauss_drift"] < 1e-4
    assert all(r.finished >= r.admitted >= r.arrival - 1e-9 for r in rep.results)
    assert rep.particle_steps == sum(sp.particles * sp.steps for sp in specs)
