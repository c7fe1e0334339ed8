"""Host-side logic without a GPU: ensemble job distribution, admission cost
model, request streams, the FIFO latency model and the autotuner's choice
of representative jobs."""
import math

import numpy as np

from picsar_b200.autotune import _key, proxy_grid, representative
from picsar_b200.ensemble import JobSpec, ensemble_jobs, job_bytes
from picsar_b200.serve import Request, fifo_latencies, percentile, poisson_requests


def test_ensemble_distribution():
    specs = ensemble_jobs(count=256, seed=2024, steps=100)
    assert len(specs) == 256
    assert specs == ensemble_jobs(count=256, seed=2024, steps=100)      # one master seed
    for s in specs:
        assert all(16 <= v <= 96 for v in s.n)
        assert s.ppc in (1, 2, 4, 8, 16) and s.order in (1, 2, 3)
        assert 1e-3 <= s.sigma <= 5e-2 and s.steps == 100
    assert len({s.seed for s in specs}) == 256
    mean_cells = np.mean([s.cells for s in specs])
    assert 1.5e5 < mean_cells < 4.5e5             # E[N^3] ~ 2.7e5 for N ~ U{16..96}
    st = ensemble_jobs(count=64, seed=1, steps_range=(50, 500))
    assert all(50 <= s.steps <= 500 for s in st)


def test_job_bytes_scales():
    a = JobSpec(n=(32, 32, 32), ppc=8, sigma=0.01, order=1)
    b = JobSpec(n=(32, 32, 32), ppc=16, sigma=0.01, order=1)
    # FP32: 7 reals and the packed cell twice (sort buffers) + rank + perm = 72 B/particle
    assert job_bytes(b, "fp32") - job_bytes(a, "fp32") == 32 ** 3 * 8 * 72
    assert job_bytes(a, "fp64") > job_bytes(a, "fp32")


def test_poisson_requests_and_percentiles():
    specs = [JobSpec(n=(16, 16, 16), ppc=1, sigma=0.01, order=1)] * 2000
    reqs = poisson_requests(specs, rate=50.0, seed=3)
    t = np.array([r.arrival for r in reqs])
    assert t[0] == 0 and np.all(np.diff(t) >= 0)
    assert abs(np.mean(np.diff(t)) - 1 / 50.0) < 0.1 / 50.0
    assert percentile([1, 2, 3, 4], 50) == 2.5


def test_fifo_latencies():
    spec = JobSpec(n=(16, 16, 16), ppc=1, sigma=0.01, order=1)
    reqs = [Request(0, spec, 0.0), Request(1, spec, 0.5), Request(2, spec, 10.0)]
    lat = fifo_latencies(reqs, {0: 2.0, 1: 2.0, 2: 1.0})
    assert lat == {0: 2.0, 1: 3.5, 2: 1.0}


def test_autotune_representative_and_proxy():
    specs = [JobSpec(n=(16, 16, 16), ppc=p, sigma=s, order=o)
             for p, s, o in [(1, 0.001, 1), (16, 0.05, 1), (16, 0.01, 1), (4, 0.02, 3)]]
    rep = representative(specs)
    assert rep[1][0] == 16 and rep[3][0] == 4
    assert rep[1][1] == 0.05
    n = proxy_grid(8, 148)
    tiles = (n[0] // 8) * (n[1] // 8) * (n[2] // 8)
    assert tiles >= 2 * 148 * 2 and math.prod(n) * 8 <= 12_000_000


def test_autotune_cache_keys():
    k = lambda **kw: _key(**{**dict(order=3, precision="fp32", ppc=8, sigma=0.01, pusher=0,
                                    device_name="GPU"), **kw})
    assert k() == k(sigma=0.011)                       # same half-decade of spread
    assert k() != k(sigma=0.05) and k() != k(ppc=16) and k() != k(order=2)
    assert k() != k(u_drift=0.2) and k(u_drift=0.2) == k(u_drift=0.2001)
    assert k().startswith("GPU|o3|fp32|ppc8|")


def test_job_spec_rejects_jobs_without_steps():
    import pytest
    for bad in (0, -3):
        with pytest.raises(ValueError, match="at least one step"):
            JobSpec(n=(16, 16, 16), ppc=1, sigma=0.01, order=1, steps=bad)
    with pytest.raises(ValueError):
        JobSpec(n=(16, 0, 16), ppc=1, sigma=0.01, order=1)
