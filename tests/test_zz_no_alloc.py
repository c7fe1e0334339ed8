"""Diagnostics entry point that allocates nothing (collected last on purpose).

Callers that cannot allocate device memory -- a runtime that gives the
library only a job descriptor, or code confined to a memory pool it must not
grow -- use pxrb_tiled_diagnostics_noalloc, whose scratch (rho grid and
partial sums) is a static device array inside libpicsar_b200.so.  This test
calls it through the C ABI twice in a row and checks each result against the
allocating entry point pxrb_tiled_diagnostics on the same state, and checks
that a job above the array's limit is refused before any GPU work.
"""
import pytest
import torch

from picsar_b200._lib import PicsarB200Error
from picsar_b200.init import thermal_plasma
from picsar_b200.tiled import TiledConfig, TiledSim
from tests._cases import random_fields

pytestmark = pytest.mark.gpu

KEYS = ("kinetic", "ex", "ey", "ez", "bx", "by", "bz", "gauss_norm", "rho_norm")
TOL = 1e-12


def _close(a, b):
    return abs(a - b) <= TOL * max(abs(a), abs(b), 1e-300)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_noalloc_diagnostics_match_allocating_entry_point(cuda, precision):
    from picsar_b200 import picsar as P
    n, g = (24, 16, 20), 3
    st = thermal_plasma(n, 4, 0.05, seed=31, shuffle=True)
    t = TiledSim(n, order=2, precision=precision, config=TiledConfig(tile=(8, 8, 8)))
    for name, a in zip(("ex", "ey", "ez", "bx", "by", "bz"), random_fields(n, g, seed=32)):
        t.import_field(name, P.to_fortran(a), g)
    t.load_state(st.to(device="cuda"))
    t.step(2)
    for _ in range(2):                      # two calls in a row
        ref = t.diagnostics(gauss=True)
        got = t.diagnostics_noalloc(gauss=True)
        torch.cuda.synchronize()
        for k in KEYS:
            assert _close(got[k], ref[k]), (k, got[k], ref[k])
        t.step(1)
    # energies only
    ref = t.diagnostics(gauss=False)
    got = t.diagnostics_noalloc(gauss=False)
    for k in ("kinetic", "ex", "ey", "ez", "bx", "by", "bz"):
        assert _close(got[k], ref[k]), (k, got[k], ref[k])


def test_noalloc_rejects_jobs_above_its_limit(cuda):
    t = TiledSim((128, 128, 72), order=1, precision="fp32", config=TiledConfig(tile=(8, 8, 8)))
    with pytest.raises(PicsarB200Error, match="status 6"):
        t.diagnostics_noalloc(gauss=True)


def test_noalloc_energies_of_a_job_above_the_rho_limit(cuda):
    # without the Gauss residual no rho grid is needed: any job size is served
    from picsar_b200 import picsar as P
    n, g = (128, 128, 72), 3
    st = thermal_plasma(n, 1, 0.02, seed=33)
    t = TiledSim(n, order=1, precision="fp32", config=TiledConfig(tile=(8, 8, 8)))
    for name, a in zip(("ex", "ey", "ez", "bx", "by", "bz"), random_fields(n, g, seed=34)):
        t.import_field(name, P.to_fortran(a), g)
    t.load_state(st.to(device="cuda"))
    t.step(1)
    for _ in range(2):
        ref = t.diagnostics(gauss=False)
        got = t.diagnostics_noalloc(gauss=False)
        for k in ("kinetic", "ex", "ey", "ez", "bx", "by", "bz"):
            assert _close(got[k], ref[k]), (k, got[k], ref[k])
