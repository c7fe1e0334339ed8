"""The small plain configuration run for its full length on the GPU against
the oracle: 32^3 cells, 8 particles per cell (262,144 electrons), u ~
N(0, 0.01^2), order 1, Boris, Esirkepov, Yee at 0.95 CFL, 100 FP64 steps.

Checked every step: the total energy (kinetic (gamma-1) w m c^2 plus the E and
B field energies, diags.F90:847-1114) of the plain FP64 path and of the tiled
FP64 engine (driven through the module surface) against the oracle's, to
HISTORY_TOL relative; at the end, the fields and particle momenta to the same
bound.  The FP64 trajectories differ only by the order of floating-point
additions in the current deposition, which a 100-step thermal run does not
amplify beyond it.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from picsar_b200 import picsar as P
from tests._cases import plasma, rel_l2

pytestmark = pytest.mark.gpu

HISTORY_TOL = 1e-10
N_, G, STEPS = (32, 32, 32), 3, 100


def _energies_plain(m):
    """Energies of the plain module's state with the oracle's own sums."""
    sp = m.species[0]
    ke = O.kinetic_energy(sp.part_gaminv.cpu().numpy(), sp.pid_w.cpu().numpy())
    fe = [O.field_energy(np.asfortranarray(getattr(m, c).cpu().numpy()), N_, G, (1.0,) * 3)
          for c in ("ex", "ey", "ez", "bx", "by", "bz")]
    return ke + sum(fe)


@pytest.fixture(scope="module")
def history():
    st = plasma(N_, 8, 0.01, seed=2026)
    o = O.OracleSim(N_, G, order=1, pusher=0, tiles=(4, 4, 4))
    o.add_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    mods = {}
    for engine in ("plain", "tiled"):
        m = P.PicsarModule(*N_, nguards=G, nox=1, particle_pusher=0, engine=engine)
        m.add_species("electron", -1.0, 1.0, st["x"], st["y"], st["z"], st["ux"], st["uy"],
                      st["uz"], st["w"])
        mods[engine] = m
    hist = {"oracle": [], "plain": [], "tiled": []}
    for _ in range(STEPS):
        o.step(1)
        d = o.diags()
        hist["oracle"].append(d["kinetic"] + sum(d[c] for c in ("ex", "ey", "ez", "bx", "by",
                                                                "bz")))
        mods["plain"].step(1)
        hist["plain"].append(_energies_plain(mods["plain"]))
        mods["tiled"].step(1)
        hist["tiled"].append(mods["tiled"].diagnostics(gauss=False)["total"])
    torch.cuda.synchronize()
    return o, mods, {k: np.array(v) for k, v in hist.items()}


@pytest.mark.parametrize("engine", ["plain", "tiled"])
def test_energy_history_matches_oracle(cuda, history, engine):
    o, mods, h = history
    rel = np.abs(h[engine] - h["oracle"]) / np.abs(h["oracle"])
    assert rel.max() <= HISTORY_TOL, (engine, rel.max(), int(rel.argmax()))


@pytest.mark.parametrize("engine", ["plain", "tiled"])
def test_final_state_matches_oracle(cuda, history, engine):
    o, mods, h = history
    m = mods[engine]
    for name in ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz"):
        assert rel_l2(getattr(m, name).cpu().numpy(), o.get_field(name)) <= HISTORY_TOL, name
    ref = o.particles()
    sp = m.species[0]
    srt = np.argsort(sp.pid_id.cpu().numpy(), kind="stable")
    for c, attr in (("ux", "part_ux"), ("uy", "part_uy"), ("uz", "part_uz")):
        assert rel_l2(getattr(sp, attr).cpu().numpy()[srt], ref[c]) <= HISTORY_TOL, c
