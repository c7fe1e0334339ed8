"""Decks run on the GPU (picsar_b200.deck.run_deck).

* The reference's Langmuir-wave acceptance case (a cold electron slab
  drifting at 0.01 c through protons, 100^3 grid points, 10 particles per
  cell, 30 steps, every temporal diagnostic), with a deck written here from
  the same parameters and the reference acceptance test's own checks
  (Acceptance_testing/Fortran_tests/test_Langmuir_wave/test_langmuir_wave.py):
  total energy within 1 % over the run, the electron kinetic energy within
  10 % of A + A cos(2 pi t / (T_p / 2)).
* A small one-species deck on both engines against the oracle stepping the
  same loaded particles: every field dump and every temporal value to
  1e-12 relative (FP64).
* A 2D (x-z) deck on the plain engine: dumps with one y plane.
"""
import math
import os
import struct

import numpy as np
import pytest

from oracle import oracle as O
from picsar_b200 import deck as D
from tests._cases import rel_l2

pytestmark = pytest.mark.gpu


def _temporal(path):
    """(dt, records) of a binary temporal file: int32 values per record and
    float64 time between records, then the records."""
    raw = open(path, "rb").read()
    nc, dt = struct.unpack_from("<id", raw, 0)
    v = np.frombuffer(raw, dtype="<f8", offset=12)
    return dt, v.reshape(-1, nc)


LANGMUIR = """ Langmuir wave: cold electron slab drifting through protons
section::main
 nx = 100
 ny = 100
 nz = 100
 xmin = -20e-6
 ymin = -20e-6
 zmin = -20e-6
 xmax = 20e-6
 ymax = 20e-6
 zmax = 20e-6
 nsteps = 30
 nguardsx = 3
 nguardsy = 3
 nguardsz = 3
 njguardsx = 3
 njguardsy = 3
 njguardsz = 3
end::main
section::solver
 nox = 1
 noy = 1
 noz = 1
end::solver
section::plasma
 nlab = 1.1e25
 gamma0 = 1.
 pdistr = 1
end::plasma
section::sorting
 activation = 1
 dx = 0.5
 dy = 0.5
 dz = 0.5
 shiftx = -0.5
 shifty = -0.5
 shiftz = -0.5
end::sorting
section::species
 name = electron
 mass = 1
 charge = -1
 nppcell = 10
 x_min = -20e-6
 y_min = -20e-6
 z_min = -10e-6
 x_max = 20e-6
 y_max = 20e-6
 z_max = 10e-6
 vdrift_z = 0.01
 sorting_period = 20
 sorting_start = 20
end::species
section::species
 name = proton
 mass = 1836
 charge = 1
 nppcell = 10
 x_min = -20e-6
 y_min = -20e-6
 z_min = -10e-6
 x_max = 20e-6
 y_max = 20e-6
 z_max = 10e-6
 sorting_period = 20
 sorting_start = 20
end::species
section::output
 output_frequency = 10
 output_step_min = 0
 output_step_max = 1000
 ex = 1
 ez = 1
 rho = 1
 dive = 1
end::output
section::temporal
 frequency = 1
 format = 0
 kinE = 1
 exE = 1
 eyE = 1
 ezE = 1
 bxE = 1
 byE = 1
 bzE = 1
 divE-rho = 1
 rho = 1
 divE = 1
end::temporal
"""


def test_langmuir_acceptance(cuda, tmp_path):
    out = str(tmp_path / "RESULTS")
    m, info = D.run_deck(D.read_input_text(LANGMUIR), out_dir=out)
    assert info["nsteps"] == 30
    assert sorted(os.path.basename(p) for p in info["dumps"]) == sorted(
        f"{f}{i}.pxr" for f in ("ex", "ez", "rho", "dive") for i in (0, 10, 20))
    dt, kin = _temporal(os.path.join(out, "kinE"))
    assert kin.shape == (30, 2)
    t = np.linspace(0, len(kin) * dt, len(kin))
    kinE = kin.T[:, 1:]
    fields = 0.0
    for name in ("exE", "eyE", "ezE", "bxE", "byE", "bzE"):
        e = _temporal(os.path.join(out, name))[1][:, 0]
        fields = fields + (e[1:] + e[:-1]) * 0.5
    total = kinE.sum(axis=0) + fields
    assert (total.max() - total.min()) / total.max() < 1e-2
    n, v = 1.1e25, 0.1
    gamma = 1.0 / math.sqrt(1.0 - v ** 2)
    wp = 1.60217662e-19 * math.sqrt(n / (9.10938356e-31 * 8.85418782e-12))
    tp = 2.0 * math.pi * math.sqrt(gamma) / wp
    a = 0.5 * kinE[0].max()
    theory = a + a * np.cos(2 * np.pi * t[1:] / (tp * 0.5))
    assert np.abs(kinE[0] - theory).max() < 0.1 * kinE[0].max()
    # charge conservation: the divE-rho record against the rho record
    dr = _temporal(os.path.join(out, "divE-rho"))[1][:, 0]
    rho = _temporal(os.path.join(out, "rho"))[1][:, 0]
    assert (dr / rho).max() < 1e-6
    hdr, ex = D.read_pxr(os.path.join(out, "ex20.pxr"))
    assert (hdr["nx"], hdr["ny"], hdr["nz"]) == (99, 99, 99) and hdr["xmin"] == -20e-6
    assert np.isfinite(ex).all() and np.abs(ex).max() > 0


# section::particle_dump precedes section::temporal: the reference reader
# (control_file.F90:1262-1311) reads the temporal section to the end of the
# file, so a section after it is never read.
SMALL = """section::main
 nx = 17
 ny = 13
 nz = 21
 xmin = -4e-6
 ymin = 0.0
 zmin = -5e-6
 xmax = 4e-6
 ymax = 6e-6
 zmax = 5e-6
 nsteps = 3
 nguardsx = 3
 nguardsy = 3
 nguardsz = 3
end::main
section::solver
 nox = {order}
 noy = {order}
 noz = {order}
end::solver
section::plasma
 nlab = 1e25
end::plasma
section::species
 name = electron
 nppcell = 4
 x_min = -4e-6
 y_min = 0.0
 z_min = -5e-6
 x_max = 4e-6
 y_max = 6e-6
 z_max = 5e-6
 vth_x = 0.05
 vth_y = 0.05
 vth_z = 0.05
end::species
section::output
 output_frequency = 1
 output_step_max = 100
 ex = 1
 ey = 1
 bz = 1
 jx = 1
 jz = 1
 rho = 1
 dive = 1
 divb = 1
end::output
section::particle_dump
 species_name = electron
 dump_ux_min = -1e9
 dump_uy_min = -1e9
 dump_uz_min = -1e9
 diag_period = 1
end::particle_dump
section::temporal
 frequency = 1
 kinE = 1
 exE = 1
 bzE = 1
 divE-rho = 1
 rho = 1
end::temporal
"""


@pytest.mark.parametrize("engine,order", [("plain", 1), ("plain", 3), ("tiled", 2)])
def test_small_deck_against_oracle(cuda, tmp_path, engine, order):
    deck = D.read_input_text(SMALL.format(order=order))
    der = deck.derived()
    out = str(tmp_path / "RESULTS")
    D.run_deck(deck, out_dir=out, engine=engine, precision="fp64", seed=11)
    # the oracle from the same loaded particles, in the reference's step order
    p, = D.load_particles(deck, seed=11)
    sp = deck.species[0]
    n, g = der["n"], 3
    o = O.OracleSim(n, g, d=(der["dx"], der["dy"], der["dz"]),
                    xmin=(deck.xmin, deck.ymin, deck.zmin), dt=der["dt"], q=sp.charge,
                    m=sp.mass, order=order, clight=D.CLIGHT, mu0=D.MU0, eps0=D.EPS0)
    o.add_particles(p["x"], p["y"], p["z"], p["ux"], p["uy"], p["uz"], p["w"])
    dv = der["dx"] * der["dy"] * der["dz"]
    inner = (slice(g, g + n[0]), slice(g, g + n[1]), slice(g, g + n[2]))
    one = (slice(g + 1, g + n[0] + 1), slice(g + 1, g + n[1] + 1), slice(g + 1, g + n[2] + 1))
    records = {k: _temporal(os.path.join(out, k))[1] for k in ("kinE", "exE", "bzE", "rho")}
    for it in range(3):
        o.step(1, diag=True)
        f = {c: o.get_field(c) for c in ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jz", "rho")}
        for c in ("ex", "ey", "bz", "jx", "jz", "rho"):
            hdr, a = D.read_pxr(os.path.join(out, f"{c}{it}.pxr"))
            assert a.shape == n
            assert rel_l2(a, f[c][inner]) <= 1e-12, (c, it)
        dive = ((f["ex"][g:g + n[0], g:g + n[1], g:g + n[2]] -
                 f["ex"][g - 1:g + n[0] - 1, g:g + n[1], g:g + n[2]]) / der["dx"] +
                (f["ey"][g:g + n[0], g:g + n[1], g:g + n[2]] -
                 f["ey"][g:g + n[0], g - 1:g + n[1] - 1, g:g + n[2]]) / der["dy"] +
                (f["ez"][g:g + n[0], g:g + n[1], g:g + n[2]] -
                 f["ez"][g:g + n[0], g:g + n[1], g - 1:g + n[2] - 1]) / der["dz"])
        assert rel_l2(D.read_pxr(os.path.join(out, f"dive{it}.pxr"))[1], dive) <= 1e-12
        # temporal records
        q = o.particles()
        ke = float(((1.0 / q["gaminv"] - 1.0) * q["w"]).sum()) * D.EMASS * D.CLIGHT ** 2
        assert abs(records["kinE"][it, 0] - ke) <= 1e-12 * ke
        exe = float((f["ex"][one] ** 2 * 0.5).sum()) * dv * D.EPS0
        assert abs(records["exE"][it, 0] - exe) <= 1e-12 * exe
        bze = float((f["bz"][one] ** 2 * 0.5).sum()) * dv * D.IMU0
        assert abs(records["bzE"][it, 0] - bze) <= 1e-12 * bze
        rn = math.sqrt(float((f["rho"][one] ** 2).sum()))
        assert abs(records["rho"][it, 0] - rn) <= 1e-12 * rn
        # particle dump: every particle (the ranges hold them all), add order
        pd = D.read_particle_dump(os.path.join(out, f"electron_it_{it}"))
        assert len(pd["x"]) == len(q["x"])
        for c in ("x", "y", "z", "ux", "uy", "uz", "w"):
            assert rel_l2(pd[c], q[c]) <= 1e-12, (c, it)


PLANE_2D = """section::cpusplit
 c_dim = 2
end::cpusplit
section::main
 nx = 33
 ny = 1
 nz = 25
 xmin = -4e-6
 zmin = -3e-6
 xmax = 4e-6
 zmax = 3e-6
 nsteps = 4
 nguardsx = 3
 nguardsz = 3
end::main
section::solver
 nox = 2
 noz = 2
end::solver
section::species
 name = electron
 nppcell = 3
 x_min = -4e-6
 z_min = -3e-6
 x_max = 4e-6
 z_max = 3e-6
 vdrift_x = 0.02
 vth_z = 0.01
end::species
section::output
 output_frequency = 3
 output_step_max = 10
 ex = 1
 jx = 1
 bz = 1
end::output
section::temporal
 frequency = 1
 kinE = 1
 exE = 1
end::temporal
"""


def test_2d_deck(cuda, tmp_path):
    out = str(tmp_path / "RESULTS")
    m, info = D.run_deck(D.read_input_text(PLANE_2D), out_dir=out, seed=2)
    assert sorted(os.path.basename(p) for p in info["dumps"]) == sorted(
        f"{c}{i}.pxr" for c in ("ex", "jx", "bz") for i in (0, 3))
    hdr, jx = D.read_pxr(os.path.join(out, "jx3.pxr"))
    assert (hdr["nx"], hdr["ny"], hdr["nz"]) == (32, 1, 24)
    assert hdr["ymin"] == -D.HUGE and hdr["ymax"] == D.HUGE
    # the last iteration's dumps hold nodes 0..n-1 of the final x-z grids
    g = m.nxguards
    for c, a in (("jx", jx), ("ex", D.read_pxr(os.path.join(out, "ex3.pxr"))[1])):
        assert np.array_equal(a[:, 0, :], getattr(m, c)[g:g + 32, g:g + 24].cpu().numpy()), c
    assert np.abs(jx).max() > 0
    _, kin = _temporal(os.path.join(out, "kinE"))
    assert kin.shape == (4, 1) and (kin > 0).all()


HOMOGENEOUS = """ Homogeneous thermal plasma (electrons at 0.1 c, protons at 0.001 c)
section::main
 nx = 100
 ny = 100
 nz = 100
 xmin = -20e-6
 ymin = -20e-6
 zmin = -20e-6
 xmax = 20e-6
 ymax = 20e-6
 zmax = 20e-6
 t_max = 2
 nguardsx = 3
 nguardsy = 3
 nguardsz = 3
 njguardsx = 3
 njguardsy = 3
 njguardsz = 3
end::main
section::solver
 nox = 1
 noy = 1
 noz = 1
end::solver
section::sorting
 activation = 1
 shiftx = -0.5
 shifty = -0.5
 shiftz = -0.5
end::sorting
section::plasma
 nlab = 1e25
 gamma0 = 1.
 pdistr = 1
end::plasma
section::species
 name = electron
 mass = 1.
 charge = -1
 nppcell = 5
 x_min = -20e-6
 y_min = -20e-6
 z_min = -20e-6
 x_max = 20e-6
 y_max = 20e-6
 z_max = 20e-6
 vth_x = 0.1
 vth_y = 0.1
 vth_z = 0.1
 sorting_period = 10
end::species
section::species
 name = proton
 mass = 1836.
 charge = 1
 nppcell = 5
 x_min = -20e-6
 y_min = -20e-6
 z_min = -20e-6
 x_max = 20e-6
 y_max = 20e-6
 z_max = 20e-6
 vth_x = 0.001
 vth_y = 0.001
 vth_z = 0.001
 sorting_period = 10
end::species
section::temporal
 frequency = 1
 kinE = 1
 exE = 1
 eyE = 1
 ezE = 1
 bxE = 1
 byE = 1
 bzE = 1
end::temporal
"""


def test_homogeneous_plasma_acceptance(cuda, tmp_path):
    """The reference's homogeneous-plasma acceptance check
    (Acceptance_testing/Fortran_tests/test_homogeneous_plasma): total
    energy within 1 % over the run; the step count comes from t_max."""
    deck = D.read_input_text(HOMOGENEOUS)
    der = deck.derived()
    assert der["nsteps"] == int(np.rint(2.0 / (der["w0_l"] * der["dt"])))
    out = str(tmp_path / "RESULTS")
    D.run_deck(deck, out_dir=out, seed=5)
    _, kin = _temporal(os.path.join(out, "kinE"))
    assert kin.shape == (der["nsteps"], 2)
    fields = 0.0
    for name in ("exE", "eyE", "ezE", "bxE", "byE", "bzE"):
        e = _temporal(os.path.join(out, name))[1][:, 0]
        fields = fields + (e[1:] + e[:-1]) * 0.5
    total = kin.T[:, 1:].sum(axis=0) + fields
    assert (total.max() - total.min()) / total.max() < 1e-2
