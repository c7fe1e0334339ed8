"""The deck reader, the particle loader and the output formats on the host.

Decks written here exercise the reference reader's rules
(src/initialization/control_file.F90:452-1311); when the reference tree is
present, every example and acceptance deck it ships is parsed and a few
values are checked, and the field dumps and temporal files written here are
read back with the reference's own post-processing readers
(utils/postprocessing/Field.py, PyLoadArrayPicsar.py).
"""
import glob
import importlib.util
import math
import os
import sys
import types

import numpy as np
import pytest

from picsar_b200 import deck as D



def _reference_root():
    """The reference tree: PICSAR_REFERENCE_ROOT, else the parent of the
    source tree that the oracle's build recipe names (oracle/Makefile,
    REF_SRC); the tests that need it are skipped when it is absent."""
    env = os.environ.get("PICSAR_REFERENCE_ROOT")
    if env:
        return env
    mk = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                      "Makefile")
    with open(mk) as f:
        for ln in f:
            if ln.startswith("REF_SRC") and "=" in ln:
                return os.path.dirname(ln.split("=", 1)[1].strip().rstrip("/"))
    return ""


REF = _reference_root()
have_ref = os.path.isdir(os.path.join(REF, "examples", "example_decks_fortran"))

BASE = """section::main
 nx = 17
 ny = 9
 nz = 33
 xmin = -1e-6
 ymin = 0.0
 zmin = -2.0d-6
 xmax = 1e-6
 ymax = 4e-7
 zmax = 2.0D-6
 nsteps = 12
end::main
section::solver
 nox = 2
 noy = 2
 noz = 2
end::solver
section::species
 name = electron
 mass = 1.
 charge = -1
 nppcell = 3
 x_min = -1e-6
 y_min = 0.0
 z_min = -1e-6
 x_max = 1e-6
 y_max = 4e-7
 z_max = 1e-6
 vdrift_z = 0.01
end::species
"""


def test_values_and_units():
    d = D.read_input_text(BASE)
    assert (d.nx_global_grid, d.ny_global_grid, d.nz_global_grid) == (17, 9, 33)
    assert d.zmin == -2e-6 and d.zmax == 2e-6             # d exponents
    assert d.nox == d.noy == d.noz == 2 and d.nsteps == 12
    sp, = d.species
    assert sp.name == "electron" and sp.nppcell == 3
    assert sp.mass == D.EMASS and sp.charge == -D.ECHARGE
    assert sp.vdrift_z == pytest.approx(0.01 * D.CLIGHT, rel=1e-15)
    der = d.derived()
    assert der["n"] == (16, 8, 32)
    assert der["dx"] == (1e-6 - -1e-6) / 16
    dt = d.dtcoef / (D.CLIGHT * math.sqrt(1 / der["dx"] ** 2 + 1 / der["dy"] ** 2 +
                                          1 / der["dz"] ** 2))
    assert der["dt"] == dt and der["nsteps"] == 12


def test_reader_rules():
    text = BASE.replace(" nx = 17\n", " nx = 17 # a comment\n nx =         1024\n nx = 17\n")
    d = D.read_input_text(text)
    # the '#' line is skipped; the (i10) field of the second line reads
    # '         1' (10 characters); the third sets 17 again
    assert d.nx_global_grid == 17
    d = D.read_input_text(BASE.replace(" nx = 17\n", " nx =         1024\n"))
    assert d.nx_global_grid == 1
    # a second main section is not read (its end flag is kept)
    d = D.read_input_text(BASE + "section::main\n nx = 65\nend::main\n")
    assert d.nx_global_grid == 17
    # species sections are read every time
    d = D.read_input_text(BASE + BASE[BASE.index("section::species"):])
    assert len(d.species) == 2
    # a commented-out header still opens its section
    d = D.read_input_text(BASE + "# section::sorting\n activation = 1\nend::sorting\n")
    assert d.sorting_activated == 1
    # the temporal section reads to the end of the file: output_frequency
    # (which holds 'frequency') set after it sets the temporal frequency too
    d = D.read_input_text(BASE + "section::temporal\n frequency = 2\n kinE = 1\nend::temporal\n"
                          "section::output\n output_frequency = 7\nend::output\n")
    assert d.temdiag_frequency == 7 and d.output_frequency == -1
    assert d.temdiag_act_list[0] == 1
    # substring matching in the reference's order: 'dive' does not hold 'ex'
    d = D.read_input_text(BASE + "section::output\n dive = 1\n ex = 1\nend::output\n")
    assert d.c_output["dive"] == 1 and d.c_output["ex"] == 1 and d.c_output["rho"] == 0
    # list-directed logicals
    d = D.read_input_text(BASE + "section::solver\n l_spectral = .TRUE.\nend::solver\n")
    assert d.l_spectral is False                      # (second solver section not read)
    d = D.read_input_text(BASE.replace(" nox = 2\n", " nox = 2\n l_staggered = F\n"))
    assert d.l_staggered is False
    with pytest.raises(D.DeckError):
        D.read_input_text(BASE.replace(" nx = 17\n", " nx = 1x\n"))


def test_particle_dump_section():
    text = BASE + ("section::particle_dump\n species_name = electron\n diag_period = 5\n"
                   " dump_ux_min = -1e9\nend::particle_dump\n")
    d = D.read_input_text(text)
    dp, = d.particle_dumps
    assert dp.ispecies == 0 and dp.diag_period == 5 and dp.dump_ux_min == -1e9
    # bounds not given default to the domain read so far and to 1e7..1e9
    assert dp.dump_x_min == d.xmin and dp.dump_z_max == d.zmax
    assert dp.dump_uy_min == 1e7 and dp.dump_uz_max == 1e9


def test_nsteps_from_t_max():
    d = D.read_input_text(BASE.replace(" nsteps = 12\n", " t_max = 0.5\n"))
    der = d.derived()
    w0 = D.ECHARGE * math.sqrt(d.nlab / (D.EMASS * D.EPS0))
    assert der["nsteps"] == int(np.rint(0.5 / (w0 * der["dt"])))


def _loader_loops(d):
    """The pdistr = 1 positions of tiling.F90:887-894, loop by loop."""
    der = d.derived()
    dx, dy, dz = der["dx"], der["dy"], der["dz"]
    sp = d.species[0]
    j0, j1 = D._box(sp.x_min, sp.x_max, d.xmin, d.xmax, dx)
    k0, k1 = D._box(sp.y_min, sp.y_max, d.ymin, d.ymax, dy)
    l0, l1 = D._box(sp.z_min, sp.z_max, d.zmin, d.zmax, dz)
    out = []
    for l in range(l0, l1):
        for k in range(k0, k1):
            for j in range(j0, j1):
                for ip in range(1, sp.nppcell + 1):
                    out.append((d.xmin + j * dx + dx / sp.nppcell * (ip - 0.5),
                                d.ymin + k * dy + dy / sp.nppcell * (ip - 0.5),
                                d.zmin + l * dz + dz / sp.nppcell * (ip - 0.5)))
    return np.array(out)


def test_loader_pdistr1():
    d = D.read_input_text(BASE)
    p, = D.load_particles(d, seed=3)
    ref = _loader_loops(d)
    assert len(p["x"]) == len(ref) == 16 * 8 * 16 * 3
    assert np.array_equal(p["x"], ref[:, 0]) and np.array_equal(p["y"], ref[:, 1])
    assert np.array_equal(p["z"], ref[:, 2])
    der = d.derived()
    assert np.all(p["w"] == der["nc"] * der["dx"] * der["dy"] * der["dz"] / 3)
    # cold drift: u = v / gamma^-1 exactly as the loader computes it
    v = 0.01 * D.CLIGHT
    gi = math.sqrt(1.0 - v * v * (1.0 / D.CLIGHT ** 2))
    assert np.all(p["uz"] == v / gi) and np.all(p["ux"] == 0.0)
    assert np.all(p["gaminv"] == gi)


def test_loader_thermal_and_uniform():
    text = BASE.replace(" vdrift_z = 0.01\n", " vth_x = 0.05\n vth_y = 0.05\n vth_z = 0.05\n")
    d = D.read_input_text(text)
    p, = D.load_particles(d, seed=1)
    # the loader's draw: v_x = vth sqrt(-2 ln r1) cos(th) cos(phi), so
    # <v_x^2> = vth^2 / 2 and <v_z^2> = vth^2
    vx, vz = (p[c] * p["gaminv"] / D.CLIGHT for c in ("ux", "uz"))
    assert abs(vx.std() / (0.05 / math.sqrt(2)) - 1) < 0.05
    assert abs(vz.std() / 0.05 - 1) < 0.05
    d = D.read_input_text(text + "section::plasma\n pdistr = 2\nend::plasma\n")
    p, = D.load_particles(d, seed=1)
    assert p["x"].min() >= d.xmin and p["x"].max() < d.xmax
    assert p["z"].min() >= d.zmin and p["z"].max() < d.zmax


def test_pxr_round_trip(tmp_path):
    a = np.random.default_rng(0).standard_normal((5, 3, 4))
    f = tmp_path / "ex7.pxr"
    D.write_pxr(f, a, (-1.0, 0.0, 2.0), (1.0, 3.0, 6.0), (5, 3, 4))
    hdr, b = D.read_pxr(f)
    assert hdr["nx"] == 5 and hdr["zmax"] == 6.0
    assert np.array_equal(a, b)
    assert os.path.getsize(f) == 60 + 8 * a.size
    assert D._step_label(7) == "7" and D._step_label(123456) == "*****"


def _import_reference(name, stub_plotting=False):
    path = os.path.join(REF, "utils", "postprocessing", name + ".py")
    if stub_plotting:
        # the reader imports matplotlib for its plot methods only
        for mod in ("matplotlib", "matplotlib.pyplot", "matplotlib.gridspec",
                    "mpl_toolkits", "mpl_toolkits.mplot3d"):
            sys.modules.setdefault(mod, types.ModuleType(mod))
        sys.modules["mpl_toolkits.mplot3d"].Axes3D = object
    spec = importlib.util.spec_from_file_location("pxr_ref_" + name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.skipif(not have_ref, reason="reference tree not present")
def test_reference_readers_read_our_files(tmp_path, capsys):
    a = np.random.default_rng(1).standard_normal((6, 4, 5))
    f = str(tmp_path / "rho3.pxr")
    D.write_pxr(f, a, (-2e-6, -1e-6, 0.0), (2e-6, 1e-6, 5e-6), (6, 4, 5))
    Field = _import_reference("Field", stub_plotting=True).Field
    fld = Field(f)
    assert (fld.nx, fld.ny, fld.nz) == (6, 4, 5)
    assert np.array_equal(fld.f, a.transpose(2, 1, 0))        # f[iz, iy, ix]
    # temporal files: the binary header and records
    d = D.read_input_text(BASE + "section::temporal\n frequency = 2\n kinE = 1\n exE = 1\n"
                          "end::temporal\n")
    der = d.derived()
    t = D._Temporal(d, der, str(tmp_path), nspecies=2)
    rows = [([1.0, 2.0], [3.0]), ([4.0, 5.0], [6.0]), ([7.0, 8.0], [9.0])]
    for ke, ex in rows:
        t.write({0: ke, 1: ex})
    read = _import_reference("PyLoadArrayPicsar").read_picsar_temporal_diags
    tt, kin = read(str(tmp_path / "kinE"))
    assert kin.shape == (2, 3) and np.array_equal(kin[:, 2], [7.0, 8.0])
    assert tt[1] == pytest.approx(2 * der["dt"] * 3 / 2)      # linspace(0, nl*dt, nl)
    _, exe = read(str(tmp_path / "exE"))
    assert np.array_equal(exe, [3.0, 6.0, 9.0])
    capsys.readouterr()


@pytest.mark.skipif(not have_ref, reason="reference tree not present")
def test_reference_decks_parse():
    decks = sorted(glob.glob(os.path.join(REF, "examples", "example_decks_fortran", "*.pixr")) +
                   glob.glob(os.path.join(REF, "Acceptance_testing", "Fortran_tests", "*",
                                          "input_file.pixr")))
    assert len(decks) >= 10
    parsed = {os.path.relpath(p, REF): D.read_input_file(p) for p in decks}
    h = parsed[os.path.join("examples", "example_decks_fortran", "homogeneous_plasma.pixr")]
    assert h.nx_global_grid == 100 and h.xmin == -20e-6 and h.tmax == 2
    assert [s.name for s in h.species] == ["electron", "proton"]
    assert h.species[1].mass == 1836.0 * D.EMASS
    assert h.species[0].vth_x == pytest.approx(0.1 * D.CLIGHT, rel=1e-15)
    assert h.output_frequency == 10 and h.c_output["rho"] == 1 and h.c_output["jx"] == 0
    assert h.temdiag_frequency == 1 and all(h.temdiag_act_list)
    assert h.sorting_activated == 1 and h.sorting_shiftx == -0.5
    assert h.derived()["dx"] == 40e-6 / 99
    lw = parsed[os.path.join("examples", "example_decks_fortran", "langmuir_wave.pixr")]
    assert lw.nsteps == 30 and lw.derived()["nsteps"] == 30
    assert lw.species[0].vdrift_z == pytest.approx(0.01 * D.CLIGHT, rel=1e-15)
    p2d = parsed[os.path.join("examples", "example_decks_fortran", "plane_wave_test_2d.pixr")]
    assert p2d.c_dim == 2 and p2d.l_spectral is True and p2d.derived is not None
    assert any(d.antenna for d in parsed.values())          # the laser decks
