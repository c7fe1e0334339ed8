"""Parity of the plain FP64 CUDA path against the CPU oracle.

Bar: relative L2 <= 1e-12 on the same seeded inputs (the FP64 bar).  Each test calls the C ABI through the Forthon-named
wrappers in picsar_b200.picsar.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from picsar_b200 import picsar as P
from tests._cases import fresh_particles, plasma, random_fields, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-12
PCOLS = ("x", "y", "z", "ux", "uy", "uz", "gaminv", "ex", "ey", "ez", "bx", "by", "bz")


def _dev(d):
    return {k: torch.tensor(v, dtype=torch.float64, device="cuda") for k, v in d.items()}


def _host(d):
    return {k: v.cpu().numpy() for k, v in d.items()}


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("pusher", [0, 1])
def test_gather_push(cuda, order, pusher):
    n, g = (16, 12, 20), 3
    grids = random_fields(n, g, seed=10 + order)
    st = plasma(n, 4, 0.2, seed=order)
    ref = fresh_particles(st)
    gpu = _dev(fresh_particles(st))
    dt = 0.5
    O.gather_push(order, ref, grids, (0, 0, 0), (1, 1, 1), n, g, -1.0, 1.0, dt, pusher)
    G = [P.to_fortran(a) for a in grids]
    fn = {1: P.field_gathering_plus_particle_pusher_1_1_1,
          2: P.field_gathering_plus_particle_pusher_2_2_2,
          3: P.field_gathering_plus_particle_pusher_3_3_3}[order]
    fn(len(st["x"]), *[gpu[c] for c in PCOLS], 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, dt, *n, g, g, g,
       *G, -1.0, 1.0, 256, True, dt=dt, particle_pusher=pusher, clight=1.0)
    torch.cuda.synchronize()
    out = _host(gpu)
    for c in PCOLS:
        assert rel_l2(out[c], ref[c]) <= TOL, c
    # displacement is compared on its own (positions hide it)
    assert rel_l2(out["x"] - st["x"], ref["x"] - st["x"]) <= 1e-11


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("nodal", [False, True])
def test_geteb3d(cuda, order, lower, nodal):
    n, g = (12, 16, 10), 3
    grids = random_fields(n, g, seed=20 + order)
    st = plasma(n, 3, 0.0, seed=5)
    N = len(st["x"])
    ref = {c: np.zeros(N) for c in ("ex", "ey", "ez", "bx", "by", "bz")}
    O.geteb3d_scalar(0, order, st["x"], st["y"], st["z"], ref["ex"], ref["ey"], ref["ez"],
                     (0, 0, 0), (1, 1, 1), n, g, grids[0], grids[1], grids[2], lower, nodal)
    O.geteb3d_scalar(1, order, st["x"], st["y"], st["z"], ref["bx"], ref["by"], ref["bz"],
                     (0, 0, 0), (1, 1, 1), n, g, grids[3], grids[4], grids[5], lower, nodal)
    d = _dev({c: st[c] for c in ("x", "y", "z")})
    f = _dev({c: np.zeros(N) for c in ("ex", "ey", "ez", "bx", "by", "bz")})
    G = [P.to_fortran(a) for a in grids]
    P.geteb3d_energy_conserving(N, d["x"], d["y"], d["z"], f["ex"], f["ey"], f["ez"], f["bx"],
                                f["by"], f["bz"], 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, *n, g, g, g,
                                order, order, order, *G, False, lower, 256, 0, l_nodal=nodal)
    torch.cuda.synchronize()
    for c, v in _host(f).items():
        assert rel_l2(v, ref[c]) <= TOL, c


def test_pushers(cuda):
    rng = np.random.default_rng(3)
    N = 5000
    base = {c: rng.standard_normal(N) * 0.3 for c in ("ux", "uy", "uz", "ex", "ey", "ez",
                                                      "bx", "by", "bz", "x", "y", "z")}
    base["gaminv"] = 1.0 / np.sqrt(1 + base["ux"] ** 2 + base["uy"] ** 2 + base["uz"] ** 2)
    q, m, dt = -1.0, 1.0, 0.4
    # Boris
    r = {k: v.copy() for k, v in base.items()}
    O.boris_push_u(r["ux"], r["uy"], r["uz"], r["gaminv"], r["ex"], r["ey"], r["ez"], r["bx"],
                   r["by"], r["bz"], q, m, dt)
    d = _dev(base)
    P.pxr_boris_push_u_3d(N, d["ux"], d["uy"], d["uz"], d["gaminv"], d["ex"], d["ey"], d["ez"],
                          d["bx"], d["by"], d["bz"], q, m, dt)
    torch.cuda.synchronize()
    for c in ("ux", "uy", "uz", "gaminv"):
        assert rel_l2(d[c].cpu().numpy(), r[c]) <= TOL
    # Vay, three variants
    for which in (0, 1, 2):
        r = {k: v.copy() for k, v in base.items()}
        O.ebcancelpush3d(r["ux"], r["uy"], r["uz"], r["gaminv"], r["ex"], r["ey"], r["ez"],
                         r["bx"], r["by"], r["bz"], q, m, dt, which)
        d = _dev(base)
        P.pxr_ebcancelpush3d(N, d["ux"], d["uy"], d["uz"], d["gaminv"], d["ex"], d["ey"],
                             d["ez"], d["bx"], d["by"], d["bz"], q, m, dt, which)
        torch.cuda.synchronize()
        for c in ("ux", "uy", "uz", "gaminv"):
            assert rel_l2(d[c].cpu().numpy(), r[c]) <= TOL, (which, c)
    # set_gamma + pushxyz
    r = {k: v.copy() for k, v in base.items()}
    O.set_gamma(r["ux"], r["uy"], r["uz"], r["gaminv"])
    O.pushxyz(r["x"], r["y"], r["z"], r["ux"], r["uy"], r["uz"], r["gaminv"], dt)
    d = _dev(base)
    P.pxr_set_gamma(N, d["ux"], d["uy"], d["uz"], d["gaminv"])
    P.pxr_pushxyz(N, d["x"], d["y"], d["z"], d["ux"], d["uy"], d["uz"], d["gaminv"], dt)
    torch.cuda.synchronize()
    for c in ("gaminv", "x", "y", "z"):
        assert rel_l2(d[c].cpu().numpy(), r[c]) <= TOL


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("algo", [0, 1])
def test_esirkepov(cuda, order, algo):
    n, g = (16, 16, 16), 3
    st = plasma(n, 4, 0.3, seed=40 + order)
    p = fresh_particles(st)
    dt = 0.5
    J = [O.zeros_grid(*n, g) for _ in range(3)]
    O.depose_jxjyjz(order, *J, p["x"], p["y"], p["z"], p["ux"], p["uy"], p["uz"], p["gaminv"],
                    p["w"], -1.0, (0, 0, 0), dt, (1, 1, 1), n, g, algo=algo)
    d = _dev(p)
    JG = [P.grid_zeros(*n, g) for _ in range(3)]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    P.depose_jxjyjz(*JG, len(p["x"]), d["x"], d["y"], d["z"], d["ux"], d["uy"], d["uz"],
                    d["gaminv"], d["w"], -1.0, 0.0, 0.0, 0.0, dt, 1.0, 1.0, 1.0, *n, g, g, g,
                    order, order, order, algo, err_flag=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    for a, b in zip(JG, J):
        assert rel_l2(a.cpu().numpy(), b) <= TOL


@pytest.mark.parametrize("order", [1, 2, 3])
def test_rho(cuda, order):
    n, g = (16, 10, 14), 3
    st = plasma(n, 4, 0.0, seed=60 + order)
    rho = O.zeros_grid(*n, g)
    O.depose_rho(order, rho, st["x"], st["y"], st["z"], st["w"], -1.0, (0, 0, 0), (1, 1, 1), n, g)
    m = P.PicsarModule(*n, nguards=g, nox=order)
    m.add_species("e", -1.0, 1.0, st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"],
                  st["w"])
    m.pxrdepose_rho_on_grid()
    torch.cuda.synchronize()
    assert rel_l2(m.rho.cpu().numpy(), rho) <= TOL


def test_yee_and_bcs(cuda):
    n, g = (20, 16, 12), 3
    f = random_fields(n, g, seed=7)
    J = random_fields(n, g, seed=8)[:3]
    ref = [a.copy(order="F") for a in f]
    O.push_bvec(*ref, n, g, 0.25, 0.3, 0.35)
    O.push_evec(*ref, *J, n, g, 0.6, 0.5, 0.45, 0.4)
    m = P.PicsarModule(*n, nguards=g)
    for name, a in zip(("ex", "ey", "ez", "bx", "by", "bz"), f):
        getattr(m, name).copy_(torch.from_numpy(a))
    for name, a in zip(("jx", "jy", "jz"), J):
        getattr(m, name).copy_(torch.from_numpy(a))
    n3, lo, hi = n, (-g,) * 3, tuple(v + g for v in n)
    P.pxrpush_em3d_bvec((0, 0, 0), n3, (0, 0, 0), n3, (0, 0, 0), n3, m.ex, lo, hi, m.ey, lo, hi,
                        m.ez, lo, hi, m.bx, lo, hi, m.by, lo, hi, m.bz, lo, hi, 0.25, 0.3, 0.35)
    P.pxrpush_em3d_evec((0, 0, 0), n3, (0, 0, 0), n3, (0, 0, 0), n3, m.ex, lo, hi, m.ey, lo, hi,
                        m.ez, lo, hi, m.bx, lo, hi, m.by, lo, hi, m.bz, lo, hi, m.jx, lo, hi,
                        m.jy, lo, hi, m.jz, lo, hi, 0.6, 0.5, 0.45, 0.4)
    torch.cuda.synchronize()
    for name, a in zip(("ex", "ey", "ez", "bx", "by", "bz"), ref):
        assert rel_l2(getattr(m, name).cpu().numpy(), a) <= TOL, name
    # guard exchange and fold
    rng = np.random.default_rng(9)
    a = rng.standard_normal(O.grid_shape(*n, g))
    a = np.asfortranarray(a)
    b = a.copy(order="F")
    O.field_bc(a, n, g)
    t = P.to_fortran(b)
    P.field_bc(t, g, g, g, *n)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), a)
    a = np.asfortranarray(rng.standard_normal(O.grid_shape(*n, g)))
    b = a.copy(order="F")
    O.summation_bcs(a, n, g)
    t = P.to_fortran(b)
    P.summation_bcs(t, g, g, g, *n)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), a)


def _module_and_oracle(n, g, order, pusher, ppc, sigma, seed):
    st = plasma(n, ppc, sigma, seed)
    o = O.OracleSim(n, g, order=order, pusher=pusher)
    o.add_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    m = P.PicsarModule(*n, nguards=g, nox=order, particle_pusher=pusher)
    m.add_species("electron", -1.0, 1.0, st["x"], st["y"], st["z"], st["ux"], st["uy"],
                  st["uz"], st["w"])
    return o, m


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("pusher", [0, 1])
def test_full_step(cuda, order, pusher):
    """Config-1 style state (thermal plasma, periodic): a few full PIC steps
    through the module drivers vs the oracle mini-app."""
    n, g = ((32, 32, 32) if order == 1 else (16, 16, 16)), 3
    o, m = _module_and_oracle(n, g, order, pusher, 8, 0.01 if order == 1 else 0.05, 100 + order)
    nsteps = 2
    o.step(nsteps)
    m.step(nsteps)
    torch.cuda.synchronize()
    m.check_errors()
    for name in ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz"):
        assert rel_l2(getattr(m, name).cpu().numpy(), o.get_field(name)) <= TOL, name
    ref = o.particles()
    sp = m.species[0]
    order_ = torch.argsort(sp.pid_id).cpu().numpy()
    for c, attr in (("x", "part_x"), ("ux", "part_ux"), ("uy", "part_uy"), ("uz", "part_uz"),
                    ("gaminv", "part_gaminv"), ("ex", "part_ex"), ("bz", "part_bz")):
        v = getattr(sp, attr).cpu().numpy()[order_]
        assert rel_l2(v, ref[c]) <= TOL, c


@pytest.mark.parametrize("norder,nodal", [((4, 4, 4), False), ((6, 2, 8), False),
                                          ((4, 6, 2), True), ((8, 8, 8), False)])
def test_yee_norder(cuda, norder, nodal):
    """pxrpush_em3d_bvec_norder / evec_norder (yee.F90:46-123, :752-821):
    B half, E, B half against the oracle (pinned to the reference's own
    routines), stencils clipped at the array ends as in the reference."""
    n, g = (12, 10, 14), 4
    f = random_fields(n, g, seed=1100)
    j = random_fields(n, g, seed=1101)[:3]
    dt = 0.3
    dts = [dt * O.fd_weights(o, nodal) for o in norder]
    half = [0.5 * c for c in dts]
    fo = [a.copy(order="F") for a in f]
    O.push_em3d_bvec_norder(*fo, *half, n, norder, g, nodal)
    O.push_em3d_evec_norder(*fo, *j, dt, *dts, n, norder, g, nodal)
    O.push_em3d_bvec_norder(*fo, *half, n, norder, g, nodal)
    fg = [P.to_fortran(a) for a in f]
    jg = [P.to_fortran(a) for a in j]
    args = (*n, *norder, g, g, g, 0, 0, 0, nodal)
    P.pxrpush_em3d_bvec_norder(*fg, *half, *args)
    P.pxrpush_em3d_evec_norder(*fg, *jg, dt, *dts, *args)
    P.pxrpush_em3d_bvec_norder(*fg, *half, *args)
    torch.cuda.synchronize()
    for a, b, c in zip(fg, fo, ("ex", "ey", "ez", "bx", "by", "bz")):
        assert rel_l2(a.cpu().numpy(), b) <= TOL, c


def test_module_norder_field_push(cuda):
    """PicsarModule with norderx/y/z = 4 (and 6 in z): push_bfield /
    push_efield take the arbitrary-order stencil with FD_weights, as
    maxwell_solver_manager.F90:61-78, :411-433 do."""
    n, g = (16, 12, 14), 4
    m = P.PicsarModule(*n, nguards=g, nox=1)
    m.norderx, m.nordery, m.norderz = 4, 4, 6
    f = random_fields(n, g, seed=1110)
    j = random_fields(n, g, seed=1111)[:3]
    for name, a in zip(("ex", "ey", "ez", "bx", "by", "bz"), f):
        setattr(m, name, P.to_fortran(a))
    for name, a in zip(("jx", "jy", "jz"), j):
        setattr(m, name, P.to_fortran(a))
    m.push_bfield()
    m.push_efield()
    fo = [a.copy(order="F") for a in f]
    c = [O.fd_weights(o) for o in (4, 4, 6)]
    O.push_em3d_bvec_norder(*fo, *[0.5 * m.dt / 1.0 * w for w in c], n, (4, 4, 6), g)
    O.push_em3d_evec_norder(*fo, *j, m.dt, *[m.dt / 1.0 * w for w in c], n, (4, 4, 6), g)
    torch.cuda.synchronize()
    for name, b in zip(("ex", "ey", "ez", "bx", "by", "bz"), fo):
        assert rel_l2(getattr(m, name).cpu().numpy(), b) <= TOL, name


@pytest.mark.parametrize("pbound", [(1, 1, 1, 1, 1, 1), (2, 2, 2, 2, 2, 2), (3, 3, 3, 3, 3, 3),
                                    (1, 2, 0, 3, 2, 1), (0, 0, 0, 0, 0, 0)])
def test_particle_bcs_cases(cuda, pbound):
    """Per-side particle boundaries (particle_boundaries.F90:1098-1300) on
    particles scattered up to 0.9 cells beyond every side, against the
    oracle; the surviving set (compared by id) and every value bit for bit."""
    n = (10, 12, 8)
    rng = np.random.default_rng(1200 + sum(pbound))
    N = 20000
    cols = {c: rng.uniform(-0.9, n[i] + 0.9, N) for i, c in enumerate(("x", "y", "z"))}
    for c in ("ux", "uy", "uz"):
        cols[c] = rng.normal(0.0, 0.1, N)
    cols["gaminv"] = 1.0 / np.sqrt(1.0 + cols["ux"] ** 2 + cols["uy"] ** 2 + cols["uz"] ** 2)
    cols["w"] = rng.uniform(0.5, 1.5, N)
    cols["id"] = np.arange(N, dtype=np.float64)
    m = P.PicsarModule(*n, nguards=3, nox=1)
    (m.pbound_x_min, m.pbound_x_max, m.pbound_y_min, m.pbound_y_max, m.pbound_z_min,
     m.pbound_z_max) = pbound
    sp = m.add_species("e", -1.0, 1.0, cols["x"], cols["y"], cols["z"], cols["ux"], cols["uy"],
                       cols["uz"], cols["w"], pid=cols["id"])
    sp.part_gaminv.copy_(torch.tensor(cols["gaminv"]))
    m.particle_bcs()
    torch.cuda.synchronize()
    ref = {c: v.copy() for c, v in cols.items()}
    k = O.particle_bcs(ref["x"], ref["y"], ref["z"], ref["ux"], ref["uy"], ref["uz"],
                       ref["gaminv"], ref["w"], ref["id"], (0.0, 0.0, 0.0), n, (1.0, 1.0, 1.0),
                       pbound, (-0.5, -0.5, -0.5), n)
    assert sp.np == k
    got = {"x": sp.part_x, "y": sp.part_y, "z": sp.part_z, "ux": sp.part_ux, "uy": sp.part_uy,
           "uz": sp.part_uz, "gaminv": sp.part_gaminv, "w": sp.pid_w, "id": sp.pid_id}
    got = {c: v.cpu().numpy() for c, v in got.items()}
    og, orf = np.argsort(got["id"]), np.argsort(ref["id"][:k])
    for c in got:
        np.testing.assert_array_equal(got[c][og], ref[c][:k][orf], err_msg=c)
    if 1 in pbound:
        assert k < N
