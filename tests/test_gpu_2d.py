"""The 2D (x-z) path on the GPU against the oracle (whose 2D routines are
pinned bit for bit to the reference's own, tests/test_oracle_vs_reference.py):
the separate gather at orders 1-3 (both l_lower_order_in_v branches, nodal
grid), the 2D Esirkepov deposition at orders 1-3, the 2D Yee pushes and
pxr_pushxz, and full 2D PIC steps of PicsarModule2D against the same steps
composed from the oracle's routines in the reference's order
(submain.F90, c_dim = 2).  Bar: relative L2 <= 1e-12 (FP64).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from picsar_b200 import picsar as P
from tests._cases import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12
N2, G = (20, 16), 3


def _grids(seed, k=6, amp=0.05):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        a = O.zeros_grid2d(*N2, G)
        a[...] = amp * rng.standard_normal(a.shape)
        out.append(a)
    return out


def _parts(seed, npart=4000, usig=0.1):
    rng = np.random.default_rng(seed)
    p = {"x": rng.uniform(0, N2[0], npart), "y": rng.uniform(0, 1, npart),
         "z": rng.uniform(0, N2[1], npart)}
    for c in ("ux", "uy", "uz"):
        p[c] = usig * rng.standard_normal(npart)
    p["gaminv"] = 1.0 / np.sqrt(1.0 + p["ux"] ** 2 + p["uy"] ** 2 + p["uz"] ** 2)
    p["w"] = rng.uniform(0.5, 1.5, npart) * N2[0] * N2[1] / npart
    return p


def _t(a):
    return torch.tensor(a, device="cuda")


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("lower,nodal", [(True, False), (False, False), (True, True)])
def test_gather_2d(cuda, order, lower, nodal):
    p = _parts(1300 + order)
    g = _grids(1310 + order)
    ref = [np.zeros(len(p["x"])) for _ in range(6)]
    O.geteb2dxz(0, p["x"], p["z"], *ref[:3], 0.0, 0.0, 1.0, 1.0, N2, G, order, *g[:3], lower,
                nodal)
    O.geteb2dxz(1, p["x"], p["z"], *ref[3:], 0.0, 0.0, 1.0, 1.0, N2, G, order, *g[3:], lower,
                nodal)
    got = [torch.zeros(len(p["x"]), dtype=torch.float64, device="cuda") for _ in range(6)]
    P.geteb2dxz_energy_conserving(len(p["x"]), _t(p["x"]), _t(p["y"]), _t(p["z"]), *got, 0.0,
                                  0.0, 0.0, 1.0, 1.0, 1.0, N2[0], 0, N2[1], G, 0, G, order, order,
                                  order, *[P.to_fortran(a) for a in g], False, lower, 256, 0,
                                  l_nodal=nodal)
    torch.cuda.synchronize()
    for a, b, c in zip(got, ref, ("ex", "ey", "ez", "bx", "by", "bz")):
        assert rel_l2(a.cpu().numpy(), b) <= TOL, c


@pytest.mark.parametrize("order", [1, 2, 3])
def test_esirkepov_2d(cuda, order):
    p = _parts(1320 + order, usig=0.3)
    dt = 0.6
    ref = [O.zeros_grid2d(*N2, G) for _ in range(3)]
    O.depose_jxjyjz_esirkepov2d(order, *ref, p["x"], p["z"], p["ux"], p["uy"], p["uz"],
                                p["gaminv"], p["w"], -1.0, 0.0, 0.0, dt, 1.0, 1.0, N2, G)
    got = [P.grid2d_zeros(*N2, G) for _ in range(3)]
    P.depose_jxjyjz_2d(*got, len(p["x"]), *[_t(p[c]) for c in ("x", "y", "z", "ux", "uy", "uz",
                                                                "gaminv", "w")],
                       -1.0, 0.0, 0.0, dt, 1.0, 1.0, N2[0], N2[1], G, G, order, order, 256)
    torch.cuda.synchronize()
    for a, b, c in zip(got, ref, ("jx", "jy", "jz")):
        assert rel_l2(a.cpu().numpy(), b) <= TOL, c


def test_yee_2d_and_pushxz(cuda):
    f = _grids(1330)
    j = _grids(1331, k=3)
    fo = [a.copy(order="F") for a in f]
    dt = 0.5
    O.push_em2d_bvec(*fo, N2, G, 0.5 * dt, 0.5 * dt)
    O.push_em2d_evec(*fo, *j, N2, G, dt, dt, dt)
    fg = [P.to_fortran(a) for a in f]
    jg = [P.to_fortran(a) for a in j]
    lo, hi, a, b = (-G, -G), (N2[0] + G, N2[1] + G), (0, 0), N2
    P.pxrpush_em2d_bvec(a, b, a, b, a, b, *sum([[x, lo, hi] for x in fg], []), 0.5 * dt, 0.0,
                        0.5 * dt)
    P.pxrpush_em2d_evec(a, b, a, b, a, b, *sum([[x, lo, hi] for x in fg + jg], []), dt, dt,
                        0.0, dt)
    p = _parts(1332)
    xo, zo = p["x"].copy(), p["z"].copy()
    O.pushxz(xo, zo, p["ux"], p["uz"], p["gaminv"], dt)
    xg, zg = _t(p["x"]), _t(p["z"])
    P.pxr_pushxz(len(xo), xg, zg, _t(p["ux"]), _t(p["uz"]), _t(p["gaminv"]), dt)
    torch.cuda.synchronize()
    for x, y, c in zip(fg, fo, ("ex", "ey", "ez", "bx", "by", "bz")):
        assert rel_l2(x.cpu().numpy(), y) <= TOL, c
    assert rel_l2(xg.cpu().numpy(), xo) <= TOL and rel_l2(zg.cpu().numpy(), zo) <= TOL


def _oracle_step_2d(f, j, p, order, pusher, dt, q=-1.0, m=1.0):
    """One 2D PIC step from the oracle's routines, in the reference's order."""
    npart = len(p["x"])
    pf = [np.zeros(npart) for _ in range(6)]
    O.geteb2dxz(0, p["x"], p["z"], *pf[:3], 0.0, 0.0, 1.0, 1.0, N2, G, order, *f[:3], True)
    O.geteb2dxz(1, p["x"], p["z"], *pf[3:], 0.0, 0.0, 1.0, 1.0, N2, G, order, *f[3:], True)
    if pusher == 1:
        O.ebcancelpush3d(p["ux"], p["uy"], p["uz"], p["gaminv"], *pf, q, m, dt, 0)
    else:
        O.boris_push_u(p["ux"], p["uy"], p["uz"], p["gaminv"], *pf, q, m, dt)
    O.pushxz(p["x"], p["z"], p["ux"], p["uz"], p["gaminv"], dt)
    for c, n in (("x", N2[0]), ("z", N2[1])):
        v = p[c]
        v[v < 0] += n
        v[v >= n] -= n
    for a in j:
        a[...] = 0.0
    O.depose_jxjyjz_esirkepov2d(order, *j, p["x"], p["z"], p["ux"], p["uy"], p["uz"],
                                p["gaminv"], p["w"], q, 0.0, 0.0, dt, 1.0, 1.0, N2, G)
    for a in j:
        O.summation_bcs_2d(a, N2, G)

    def bc(arrs):
        for a in arrs:
            O.field_bc_2d(a, N2, G)
    O.push_em2d_bvec(*f, N2, G, 0.5 * dt, 0.5 * dt)
    bc(f[3:])
    O.push_em2d_evec(*f, *j, N2, G, dt, dt, dt)
    bc(f[:3])
    O.push_em2d_bvec(*f, N2, G, 0.5 * dt, 0.5 * dt)
    bc(f[3:])


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("pusher", [0, 1])
def test_module_2d_steps(cuda, order, pusher):
    p = _parts(1340 + order, npart=6000, usig=0.05)
    f = _grids(1350 + order, amp=0.02)
    for a in f:
        O.field_bc_2d(a, N2, G)
    m = P.PicsarModule2D(*N2, nguards=G, nox=order, particle_pusher=pusher)
    for name, a in zip(("ex", "ey", "ez", "bx", "by", "bz"), f):
        setattr(m, name, P.to_fortran(a))
    m.add_species("electron", -1.0, 1.0, p["x"], p["y"], p["z"], p["ux"], p["uy"], p["uz"],
                  p["w"])
    po = {c: v.copy() for c, v in p.items()}
    po["gaminv"] = m.species[0].part_gaminv.cpu().numpy().copy()
    fo = [a.copy(order="F") for a in f]
    jo = [O.zeros_grid2d(*N2, G) for _ in range(3)]
    for _ in range(3):
        _oracle_step_2d(fo, jo, po, order, pusher, m.dt)
    m.step(3)
    torch.cuda.synchronize()
    for name, b in zip(("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz"), fo + jo):
        assert rel_l2(getattr(m, name).cpu().numpy(), b) <= TOL, name
    sp = m.species[0]
    for c in ("x", "z", "ux", "uy", "uz", "gaminv"):
        attr = "part_" + c
        assert rel_l2(getattr(sp, attr).cpu().numpy(), po[c]) <= TOL, c
