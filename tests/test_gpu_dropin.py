"""The Forthon-named module surface (``PicsarModule``) driving the tiled engine,
and ``pxr_particle_sorting`` on both engines, against the CPU oracle.

FP64 bar: relative L2 <= 1e-12 after full PIC steps (fields E, B, J and the
particles' u, gamma^-1 and x).  FP32 mixed precision: the engine's stated bars
after one step (2e-5 for fields, 1e-6 for momenta).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from picsar_b200 import picsar as P
from picsar_b200.tiled import TiledConfig
from tests._cases import plasma, random_fields, rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz")


def _oracle(n, g, order, pusher, st, fields=None, sorting_period=0):
    o = O.OracleSim(n, g, order=order, pusher=pusher, sorting_period=sorting_period)
    if fields is not None:
        for name, a in zip(FIELDS[:6], fields):
            o.set_field(name, a)
    o.add_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    return o


def _module(n, g, order, pusher, st, fields=None, **kw):
    m = P.PicsarModule(*n, nguards=g, nox=order, particle_pusher=pusher, **kw)
    if fields is not None:
        for name, a in zip(FIELDS[:6], fields):
            setattr(m, name, P.to_fortran(a))
    m.add_species("electron", -1.0, 1.0, st["x"], st["y"], st["z"], st["ux"], st["uy"],
                  st["uz"], st["w"])
    return m


def _check(m, o, ftol, ptol, fields=FIELDS):
    torch.cuda.synchronize()
    m.check_errors()
    for name in fields:
        err = rel_l2(getattr(m, name).cpu().numpy(), o.get_field(name))
        assert err <= ftol, (name, err)
    ref = o.particles()
    sp = m.species[0]
    ids = sp.pid_id.cpu().numpy()
    srt = np.argsort(ids, kind="stable")
    assert np.array_equal(ids[srt], ref["id"])
    for c, attr in (("ux", "part_ux"), ("uy", "part_uy"), ("uz", "part_uz"),
                    ("gaminv", "part_gaminv")):
        err = rel_l2(getattr(sp, attr).cpu().numpy()[srt], ref[c])
        assert err <= ptol, (c, err)
    for c, attr, L in (("x", "part_x", o.n[0]), ("y", "part_y", o.n[1]), ("z", "part_z", o.n[2])):
        d = (getattr(sp, attr).cpu().numpy()[srt] - ref[c] + L / 2) % L - L / 2
        assert np.linalg.norm(d) / np.linalg.norm(ref[c]) <= ptol, c


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("pusher", [0, 1])
def test_module_step_on_tiled_fp64(cuda, order, pusher):
    """PicsarModule(engine='tiled', precision='fp64').step(n) == oracle."""
    n, g = (16, 24, 16), 3
    st = plasma(n, 4, 0.05, seed=900 + order)
    fields = random_fields(n, g, seed=910 + order, amp=0.02)
    o = _oracle(n, g, order, pusher, st, fields)
    m = _module(n, g, order, pusher, st, fields, engine="tiled", precision="fp64",
                tiled_config=TiledConfig(tile=(8, 8, 8), sort_interval=2, relayout_interval=0))
    o.step(3)
    m.step(3)
    _check(m, o, 1e-12, 1e-12)


@pytest.mark.parametrize("order", [1, 3])
def test_module_drivers_on_tiled_fp64(cuda, order):
    """The reference's driver sequence (submain.F90:113-174) called routine by
    routine, with a module array edited in place between steps, gives the
    oracle's state; the boundary routines are no-ops on the tiled engine."""
    n, g = (16, 16, 16), 3
    st = plasma(n, 4, 0.05, seed=920 + order)
    fields = random_fields(n, g, seed=930 + order, amp=0.02)
    o = _oracle(n, g, order, 0, st, fields)
    m = _module(n, g, order, 0, st, fields, engine="tiled", precision="fp64")
    for _ in range(2):
        m.field_gathering_plus_particle_pusher()
        m.particle_bcs()
        m.pxr_particle_sorting()
        m.pxrdepose_currents_on_grid_jxjyjz()
        m.current_bcs()
        m.push_bfield(); m.bfield_bcs()
        m.push_efield(); m.efield_bcs()
        m.push_bfield(); m.bfield_bcs()
    o.step(2)
    _check(m, o, 1e-12, 1e-12)
    # edit a module array in place, as a Forthon caller would, and continue
    bump = random_fields(n, g, seed=940, amp=0.01)[0]
    m.ez.add_(P.to_fortran(bump))
    o.set_field("ez", o.get_field("ez") + bump)
    m.step(1)
    o.step(1)
    _check(m, o, 1e-12, 1e-12)


def test_module_deposit_needs_the_fused_kernel(cuda):
    n, g = (16, 16, 16), 3
    st = plasma(n, 1, 0.05, seed=950)
    m = _module(n, g, 1, 0, st, engine="tiled", precision="fp64")
    with pytest.raises(P.PicsarB200Error, match="fused"):
        m.pxrdepose_currents_on_grid_jxjyjz()


@pytest.mark.parametrize("order", [1, 2, 3])
def test_module_step_on_tiled_fp32(cuda, order):
    n, g = (16, 16, 24), 3
    st = plasma(n, 8, 0.05, seed=960 + order)
    fields = random_fields(n, g, seed=970 + order, amp=0.02)
    o = _oracle(n, g, order, 0, st, fields)
    m = _module(n, g, order, 0, st, fields, engine="tiled", precision="fp32")
    o.step(1)
    m.step(1)
    _check(m, o, 2e-5, 1e-6)


def test_particle_particles_in_original_order(cuda):
    """part_* arrays of the tiled engine come back in the order the
    particles were added, whatever the engine's internal sorting."""
    n, g = (16, 16, 16), 3
    st = plasma(n, 2, 0.05, seed=980)
    m = _module(n, g, 2, 0, st, engine="tiled", precision="fp64")
    sp = m.species[0]
    assert np.array_equal(sp.pid_id.cpu().numpy(), np.arange(len(st["x"]), dtype=np.float64))
    assert np.allclose(sp.part_x.cpu().numpy(), st["x"], rtol=0, atol=1e-12)
    assert np.array_equal(sp.pid_w.cpu().numpy(), st["w"])


# ---------------------------------------------------------------------------
# pxr_particle_sorting / pxr_particle_bin_sorting (sorting.F90:67-361)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("dbin", [(1.0, 1.0, 1.0), (2.0, 1.0, 3.0)])
def test_bin_sorting_matches_oracle(cuda, dbin):
    n = (16, 12, 20)
    st = plasma(n, 3, 0.05, seed=990)
    gam = 1.0 / np.sqrt(1.0 + st["ux"] ** 2 + st["uy"] ** 2 + st["uz"] ** 2)
    cols = [st[c].copy() for c in ("x", "y", "z", "ux", "uy", "uz")] + [gam, st["w"].copy()]
    dev = [torch.tensor(c, device="cuda") for c in cols]
    lo = (0.5, 0.0, -0.25)
    hi = (n[0] + dbin[0], n[1] + dbin[1], n[2] + dbin[2])
    O.particle_bin_sorting(*cols, lo, hi, dbin)
    P.pxr_particle_bin_sorting(len(st["x"]), *dev[:7], dev[7], *lo, *hi, *dbin)
    torch.cuda.synchronize()
    for a, b in zip(dev, cols):
        assert np.array_equal(a.cpu().numpy(), b)


@pytest.mark.parametrize("order", [1, 3])
def test_module_sorting_plain_engine(cuda, order):
    """sorting_activated with a species sorting period: the plain engine sorts
    between push and deposit, as the reference's step (submain.F90:113-134),
    and matches the oracle mini-app with the same period, particle order
    included."""
    n, g = (16, 16, 16), 3
    st = plasma(n, 4, 0.05, seed=1000 + order)
    o = _oracle(n, g, order, 0, st, sorting_period=2)
    m = P.PicsarModule(*n, nguards=g, nox=order)
    m.sorting_activated = 1
    m.add_species("electron", -1.0, 1.0, st["x"], st["y"], st["z"], st["ux"], st["uy"],
                  st["uz"], st["w"], sorting_period=2)
    o.step(4)
    m.step(4)
    torch.cuda.synchronize()
    ref = o.particles(sort_by_id=False)
    sp = m.species[0]
    assert np.array_equal(sp.pid_w.cpu().numpy(), ref["w"])
    for c, attr in (("x", "part_x"), ("ux", "part_ux"), ("gaminv", "part_gaminv")):
        assert rel_l2(getattr(sp, attr).cpu().numpy(), ref[c]) <= 1e-12, c
    for name in FIELDS:
        assert rel_l2(getattr(m, name).cpu().numpy(), o.get_field(name)) <= 1e-12, name
