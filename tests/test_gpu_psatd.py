"""The spectral (PSATD) field push on the GPU against the oracle's restatement
(oracle/psatd.py) of the reference's local-FFT push: random guarded fields,
currents and charge densities on small domains with odd and even FFT
extents, staggered and centred stencils of several orders and the infinite
order; then the module's spectral PIC steps (submain.F90:101-150 with
l_spectral) against the same steps with the oracle's push.
Bar: relative L2 <= 1e-12 (FP64; the FFT libraries differ).
"""
import numpy as np
import pytest
import torch

from oracle import psatd as OP
from picsar_b200 import picsar as P
from picsar_b200.psatd import PsatdSolver, fd_weights_hvincenti, k_vectors
from tests._cases import rel_l2

pytestmark = pytest.mark.gpu

NAMES = ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz", "rho", "rhoold")


def _fields(n, g, seed):
    rng = np.random.default_rng(seed)
    shape = tuple(n[a] + 1 + 2 * g[a] for a in range(3))
    return {k: np.asfortranarray(rng.standard_normal(shape)) for k in NAMES}


def test_setup_matches_oracle():
    for p in (2, 4, 8, 16):
        for stg in (True, False):
            assert np.array_equal(fd_weights_hvincenti(p, stg), OP.fd_weights_hvincenti(p, stg))
    for nfft, p, stg in ((18, 2, True), (19, 4, True), (20, 6, False), (17, 0, True)):
        a, b = k_vectors(nfft, p, 0.7, stg), OP.compute_k_1d(nfft, p, 0.7, stg)
        for x, y in zip(a, b):
            assert np.allclose(x, y, rtol=0, atol=1e-14 * np.abs(y).max())


@pytest.mark.parametrize("n,g,order,stg", [((12, 10, 14), (3, 3, 3), (2, 2, 2), True),
                                           ((13, 9, 11), (2, 3, 4), (4, 6, 8), True),
                                           ((12, 12, 12), (3, 3, 3), (2, 4, 2), False),
                                           ((10, 11, 12), (3, 3, 3), (0, 0, 0), True)])
def test_psatd_push_matches_oracle(cuda, n, g, order, stg):
    d, dt, c, eps0, mu0 = (0.7, 0.9, 1.1), 0.35, 1.3, 0.8, 1.0 / (1.3 ** 2 * 0.8)
    f = _fields(n, g, seed=sum(n) + order[0])
    ref = {k: v.copy(order="F") for k, v in f.items()}
    OP.Psatd(n, g, d, dt, order, stg, c, eps0, mu0).push(ref)
    got = {k: P.to_fortran(v) for k, v in f.items()}
    s = PsatdSolver(n, g, d, dt, order, stg, c, eps0, mu0)
    s.push(*[got[k] for k in NAMES])
    torch.cuda.synchronize()
    for k in ("ex", "ey", "ez", "bx", "by", "bz"):
        assert rel_l2(got[k].cpu().numpy(), ref[k]) <= 1e-12, k
    for k in ("jx", "rho", "rhoold"):                     # inputs untouched
        assert np.array_equal(got[k].cpu().numpy(), f[k]), k


def _module(seed, n=(12, 10, 14), g=3):
    rng = np.random.default_rng(seed)
    m = P.PicsarModule(*n, nguards=g, nox=2, dx=0.8, dy=0.9, dz=1.0, dt=0.45)
    m.l_spectral = True
    npart = 3000
    x = rng.uniform(0, n[0] * 0.8, npart)
    y = rng.uniform(0, n[1] * 0.9, npart)
    z = rng.uniform(0, n[2] * 1.0, npart)
    u = 0.05 * rng.standard_normal((3, npart))
    w = np.full(npart, 0.3)
    m.add_species("electron", -1.0, 1.0, x, y, z, *u, w)
    return m


def test_spectral_steps_against_oracle_push(cuda):
    """Two modules on the same particles: one steps with the GPU push, the
    other with the same drivers in the same order and the oracle's push."""
    a, b = _module(5), _module(5)
    a.step(3)
    n, g = (b.nx, b.ny, b.nz), (b.nxguards,) * 3
    ref = OP.Psatd(n, g, (b.dx, b.dy, b.dz), b.dt, (2, 2, 2), True, b.clight, b.eps0, b.mu0)
    b.rho.zero_()
    b.rhoold.zero_()
    for _ in range(3):
        b.field_gathering_plus_particle_pusher()
        b.particle_bcs()
        b.rhoold.copy_(b.rho)
        b.pxrdepose_rho_on_grid()
        b.charge_bcs()
        b.pxr_particle_sorting()
        b.pxrdepose_currents_on_grid_jxjyjz()
        b.current_bcs()
        grids = {k: getattr(b, k).cpu().numpy().copy(order="F") for k in NAMES}
        ref.push(grids)
        for k in ("ex", "ey", "ez", "bx", "by", "bz"):
            getattr(b, k).copy_(P.to_fortran(grids[k]))
        b.efield_bcs()
        b.bfield_bcs()
    torch.cuda.synchronize()
    for k in ("ex", "ey", "ez", "bx", "by", "bz", "jx", "rho"):
        assert rel_l2(getattr(a, k).cpu().numpy(), getattr(b, k).cpu().numpy()) <= 1e-12, k
    for c in ("part_x", "part_ux", "part_uz"):
        assert rel_l2(getattr(a.species[0], c).cpu().numpy(),
                      getattr(b.species[0], c).cpu().numpy()) <= 1e-12, c


@pytest.mark.parametrize("norder", [2, 8, 0])
def test_vacuum_plane_wave_keeps_its_energy(cuda, norder):
    """A vacuum plane wave along z whose wavelength divides both the domain
    (32 cells) and the FFT extent (32 + 2 * 8 guards): 64 spectral pushes
    (with the periodic field exchanges) keep its E^2 + B^2 to 1e-12 and keep
    it uniform in x and y."""
    import math
    n, g = 32, 8
    m = P.PicsarModule(n, n, n, nguards=g, dx=1.0, dy=1.0, dz=1.0, dt=0.5)
    m.l_spectral = True
    m.norderx = m.nordery = m.norderz = norder
    z = torch.arange(-g, n + g + 1, dtype=torch.float64, device="cuda")
    k = 2 * math.pi / 16
    full = (n + 1 + 2 * g,) * 3
    m.ex.copy_(torch.cos(k * z)[None, None, :].expand(full))
    m.by.copy_(torch.cos(k * (z + 0.5) + k * 0.25)[None, None, :].expand(full))
    inner = (slice(g, g + n),) * 3
    energy = lambda: float((m.ex[inner] ** 2).sum() + (m.by[inner] ** 2).sum() +
                           (m.ez[inner] ** 2).sum() + (m.bx[inner] ** 2).sum())
    e0 = energy()
    for _ in range(64):
        m.push_psatd_ebfield()
        m.efield_bcs()
        m.bfield_bcs()
    torch.cuda.synchronize()
    assert abs(energy() / e0 - 1.0) < 1e-12
    ex = m.ex[inner]
    assert float((ex - ex[:1, :1, :]).abs().max()) < 1e-12
