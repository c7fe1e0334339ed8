"""CPU tests of the oracle: the reference's own cross-variant checks and
physics invariants, restated on seeded inputs (no GPU).

The reference's test programs compare variants of the same routine and check
invariants of the full loop:
  * Esirkepov specialised vs arbitrary order (Acceptance_testing/Gcov_tests/
    esirkepov_3d_test.F90:173-306, bound 1e-3 on sum J);
  * scalar vs fused gather (field_gathering_test.F90:108,206-554, 1e-6);
  * tiled gather+push variants (tile_particle_push_3d_test.F90:127, 1e-6);
  * tiled vs untiled current (tile_curr_depo_3d_test.F90:116, 1e-5);
  * energy of the homogeneous plasma (Fortran_tests/test_homogeneous_plasma/
    test_homogeneous_plasma.py:157, 1e-2);
  * Yee plane wave vs analytic (maxwell_3d_test.F90:146, 5e-2);
  * Langmuir oscillation period (test_langmuir_wave.py:222);
  * charge continuity d(rho)/dt + div J = 0 (Python_tests/test_Langmuir_wave/
    test_Langmuir_wave_3d.py:582, 1e-5).
The bounds here are tighter where a faithful FP64 restatement allows.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests._cases import fresh_particles, plasma, random_fields, rel_l2

N, G = (12, 10, 14), 3


def _part(seed, n=N, ppc=2, sigma=0.2):
    return fresh_particles(plasma(n, ppc, sigma, seed))


def _dt(d=(1.0, 1.0, 1.0)):
    return 0.95 / np.sqrt(sum(1 / x ** 2 for x in d))


# ---------------------------------------------------------------------------
@pytest.mark.parametrize("order", [1, 2, 3])
def test_esirkepov_specialised_vs_arbitrary_order(order):
    p = _part(10 + order)
    dt = _dt()
    js = [[O.zeros_grid(*N, G) for _ in range(3)] for _ in range(2)]
    for algo, j in zip((0, 1), js):
        O.depose_jxjyjz(order, *j, p["x"], p["y"], p["z"], p["ux"], p["uy"], p["uz"],
                        p["gaminv"], p["w"], -1.0, (0, 0, 0), dt, (1, 1, 1), N, G, algo=algo)
    for a, b in zip(*js):
        assert rel_l2(a, b) < 1e-13
        assert abs(a.sum() - b.sum()) <= 1e-12 * np.abs(a).sum()


@pytest.mark.parametrize("order", [1, 2, 3])
def test_scalar_gather_matches_fused_gather(order):
    p = _part(20 + order)
    grids = random_fields(N, G, seed=30 + order, amp=0.1)
    dt = _dt()
    fused = {k: v.copy() for k, v in p.items()}
    O.gather_push(order, fused, grids, (0, 0, 0), (1, 1, 1), N, G, -1.0, 1.0, dt, 0)
    e = [np.zeros_like(p["x"]) for _ in range(3)]
    b = [np.zeros_like(p["x"]) for _ in range(3)]
    O.geteb3d_scalar(0, order, p["x"], p["y"], p["z"], *e, (0, 0, 0), (1, 1, 1), N, G,
                     *grids[:3])
    O.geteb3d_scalar(1, order, p["x"], p["y"], p["z"], *b, (0, 0, 0), (1, 1, 1), N, G,
                     *grids[3:])
    for a, c in zip(e + b, ("ex", "ey", "ez", "bx", "by", "bz")):
        assert rel_l2(fused[c], a) < 1e-14, c


def test_pushers_limits():
    """Boris and Vay agree for E-only fields (both exact leapfrog in u), and
    a pure-B rotation conserves |u| to round-off."""
    rng = np.random.default_rng(3)
    n = 1000
    u = [rng.standard_normal(n) for _ in range(3)]
    gi = 1 / np.sqrt(1 + u[0] ** 2 + u[1] ** 2 + u[2] ** 2)
    e = [0.3 * rng.standard_normal(n) for _ in range(3)]
    z = [np.zeros(n) for _ in range(3)]
    a = [x.copy() for x in u] + [gi.copy()]
    b = [x.copy() for x in u] + [gi.copy()]
    O.boris_push_u(*a, *e, *z, -1.0, 1.0, 0.5)
    O.ebcancelpush3d(*b, *e, *z, -1.0, 1.0, 0.5, 0)
    for x, y in zip(a[:3], b[:3]):
        assert rel_l2(x, y) < 1e-14
    bf = [0.8 * rng.standard_normal(n) for _ in range(3)]
    c = [x.copy() for x in u] + [gi.copy()]
    O.boris_push_u(*c, *z, *bf, -1.0, 1.0, 0.5)
    n0 = np.sqrt(u[0] ** 2 + u[1] ** 2 + u[2] ** 2)
    n1 = np.sqrt(c[0] ** 2 + c[1] ** 2 + c[2] ** 2)
    assert np.max(np.abs(n1 - n0) / n0) < 1e-14


# ---------------------------------------------------------------------------
def _sim(tiles, order=2, pusher=0, n=(16, 16, 16), seed=5, steps=3, sigma=0.05, ppc=2,
         fields_seed=6):
    st = plasma(n, ppc, sigma, seed)
    s = O.OracleSim(n, G, order=order, pusher=pusher, tiles=tiles)
    for name, a in zip(("ex", "ey", "ez", "bx", "by", "bz"),
                       random_fields(n, G, seed=fields_seed, amp=0.02)):
        s.set_field(name, a)
    s.add_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    s.step(steps)
    return s


@pytest.mark.parametrize("order", [1, 2, 3])
def test_tiled_vs_untiled(order):
    """Particles are identical bit for bit (gather and push do not depend on
    tiling); fields agree to summation-order round-off."""
    a = _sim((1, 1, 1), order=order)
    b = _sim((4, 2, 4), order=order)
    pa, pb = a.particles(), b.particles()
    for c in ("x", "y", "z", "ux", "uy", "uz", "gaminv"):
        assert rel_l2(pa[c], pb[c]) < 1e-13, c
    for f in ("jx", "jy", "jz", "ex", "ey", "ez", "bx", "by", "bz"):
        assert rel_l2(a.get_field(f), b.get_field(f)) < 1e-12, f


@pytest.mark.parametrize("order", [1, 2, 3])
def test_charge_continuity(order):
    """(rho(n+1) - rho(n))/dt + div J(n+1/2) = 0 for Esirkepov + depose_rho."""
    n = (12, 12, 12)
    st = plasma(n, 4, 0.1, 40 + order)
    p = fresh_particles(st)
    dt = _dt()
    r0, r1 = O.zeros_grid(*n, G), O.zeros_grid(*n, G)
    O.depose_rho(order, r0, p["x"], p["y"], p["z"], p["w"], -1.0, (0, 0, 0), (1, 1, 1), n, G)
    O.pushxyz(p["x"], p["y"], p["z"], p["ux"], p["uy"], p["uz"], p["gaminv"], dt)
    O.depose_rho(order, r1, p["x"], p["y"], p["z"], p["w"], -1.0, (0, 0, 0), (1, 1, 1), n, G)
    j = [O.zeros_grid(*n, G) for _ in range(3)]
    O.depose_jxjyjz(order, *j, p["x"], p["y"], p["z"], p["ux"], p["uy"], p["uz"],
                    p["gaminv"], p["w"], -1.0, (0, 0, 0), dt, (1, 1, 1), n, G)
    for a in (r0, r1, *j):
        O.summation_bcs(a, n, G)
    s = slice(G, G + n[0])
    jx, jy, jz = j
    div = (jx[s, s, s] - jx[G - 1:G - 1 + n[0], s, s]) + (jy[s, s, s] - jy[s, G - 1:G - 1 + n[1], s]) \
        + (jz[s, s, s] - jz[s, s, G - 1:G - 1 + n[2]])
    drho = (r1[s, s, s] - r0[s, s, s]) / dt
    res = np.linalg.norm(drho + div) / np.linalg.norm(drho)
    assert res < 1e-12, res


@pytest.mark.parametrize("pusher", [0, 1])
def test_homogeneous_plasma_energy(pusher):
    """Total (kinetic + field) energy of a thermal plasma stays within 1 % of
    its maximum over about two plasma periods.  As in the reference's run,
    the Debye length is resolved (lambda_D = u_th/omega_p = 0.5 cells here:
    n0 = 0.04, omega_p = 0.2, u_th = 0.1), order-1 shapes."""
    from picsar_b200.init import thermal_plasma
    n = (16, 16, 16)
    st = thermal_plasma(n, 8, 0.1, 50, n0=0.04).numpy()
    s = O.OracleSim(n, G, order=1, pusher=pusher, tiles=(2, 2, 2))
    s.add_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    tot = []
    for _ in range(12):
        s.step(5)
        tot.append(s.diags()["total"])
    tot = np.array(tot)
    assert (tot.max() - tot.min()) / tot.max() < 1e-2, tot


def test_yee_plane_wave():
    """Vacuum plane wave along x through 40 full steps of the field solver
    (B half-push, E push, B half-push) against the discrete analytic wave:
    omega = 2/dt asin(dt/dx sin(k dx/2)), and B stored at integer time levels
    is E * cos(omega dt/2) at the half-integer x of B_z."""
    n = (64, 4, 4)
    dt = 0.5
    s = O.OracleSim(n, G, dt=dt, tiles=(1, 1, 1))
    k = 2 * np.pi / n[0]
    w = 2 / dt * np.arcsin(dt * np.sin(k / 2))
    i = np.arange(-G, n[0] + G + 1)
    shape = O.grid_shape(*n, G)
    ey = np.zeros(shape, order="F")
    bz = np.zeros(shape, order="F")
    ey[...] = np.sin(k * i)[:, None, None]
    bz[...] = (np.cos(w * dt / 2) * np.sin(k * (i + 0.5)))[:, None, None]
    s.set_field("ey", ey)
    s.set_field("bz", bz)
    steps = 40
    s.step(steps)
    got = s.get_field("ey")[G:G + n[0], G + 1, G + 1]
    ref = np.sin(k * np.arange(n[0]) - w * steps * dt)
    err = np.max(np.abs(got - ref))
    assert err < 1e-10, err


def test_langmuir_period():
    """Cold plasma with a sinusoidal velocity perturbation oscillates at the
    plasma frequency (omega_p = 1 in normalised units, n0 = 1): the field
    energy peaks every half period, corrected for the leapfrog's numerical
    frequency 2/dt*asin(omega_p*dt/2)."""
    n = (16, 4, 4)
    st = plasma(n, 8, 0.0, 60)
    k = 2 * np.pi / n[0]
    st["ux"] = 0.01 * np.sin(k * st["x"])
    dt = _dt()
    s = O.OracleSim(n, G, order=1, tiles=(1, 1, 1))
    s.add_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    ef = []
    for _ in range(60):
        s.step(1)
        ef.append(s.diags()["ex"])
    ef = np.array(ef)
    peaks = [i for i in range(1, len(ef) - 1) if ef[i] > ef[i - 1] and ef[i] >= ef[i + 1]]
    assert len(peaks) >= 4
    half = np.mean(np.diff(peaks)) * dt
    w_num = 2 / dt * np.arcsin(dt / 2)
    assert abs(half - np.pi / w_num) / (np.pi / w_num) < 0.08, (half, np.pi / w_num)


def test_field_bc_and_summation_bcs_periodic():
    n = (6, 5, 7)
    rng = np.random.default_rng(9)
    a = O.zeros_grid(*n, G)
    a[...] = rng.standard_normal(a.shape)
    b = a.copy(order="F")
    O.field_bc(b, n, G)
    # guard images: index -g..-1 <- n-g..n-1, n+1..n+g <- 1..g (node n is the periodic image of 0
    # kept as computed), for every axis
    for ax in range(3):
        sl = [slice(None)] * 3
        sl[ax] = slice(0, G)
        src = [slice(None)] * 3
        src[ax] = slice(n[ax], n[ax] + G)
        np.testing.assert_array_equal(b[tuple(sl)], b[tuple(src)])
    c = a.copy(order="F")
    tot = c[G:G + n[0], G:G + n[1], G:G + n[2]].sum() + 0.0
    O.summation_bcs(c, n, G)
    # folding the guards conserves the total over the periodic box
    full = a.sum()
    inner = c[G:G + n[0], G:G + n[1], G:G + n[2]].sum()
    assert abs(inner - full) < 1e-10 * np.abs(a).sum(), (inner, full, tot)


def test_golden_fixtures_reproduce():
    """The committed golden fixtures (tests/golden/oracle_steps.npz, made by
    tests/golden/make_golden.py) are reproduced exactly by the oracle."""
    from tests.golden import make_golden
    fx = np.load(make_golden.PATH)
    for case in make_golden.CASES:
        out = make_golden.run_case(**case)
        tag = make_golden.tag(**case)
        for k, v in out.items():
            np.testing.assert_array_equal(v, fx[f"{tag}/{k}"], err_msg=f"{tag}/{k}")


def test_bin_sorting_is_a_stable_sort_by_bin():
    """The oracle's pxr_particle_bin_sorting (sorting.F90:247-361) equals a
    stable argsort by the reference's bin number."""
    from oracle import oracle as O
    rng = np.random.default_rng(5)
    n = 5000
    lo, hi, d = (0.0, -1.0, 2.0), (8.0, 5.0, 12.0), (1.0, 0.5, 2.0)
    x = rng.uniform(lo[0], hi[0], n)
    y = rng.uniform(lo[1], hi[1], n)
    z = rng.uniform(lo[2], hi[2], n)
    cols = [x, y, z] + [rng.standard_normal(n) for _ in range(4)] + [np.arange(n, dtype=np.float64)]
    nb = [int(np.ceil((h - l) / dd)) for l, h, dd in zip(lo, hi, d)]
    key = (np.floor((z - lo[2]) / d[2]) * nb[0] * nb[1] + np.floor((y - lo[1]) / d[1]) * nb[0]
           + np.floor((x - lo[0]) / d[0])).astype(np.int64)
    perm = np.argsort(key, kind="stable")
    want = [c[perm] for c in cols]
    got = [c.copy() for c in cols]
    O.particle_bin_sorting(*got, lo, hi, d)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("norder", [2, 4, 6, 8, 16, 32])
@pytest.mark.parametrize("nodal", [False, True])
def test_library_fd_weights_match_oracle(norder, nodal):
    """pxrb_fd_weights (a host function of the library, no GPU needed) gives
    the oracle's FD_weights (itself pinned to the reference's routine) bit
    for bit."""
    from picsar_b200 import picsar as P
    got = P.FD_weights(np.zeros(norder // 2), norder, nodal)
    np.testing.assert_array_equal(got, O.fd_weights(norder, nodal))
