"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py``.  Nothing in the ``picsar_b200``
package imports this module.

The oracle restates PICSAR's Fortran hot path (see the header of
``pxr_oracle.cpp`` for the routine-by-routine citations).  Arrays follow the
Fortran convention: float64, column-major, lower bound ``-g`` per axis, i.e.
a numpy array of shape ``(nx+1+2g, ny+1+2g, nz+1+2g)`` in Fortran order.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

i64 = C.c_int64
f64 = C.c_double
vp = C.c_void_p


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    src = os.path.join(_HERE, "pxr_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "-s", "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _p(a):
    if a is None:
        return None
    if a.dtype != np.float64 and a.dtype != np.int64:
        raise TypeError(f"oracle arrays must be float64/int64, got {a.dtype}")
    if a.ndim >= 2 and not a.flags.f_contiguous:
        raise ValueError("oracle grids must be Fortran-ordered (np.asfortranarray)")
    if a.ndim < 2 and not a.flags.c_contiguous:
        raise ValueError("oracle particle arrays must be contiguous")
    return a.ctypes.data_as(vp)


def _declare(L):
    P = vp
    L.orc_boris_push_u_3d.argtypes = [i64] + [P] * 10 + [f64] * 4
    L.orc_set_gamma.argtypes = [i64, P, P, P, P, f64]
    L.orc_pushxyz.argtypes = [i64] + [P] * 7 + [f64]
    L.orc_ebcancelpush3d.argtypes = [i64] + [P] * 10 + [f64] * 3 + [i64, f64]
    fgp = [i64] + [P] * 13 + [f64] * 6 + [i64] * 6 + [P] * 6 + [f64, f64, i64, f64, i64, f64]
    for o in (1, 2, 3):
        getattr(L, f"orc_field_gathering_plus_particle_pusher_{o}_{o}_{o}").argtypes = fgp
    L.orc_geteb3d_energy_conserving_scalar.argtypes = (
        [i64, i64] + [P] * 6 + [f64] * 6 + [i64] * 7 + [P] * 3 + [i64, i64])
    dep = [P, P, P, i64] + [P] * 8 + [f64] * 8 + [i64] * 6
    L.orc_depose_jxjyjz_esirkepov_1_1_1.argtypes = dep
    L.orc_depose_jxjyjz_esirkepov_2_2_2.argtypes = dep
    L.orc_depose_jxjyjz_esirkepov_3_3_3.argtypes = dep
    L.orc_pxr_depose_jxjyjz_esirkepov_n.argtypes = dep + [i64, i64, i64, f64]
    L.orc_depose_jxjyjz.argtypes = dep + [i64, i64, i64, i64, f64]
    L.orc_depose_rho_scalar.argtypes = [i64, P, i64, P, P, P, P] + [f64] * 7 + [i64] * 6
    L.orc_pxrpush_em3d_evec.argtypes = [P] + [P] * 9 + [P, P] + [f64] * 4
    L.orc_pxrpush_em3d_bvec.argtypes = [P] + [P] * 6 + [P, P] + [f64] * 3
    L.orc_field_bc_periodic.argtypes = [P] + [i64] * 6
    L.orc_summation_bcs_periodic.argtypes = [P] + [i64] * 6
    L.orc_calc_field_div.argtypes = [P, P, P, P] + [i64] * 6 + [f64] * 3
    L.orc_field_energy.argtypes = [P] + [i64] * 6 + [f64] * 3
    L.orc_field_energy.restype = f64
    L.orc_kinetic_energy.argtypes = [i64, P, P]
    L.orc_kinetic_energy.restype = f64
    L.orc_norm_diverho.argtypes = [P, P] + [i64] * 6 + [f64]
    L.orc_norm_diverho.restype = f64
    L.orc_sim_new.argtypes = [i64] * 4 + [f64] * 12 + [i64] * 7
    L.orc_sim_new.restype = vp
    L.orc_sim_free.argtypes = [vp]
    L.orc_sim_grid_size.argtypes = [vp]
    L.orc_sim_grid_size.restype = i64
    L.orc_sim_field.argtypes = [vp, i64, P, i64]
    L.orc_sim_add_particles.argtypes = [vp, i64] + [P] * 8
    L.orc_sim_np.argtypes = [vp]
    L.orc_sim_np.restype = i64
    L.orc_sim_get_particles.argtypes = [vp, P]
    L.orc_sim_step.argtypes = [vp, i64, i64]
    L.orc_sim_diags.argtypes = [vp, P]
    L.orc_sim_phase.argtypes = [vp, i64]
    L.orc_num_threads.restype = C.c_int
    L.orc_particle_bin_sorting.argtypes = [i64] + [P] * 8 + [f64] * 9
    L.orc_sim_get_particle_columns.argtypes = [vp, P, i64, P]
    L.orc_pxrpush_em3d_evec_norder.argtypes = [P] * 9 + [f64, P, P, P] + [i64] * 13
    L.orc_pxrpush_em3d_bvec_norder.argtypes = [P] * 6 + [P, P, P] + [i64] * 13
    L.orc_FD_weights.argtypes = [P, i64, i64]
    L.orc_particle_bcs.argtypes = [i64] + [P] * 9 + [P] * 4 + [P, P]
    L.orc_particle_bcs.restype = i64
    L.orc_geteb2dxz_energy_conserving_scalar.argtypes = (
        [i64, i64, P, P, P, P, P] + [f64] * 4 + [i64] * 5 + [P] * 3 + [i64, i64])
    L.orc_depose_jxjyjz_esirkepov2d.argtypes = ([i64] + [P] * 3 + [i64] + [P] * 7 +
                                                [f64] * 6 + [i64] * 4)
    L.orc_pxrpush_em2d_evec.argtypes = [P] + [P] * 9 + [i64] * 3 + [f64] * 3
    L.orc_pxrpush_em2d_bvec.argtypes = [P] + [P] * 6 + [i64] * 3 + [f64] * 2
    L.orc_pushxz.argtypes = [i64] + [P] * 5 + [f64]
    L.orc_field_bc_periodic_2d.argtypes = [P] + [i64] * 4
    L.orc_summation_bcs_periodic_2d.argtypes = [P] + [i64] * 4


def _c(a):
    """Contiguous float64 view (Fortran order for 3-D grids)."""
    a = np.asarray(a)
    if a.ndim == 3:
        return np.asfortranarray(a, dtype=np.float64)
    return np.ascontiguousarray(a, dtype=np.float64)


def grid_shape(nx, ny, nz, g):
    return (nx + 1 + 2 * g, ny + 1 + 2 * g, nz + 1 + 2 * g)


def zeros_grid(nx, ny, nz, g):
    return np.zeros(grid_shape(nx, ny, nz, g), dtype=np.float64, order="F")


# ---------------------------------------------------------------------------
# Kernel-level wrappers (in place on numpy arrays)
# ---------------------------------------------------------------------------
def boris_push_u(ux, uy, uz, gaminv, ex, ey, ez, bx, by, bz, q, m, dt, clight=1.0):
    lib().orc_boris_push_u_3d(len(ux), _p(ux), _p(uy), _p(uz), _p(gaminv), _p(ex), _p(ey),
                              _p(ez), _p(bx), _p(by), _p(bz), q, m, dt, clight)


def set_gamma(ux, uy, uz, gaminv, clight=1.0):
    lib().orc_set_gamma(len(ux), _p(ux), _p(uy), _p(uz), _p(gaminv), clight)


def pushxyz(x, y, z, ux, uy, uz, gaminv, dt):
    lib().orc_pushxyz(len(x), _p(x), _p(y), _p(z), _p(ux), _p(uy), _p(uz), _p(gaminv), dt)


def particle_bcs(x, y, z, ux, uy, uz, gi, w, ids, lo, hi, d, pbound, tlo, thi):
    """particle_bcs of one domain with per-side codes (in place); returns the
    number of particles left (the first n entries of every array)."""
    v = [np.ascontiguousarray(a, dtype=np.float64) for a in (lo, hi, d, tlo, thi)]
    pb = np.ascontiguousarray(pbound, dtype=np.int64)
    return lib().orc_particle_bcs(len(x), _p(x), _p(y), _p(z), _p(ux), _p(uy), _p(uz), _p(gi),
                                  _p(w), _p(ids), _p(v[0]), _p(v[1]), _p(v[2]), _p(pb),
                                  _p(v[3]), _p(v[4]))


def zeros_grid2d(nx, nz, g):
    """A 2-D (x-z) PICSAR grid (-g:n+g) per axis, Fortran order."""
    return np.zeros((nx + 1 + 2 * g, nz + 1 + 2 * g), dtype=np.float64, order="F")


def geteb2dxz(which, xp, zp, f1, f2, f3, xmin, zmin, dx, dz, n, g, order, g1, g2, g3,
              lower=True, nodal=False):
    """2-D energy-conserving gather (which 0: E, 1: B), accumulating."""
    lib().orc_geteb2dxz_energy_conserving_scalar(
        which, len(xp), _p(xp), _p(zp), _p(f1), _p(f2), _p(f3), xmin, zmin, dx, dz, n[0],
        n[1], g, g, order, _p(g1), _p(g2), _p(g3), int(bool(lower)), int(bool(nodal)))


def depose_jxjyjz_esirkepov2d(order, jx, jy, jz, x, z, ux, uy, uz, gi, w, q, xmin, zmin, dt,
                              dx, dz, n, g):
    lib().orc_depose_jxjyjz_esirkepov2d(order, _p(jx), _p(jy), _p(jz), len(x), _p(x), _p(z),
                                        _p(ux), _p(uy), _p(uz), _p(gi), _p(w), q, xmin, zmin, dt,
                                        dx, dz, n[0], n[1], g, g)


def push_em2d_evec(ex, ey, ez, bx, by, bz, jx, jy, jz, n, g, mudt, dtsdx, dtsdz, bnds=None):
    b = np.ascontiguousarray(bnds if bnds is not None else [0, 0, n[0], n[1]] * 3, dtype=np.int64)
    lib().orc_pxrpush_em2d_evec(_p(b), *[_p(a) for a in (ex, ey, ez, bx, by, bz, jx, jy, jz)],
                                n[0], n[1], g, mudt, dtsdx, dtsdz)


def push_em2d_bvec(ex, ey, ez, bx, by, bz, n, g, dtsdx, dtsdz, bnds=None):
    b = np.ascontiguousarray(bnds if bnds is not None else [0, 0, n[0], n[1]] * 3, dtype=np.int64)
    lib().orc_pxrpush_em2d_bvec(_p(b), *[_p(a) for a in (ex, ey, ez, bx, by, bz)], n[0], n[1],
                                g, dtsdx, dtsdz)


def field_bc_2d(f, n, g):
    lib().orc_field_bc_periodic_2d(_p(f), n[0], n[1], g, g)


def summation_bcs_2d(f, n, g):
    lib().orc_summation_bcs_periodic_2d(_p(f), n[0], n[1], g, g)


def pushxz(x, z, ux, uz, gi, dt):
    lib().orc_pushxz(len(x), _p(x), _p(z), _p(ux), _p(uz), _p(gi), dt)


def fd_weights(norder, nodal=False):
    """FD_weights: the norder/2 first-derivative weights."""
    c = np.zeros(max(norder // 2, 1), dtype=np.float64)
    lib().orc_FD_weights(_p(c), norder, int(bool(nodal)))
    return c[:norder // 2]


def push_em3d_evec_norder(ex, ey, ez, bx, by, bz, jx, jy, jz, mudt, dtsdx, dtsdy, dtsdz, n,
                          norder, g, nodal=False, ns=(0, 0, 0)):
    """pxrpush_em3d_evec_norder on Fortran-ordered (-g:n+g)^3 grids, in place."""
    c = [np.ascontiguousarray(v, dtype=np.float64) for v in (dtsdx, dtsdy, dtsdz)]
    lib().orc_pxrpush_em3d_evec_norder(*[_p(a) for a in (ex, ey, ez, bx, by, bz, jx, jy, jz)],
                                       mudt, *[_p(a) for a in c], *n, *norder, g, g, g, *ns,
                                       int(bool(nodal)))


def push_em3d_bvec_norder(ex, ey, ez, bx, by, bz, dtsdx, dtsdy, dtsdz, n, norder, g,
                          nodal=False, ns=(0, 0, 0)):
    """pxrpush_em3d_bvec_norder on Fortran-ordered (-g:n+g)^3 grids, in place."""
    c = [np.ascontiguousarray(v, dtype=np.float64) for v in (dtsdx, dtsdy, dtsdz)]
    lib().orc_pxrpush_em3d_bvec_norder(*[_p(a) for a in (ex, ey, ez, bx, by, bz)],
                                       *[_p(a) for a in c], *n, *norder, g, g, g, *ns,
                                       int(bool(nodal)))


def particle_bin_sorting(x, y, z, ux, uy, uz, gam, w, lo, hi, dbin):
    """pxr_particle_bin_sorting on flat float64 arrays, in place; w may be None."""
    lib().orc_particle_bin_sorting(len(x), _p(x), _p(y), _p(z), _p(ux), _p(uy), _p(uz),
                                   _p(gam), None if w is None else _p(w), *lo, *hi, *dbin)


def ebcancelpush3d(ux, uy, uz, gi, ex, ey, ez, bx, by, bz, q, m, dt, which, clight=1.0):
    lib().orc_ebcancelpush3d(len(ux), _p(ux), _p(uy), _p(uz), _p(gi), _p(ex), _p(ey), _p(ez),
                             _p(bx), _p(by), _p(bz), q, m, dt, which, clight)


def gather_push(order, part, grids, xmin, d, n, g, q, m, dt, pusher, lvect=256, clight=1.0):
    """Fused gather + push of order 1..3.  ``part`` is a dict of float64 arrays
    x y z ux uy uz gaminv ex ey ez bx by bz (modified in place); ``grids`` the
    six guarded field arrays ex..bz."""
    fn = getattr(lib(), f"orc_field_gathering_plus_particle_pusher_{order}_{order}_{order}")
    k = part
    fn(len(k["x"]), *[_p(k[c]) for c in ("x", "y", "z", "ux", "uy", "uz", "gaminv",
                                         "ex", "ey", "ez", "bx", "by", "bz")],
       xmin[0], xmin[1], xmin[2], d[0], d[1], d[2], n[0], n[1], n[2], g, g, g,
       *[_p(a) for a in grids], q, m, lvect, dt, pusher, clight)


def geteb3d_scalar(which, order, x, y, z, f1, f2, f3, xmin, d, n, g, g1, g2, g3,
                   lower=True, nodal=False):
    lib().orc_geteb3d_energy_conserving_scalar(
        which, len(x), _p(x), _p(y), _p(z), _p(f1), _p(f2), _p(f3), xmin[0], xmin[1], xmin[2],
        d[0], d[1], d[2], n[0], n[1], n[2], g, g, g, order, _p(g1), _p(g2), _p(g3),
        int(bool(lower)), int(bool(nodal)))


def depose_jxjyjz(order, jx, jy, jz, x, y, z, ux, uy, uz, gaminv, w, q, xmin, dt, d, n, g,
                  algo=0, clight=1.0):
    """depose_jxjyjz_generic: algo 0 -> specialised Esirkepov, 1 -> generic _n."""
    lib().orc_depose_jxjyjz(_p(jx), _p(jy), _p(jz), len(x), _p(x), _p(y), _p(z), _p(ux), _p(uy),
                            _p(uz), _p(gaminv), _p(w), q, xmin[0], xmin[1], xmin[2], dt,
                            d[0], d[1], d[2], n[0], n[1], n[2], g, g, g, order, order, order,
                            algo, clight)


def depose_rho(order, rho, x, y, z, w, q, xmin, d, n, g):
    lib().orc_depose_rho_scalar(order, _p(rho), len(x), _p(x), _p(y), _p(z), _p(w), q,
                                xmin[0], xmin[1], xmin[2], d[0], d[1], d[2], n[0], n[1],
                                n[2], g, g, g)


def push_evec(ex, ey, ez, bx, by, bz, jx, jy, jz, n, g, mudt, dtsdx, dtsdy, dtsdz):
    bnds = np.array([0, 0, 0, n[0], n[1], n[2]] * 3, dtype=np.int64)
    lo = np.array([-g] * 27, dtype=np.int64)
    hi = np.array([n[0] + g, n[1] + g, n[2] + g] * 9, dtype=np.int64)
    lib().orc_pxrpush_em3d_evec(_p(bnds), _p(ex), _p(ey), _p(ez), _p(bx), _p(by), _p(bz),
                                _p(jx), _p(jy), _p(jz), _p(lo), _p(hi), mudt, dtsdx, dtsdy,
                                dtsdz)


def push_bvec(ex, ey, ez, bx, by, bz, n, g, dtsdx, dtsdy, dtsdz):
    bnds = np.array([0, 0, 0, n[0], n[1], n[2]] * 3, dtype=np.int64)
    lo = np.array([-g] * 18, dtype=np.int64)
    hi = np.array([n[0] + g, n[1] + g, n[2] + g] * 6, dtype=np.int64)
    lib().orc_pxrpush_em3d_bvec(_p(bnds), _p(ex), _p(ey), _p(ez), _p(bx), _p(by), _p(bz),
                                _p(lo), _p(hi), dtsdx, dtsdy, dtsdz)


def field_bc(f, n, g):
    lib().orc_field_bc_periodic(_p(f), n[0], n[1], n[2], g, g, g)


def summation_bcs(f, n, g):
    lib().orc_summation_bcs_periodic(_p(f), n[0], n[1], n[2], g, g, g)


def calc_field_div(dive, ex, ey, ez, n, g, d):
    lib().orc_calc_field_div(_p(dive), _p(ex), _p(ey), _p(ez), n[0], n[1], n[2], g, g, g,
                             d[0], d[1], d[2])


def field_energy(f, n, g, d):
    return lib().orc_field_energy(_p(f), n[0], n[1], n[2], g, g, g, d[0], d[1], d[2])


def kinetic_energy(gaminv, w):
    return lib().orc_kinetic_energy(len(gaminv), _p(gaminv), _p(w))


def norm_diverho(dive, rho, n, g, eps0=1.0):
    return lib().orc_norm_diverho(_p(dive), _p(rho), n[0], n[1], n[2], g, g, g, eps0)


# ---------------------------------------------------------------------------
# Mini-app (tile drivers + step loop)
# ---------------------------------------------------------------------------
FIELD_NAMES = ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz", "rho", "dive")
PART_COLS = ("x", "y", "z", "ux", "uy", "uz", "gaminv", "ex", "ey", "ez", "bx", "by", "bz",
             "w", "id")


class OracleSim:
    """CPU restatement of the PICSAR mini-app step() for one species on a
    periodic single domain."""

    def __init__(self, n, g, d=(1.0, 1.0, 1.0), xmin=(0.0, 0.0, 0.0), dt=None, q=-1.0,
                 m=1.0, order=1, pusher=0, tiles=(1, 1, 1), lvect=256, sorting_period=0,
                 clight=1.0, mu0=1.0, eps0=1.0):
        if dt is None:
            dt = 0.95 / (clight * np.sqrt(1 / d[0] ** 2 + 1 / d[1] ** 2 + 1 / d[2] ** 2))
        self.n, self.g, self.d, self.xmin = tuple(n), g, tuple(d), tuple(xmin)
        self.dt, self.q, self.m, self.order, self.pusher = dt, q, m, order, pusher
        self.clight, self.mu0, self.eps0 = clight, mu0, eps0
        self.h = lib().orc_sim_new(n[0], n[1], n[2], g, d[0], d[1], d[2], xmin[0], xmin[1],
                                   xmin[2], dt, q, m, clight, mu0, eps0, order, pusher,
                                   tiles[0], tiles[1], tiles[2], lvect, sorting_period)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_sim_free(self.h)
            self.h = None

    def set_field(self, name, arr):
        a = _c(arr)
        assert a.shape == grid_shape(*self.n, self.g)
        lib().orc_sim_field(self.h, FIELD_NAMES.index(name), _p(a), 0)

    def get_field(self, name):
        a = zeros_grid(*self.n, self.g)
        lib().orc_sim_field(self.h, FIELD_NAMES.index(name), _p(a), 1)
        return a

    def add_particles(self, x, y, z, ux, uy, uz, w, pid=None):
        arrs = [_c(a) for a in (x, y, z, ux, uy, uz, w)]
        if pid is None:
            pid = np.arange(len(x), dtype=np.float64)
        pid = _c(pid)
        lib().orc_sim_add_particles(self.h, len(arrs[0]), *[_p(a) for a in arrs], _p(pid))

    def particles(self, sort_by_id=True):
        np_ = lib().orc_sim_np(self.h)
        buf = np.zeros(15 * np_, dtype=np.float64)
        lib().orc_sim_get_particles(self.h, _p(buf))
        cols = {c: buf[i * np_:(i + 1) * np_] for i, c in enumerate(PART_COLS)}
        if sort_by_id:
            o = np.argsort(cols["id"], kind="stable")
            cols = {c: v[o] for c, v in cols.items()}
        return cols

    def columns(self, names):
        """Selected particle columns (PART_COLS names) in the oracle's tile
        order, without copying the others (large particle counts)."""
        np_ = lib().orc_sim_np(self.h)
        idx = np.array([PART_COLS.index(c) for c in names], dtype=np.int64)
        buf = np.empty(len(names) * np_, dtype=np.float64)
        lib().orc_sim_get_particle_columns(self.h, _p(idx), len(names), _p(buf))
        return {c: buf[i * np_:(i + 1) * np_] for i, c in enumerate(names)}

    def step(self, nsteps=1, diag=False):
        lib().orc_sim_step(self.h, nsteps, int(bool(diag)))

    def phase(self, p):
        lib().orc_sim_phase(self.h, p)

    def diags(self):
        out = np.zeros(8)
        lib().orc_sim_diags(self.h, _p(out))
        return {"kinetic": out[0], "ex": out[1], "ey": out[2], "ez": out[3], "bx": out[4],
                "by": out[5], "bz": out[6], "gauss_norm": out[7],
                "field": float(out[1:7].sum()), "total": float(out[0] + out[1:7].sum())}


def num_threads():
    return lib().orc_num_threads()
