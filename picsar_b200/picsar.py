"""Drop-in surface for PICSAR's Forthon module (``picsarpy.picsar``) on B200.

Two layers, both named after the reference:

* Kernel routines with the Forthon names and positional argument order
  (``field_gathering_plus_particle_pusher_1_1_1``, ``geteb3d_energy_conserving``,
  ``pxr_boris_push_u_3d``, ``pxr_ebcancelpush3d``, ``pxr_set_gamma``,
  ``pxr_pushxyz``, ``depose_jxjyjz``, ``depose_jxjyjz_esirkepov``,
  ``pxrpush_em3d_evec``, ``pxrpush_em3d_bvec``).  Arrays are torch CUDA float64
  tensors; grids use PICSAR's layout (Fortran order, lower bound -guard).
  Values the Fortran reads from module variables (``dt``,
  ``particle_pusher``, ``clight``) are keyword arguments defaulting to the
  module state.  They accumulate into their outputs exactly like the
  reference, and raise ``PicsarB200Error`` where the Fortran would STOP.

* ``PicsarModule``: module variables (``nx``, ``dt``, ``ex`` ... ) and the
  global drivers acting on them (``field_gathering_plus_particle_pusher``,
  ``particle_bcs``, ``pxrdepose_currents_on_grid_jxjyjz``, ``current_bcs``,
  ``push_bfield``, ``bfield_bcs``, ``push_efield``, ``efield_bcs``,
  ``calc_diags``, ``step``), the plain FP64 GPU path of the step loop of
  src/submain.F90:104-195.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import PicsarB200Error

# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------


def fortran_zeros(shape, dtype=torch.float64, device="cuda"):
    """Zero tensor of the given shape with Fortran (column-major) strides."""
    t = torch.zeros(tuple(reversed(shape)), dtype=dtype, device=device)
    return t.permute(*reversed(range(len(shape))))


def grid_zeros(nx, ny, nz, nxg, nyg=None, nzg=None, dtype=torch.float64, device="cuda"):
    """A PICSAR grid array (-g:n+g per axis) as a Fortran-ordered tensor."""
    nyg = nxg if nyg is None else nyg
    nzg = nxg if nzg is None else nzg
    return fortran_zeros((nx + 1 + 2 * nxg, ny + 1 + 2 * nyg, nz + 1 + 2 * nzg), dtype, device)


def to_fortran(a, device="cuda", dtype=torch.float64):
    """Copy a numpy/torch 3-D array into a Fortran-ordered CUDA tensor."""
    t = torch.as_tensor(np.asarray(a) if not torch.is_tensor(a) else a)
    out = fortran_zeros(tuple(t.shape), dtype=dtype, device=device)
    out.copy_(t.to(dtype))
    return out


def is_fortran(t: torch.Tensor) -> bool:
    if t.dim() != 3:
        return False
    s0, s1, s2 = t.shape
    return t.stride() == (1, s0, s0 * s1)


def _ptr(t, name="array", grid=False, dtype=torch.float64):
    if t is None:
        return None
    if not torch.is_tensor(t):
        raise TypeError(f"{name}: expected a torch tensor")
    if not t.is_cuda:
        raise PicsarB200Error(f"{name}: tensor must live on a CUDA device")
    if t.dtype != dtype:
        raise TypeError(f"{name}: expected {dtype}, got {t.dtype}")
    if grid:
        if not is_fortran(t):
            raise ValueError(f"{name}: grid arrays must be Fortran-ordered (x fastest)")
    elif not t.is_contiguous():
        raise ValueError(f"{name}: particle arrays must be contiguous")
    return t.data_ptr()


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _ng(a, n):
    """guard size of a grid of n cells from its extent."""
    g2 = a - 1 - n
    if g2 < 0 or g2 % 2:
        raise ValueError("grid extent inconsistent with cell count")
    return g2 // 2


# ---------------------------------------------------------------------------
# Module state
# ---------------------------------------------------------------------------


@dataclass
class Species:
    """One particle species as flat SoA tensors (the reference keeps them per
    tile, src/modules/modules.F90:335-453; the plain GPU path keeps one array)."""
    name: str
    charge: float
    mass: float
    part_x: torch.Tensor = None
    part_y: torch.Tensor = None
    part_z: torch.Tensor = None
    part_ux: torch.Tensor = None
    part_uy: torch.Tensor = None
    part_uz: torch.Tensor = None
    part_gaminv: torch.Tensor = None
    part_ex: torch.Tensor = None
    part_ey: torch.Tensor = None
    part_ez: torch.Tensor = None
    part_bx: torch.Tensor = None
    part_by: torch.Tensor = None
    part_bz: torch.Tensor = None
    pid_w: torch.Tensor = None        # pid(:, wpid): macro-particle weight
    pid_id: torch.Tensor = None       # a particle identifier column
    ldodepos: bool = True

    @property
    def np(self):
        return 0 if self.part_x is None else int(self.part_x.numel())


class PicsarModule:
    """Module variables and global drivers of the plain FP64 GPU path."""

    def __init__(self, nx, ny, nz, nguards=3, dx=1.0, dy=1.0, dz=1.0, xmin=0.0, ymin=0.0,
                 zmin=0.0, dtcoef=0.95, dt=None, nox=1, particle_pusher=0, clight=1.0,
                 mu0=1.0, eps0=1.0, device="cuda"):
        self.device = torch.device(device)
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.nxguards = self.nyguards = self.nzguards = int(nguards)
        self.nxjguards = self.nyjguards = self.nzjguards = int(nguards)
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)
        self.xmin, self.ymin, self.zmin = float(xmin), float(ymin), float(zmin)
        self.xmax = self.xmin + self.nx * self.dx
        self.ymax = self.ymin + self.ny * self.dy
        self.zmax = self.zmin + self.nz * self.dz
        self.clight, self.mu0, self.eps0 = float(clight), float(mu0), float(eps0)
        self.dtcoef = float(dtcoef)
        if dt is None:
            dt = self.dtcoef / (self.clight * math.sqrt(1.0 / self.dx ** 2 + 1.0 / self.dy ** 2
                                                        + 1.0 / self.dz ** 2))
        self.dt = float(dt)
        self.nox = self.noy = self.noz = int(nox)
        self.particle_pusher = int(particle_pusher)
        self.l_lower_order_in_v = True
        self.currdepo = 0
        self.it = 0
        g = self.nxguards
        mk = lambda: grid_zeros(self.nx, self.ny, self.nz, g, device=self.device)
        self.ex, self.ey, self.ez = mk(), mk(), mk()
        self.bx, self.by, self.bz = mk(), mk(), mk()
        self.jx, self.jy, self.jz = mk(), mk(), mk()
        self.rho, self.dive = mk(), mk()
        self.species = []
        self._err = torch.zeros(1, dtype=torch.int32, device=self.device)

    # -- particles ----------------------------------------------------------
    def add_species(self, name, charge, mass, x, y, z, ux, uy, uz, w, pid=None):
        dev, f = self.device, torch.float64
        t = lambda a: torch.as_tensor(a, dtype=f).to(dev).contiguous()
        sp = Species(name, float(charge), float(mass))
        sp.part_x, sp.part_y, sp.part_z = t(x), t(y), t(z)
        sp.part_ux, sp.part_uy, sp.part_uz = t(ux), t(uy), t(uz)
        n = sp.part_x.numel()
        sp.part_gaminv = torch.empty(n, dtype=f, device=dev)
        pxr_set_gamma(n, sp.part_ux, sp.part_uy, sp.part_uz, sp.part_gaminv, clight=self.clight)
        for c in ("ex", "ey", "ez", "bx", "by", "bz"):
            setattr(sp, "part_" + c, torch.zeros(n, dtype=f, device=dev))
        sp.pid_w = t(w)
        sp.pid_id = t(pid) if pid is not None else torch.arange(n, dtype=f, device=dev)
        self.species.append(sp)
        return sp

    # -- drivers (module-level routines) -----------------------------------
    def field_gathering_plus_particle_pusher(self):
        """particle_pusher_manager_3d.F90:50-112 with one tile spanning the
        domain: zero the particle fields, fused gather + push."""
        fn = {1: field_gathering_plus_particle_pusher_1_1_1,
              2: field_gathering_plus_particle_pusher_2_2_2,
              3: field_gathering_plus_particle_pusher_3_3_3}[self.nox]
        for sp in self.species:
            if sp.np == 0:
                continue
            for c in ("ex", "ey", "ez", "bx", "by", "bz"):
                getattr(sp, "part_" + c).zero_()
            fn(sp.np, sp.part_x, sp.part_y, sp.part_z, sp.part_ux, sp.part_uy, sp.part_uz,
               sp.part_gaminv, sp.part_ex, sp.part_ey, sp.part_ez, sp.part_bx, sp.part_by,
               sp.part_bz, self.xmin, self.ymin, self.zmin, self.dx, self.dy, self.dz, self.dt,
               self.nx, self.ny, self.nz, self.nxguards, self.nyguards, self.nzguards,
               self.ex, self.ey, self.ez, self.bx, self.by, self.bz, sp.charge, sp.mass, 256,
               self.l_lower_order_in_v, dt=self.dt, particle_pusher=self.particle_pusher,
               clight=self.clight)

    def particle_bcs(self):
        """Periodic wrap of every species (particle_boundaries.F90:1109-1300)."""
        for sp in self.species:
            if sp.np == 0:
                continue
            _lib.call("pxrb_particle_bcs_periodic", sp.np, _ptr(sp.part_x), _ptr(sp.part_y),
                      _ptr(sp.part_z), self.xmin, self.ymin, self.zmin, self.xmax, self.ymax,
                      self.zmax, _stream())

    def pxrdepose_currents_on_grid_jxjyjz(self):
        """J = 0, then Esirkepov deposition of every species
        (current_deposition_manager_3d.F90:224-494, currdepo = 0)."""
        self.jx.zero_(); self.jy.zero_(); self.jz.zero_()
        for sp in self.species:
            if sp.np == 0 or not sp.ldodepos:
                continue
            depose_jxjyjz(self.jx, self.jy, self.jz, sp.np, sp.part_x, sp.part_y, sp.part_z,
                          sp.part_ux, sp.part_uy, sp.part_uz, sp.part_gaminv, sp.pid_w,
                          sp.charge, self.xmin, self.ymin, self.zmin, self.dt, self.dx,
                          self.dy, self.dz, self.nx, self.ny, self.nz, self.nxjguards,
                          self.nyjguards, self.nzjguards, self.nox, self.noy, self.noz,
                          self.currdepo, err_flag=self._err)

    def current_bcs(self):
        _summation_bcs(self.jx, self.jy, self.jz, self.nx, self.ny, self.nz, self.nxjguards)

    def charge_bcs(self):
        _summation_bcs(self.rho, None, None, self.nx, self.ny, self.nz, self.nxjguards)

    def push_bfield(self):
        """B half step, order-2 Yee (maxwell_solver_manager.F90:44-85)."""
        n = (self.nx, self.ny, self.nz)
        g = self.nxguards
        pxrpush_em3d_bvec((0, 0, 0), n, (0, 0, 0), n, (0, 0, 0), n,
                          self.ex, (-g,) * 3, tuple(v + g for v in n),
                          self.ey, (-g,) * 3, tuple(v + g for v in n),
                          self.ez, (-g,) * 3, tuple(v + g for v in n),
                          self.bx, (-g,) * 3, tuple(v + g for v in n),
                          self.by, (-g,) * 3, tuple(v + g for v in n),
                          self.bz, (-g,) * 3, tuple(v + g for v in n),
                          0.5 * self.dt / self.dx, 0.5 * self.dt / self.dy,
                          0.5 * self.dt / self.dz)

    def push_efield(self):
        """E full step (maxwell_solver_manager.F90:393-439)."""
        n = (self.nx, self.ny, self.nz)
        g = self.nxguards
        lo, hi = (-g,) * 3, tuple(v + g for v in n)
        c2 = self.clight ** 2
        pxrpush_em3d_evec((0, 0, 0), n, (0, 0, 0), n, (0, 0, 0), n,
                          self.ex, lo, hi, self.ey, lo, hi, self.ez, lo, hi,
                          self.bx, lo, hi, self.by, lo, hi, self.bz, lo, hi,
                          self.jx, lo, hi, self.jy, lo, hi, self.jz, lo, hi,
                          c2 * self.mu0 * self.dt, c2 * self.dt / self.dx,
                          c2 * self.dt / self.dy, c2 * self.dt / self.dz)

    def efield_bcs(self):
        _field_bc(self.ex, self.ey, self.ez, self.nx, self.ny, self.nz, self.nxguards)

    def bfield_bcs(self):
        _field_bc(self.bx, self.by, self.bz, self.nx, self.ny, self.nz, self.nxguards)

    def pxrdepose_rho_on_grid(self):
        self.rho.zero_()
        for sp in self.species:
            if sp.np == 0:
                continue
            _lib.call("pxrb_depose_rho", self.nox, _ptr(self.rho, "rho", grid=True), sp.np,
                      _ptr(sp.part_x), _ptr(sp.part_y), _ptr(sp.part_z), _ptr(sp.pid_w),
                      sp.charge, self.xmin, self.ymin, self.zmin, self.dx, self.dy, self.dz,
                      self.nx, self.ny, self.nz, self.nxjguards, self.nyjguards,
                      self.nzjguards, _stream())

    def calc_diags(self):
        """rho deposition + charge_bcs (diags.F90:63-127)."""
        self.pxrdepose_rho_on_grid()
        self.charge_bcs()

    def step(self, nst=1, diags=False):
        """PIC loop of src/submain.F90:104-195 (Yee solver, l_plasma)."""
        for _ in range(nst):
            self.field_gathering_plus_particle_pusher()
            self.particle_bcs()
            self.pxrdepose_currents_on_grid_jxjyjz()
            self.current_bcs()
            self.push_bfield(); self.bfield_bcs()
            self.push_efield(); self.efield_bcs()
            self.push_bfield(); self.bfield_bcs()
            if diags:
                self.calc_diags()
            self.it += 1

    def check_errors(self):
        if int(self._err.item()) != 0:
            raise PicsarB200Error("a particle moved more than one cell in one step")


def _field_bc(a, b, c, nx, ny, nz, g):
    _lib.call("pxrb_field_bc_periodic", _ptr(a, "f1", grid=True), _ptr(b, "f2", grid=True),
              _ptr(c, "f3", grid=True), nx, ny, nz, g, g, g, _stream())


def _summation_bcs(a, b, c, nx, ny, nz, g):
    _lib.call("pxrb_summation_bcs_periodic", _ptr(a, "f1", grid=True), _ptr(b, "f2", grid=True),
              _ptr(c, "f3", grid=True), nx, ny, nz, g, g, g, _stream())


def field_bc(field, nxg, nyg, nzg, nx_local, ny_local, nz_local):
    """field_bc (field_boundaries.F90:81) for one periodic domain."""
    _lib.call("pxrb_field_bc_periodic", _ptr(field, "field", grid=True), None, None,
              nx_local, ny_local, nz_local, nxg, nyg, nzg, _stream())


def summation_bcs(array, nxg, nyg, nzg, nx_local, ny_local, nz_local):
    """summation_bcs (field_boundaries.F90:403) for one periodic domain."""
    _lib.call("pxrb_summation_bcs_periodic", _ptr(array, "array", grid=True), None, None,
              nx_local, ny_local, nz_local, nxg, nyg, nzg, _stream())


# ---------------------------------------------------------------------------
# Kernel routines (Forthon names and argument order)
# ---------------------------------------------------------------------------
_DEFAULT_MODULE = {"dt": None, "particle_pusher": 0, "clight": 1.0}


def _fgp(order, np_, xp, yp, zp, uxp, uyp, uzp, gaminv, ex, ey, ez, bx, by, bz, xmin, ymin,
         zmin, dx, dy, dz, dtt, nx, ny, nz, nxguard, nyguard, nzguard, exg, eyg, ezg, bxg, byg,
         bzg, q, m, lvect, l_lower_order_in_v, dt=None, particle_pusher=None, clight=None):
    if dt is None:
        dt = _DEFAULT_MODULE["dt"] if _DEFAULT_MODULE["dt"] is not None else dtt
    pp =_DEFAULT_MODULE["particle_pusher"] if particle_pusher is None else particle_pusher
    cl = _DEFAULT_MODULE["clight"] if clight is None else clight
    parts = [_ptr(a, n) for a, n in zip(
        (xp, yp, zp, uxp, uyp, uzp, gaminv, ex, ey, ez, bx, by, bz),
        ("xp", "yp", "zp", "uxp", "uyp", "uzp", "gaminv", "ex", "ey", "ez", "bx", "by", "bz"))]
    grids = [_ptr(a, n, grid=True) for a, n in zip(
        (exg, eyg, ezg, bxg, byg, bzg), ("exg", "eyg", "ezg", "bxg", "byg", "bzg"))]
    _lib.call("pxrb_field_gathering_plus_particle_pusher", order, int(np_), *parts,
              float(xmin), float(ymin), float(zmin), float(dx), float(dy), float(dz),
              float(dtt), int(nx), int(ny), int(nz), int(nxguard), int(nyguard), int(nzguard),
              *grids, float(q), float(m), int(lvect), int(bool(l_lower_order_in_v)), float(dt),
              int(pp), float(cl), _stream())


def field_gathering_plus_particle_pusher_1_1_1(*args, **kw):
    """particle_pusher_manager_3d.F90:1287."""
    _fgp(1, *args, **kw)


def field_gathering_plus_particle_pusher_2_2_2(*args, **kw):
    """particle_pusher_manager_3d.F90:1522."""
    _fgp(2, *args, **kw)


def field_gathering_plus_particle_pusher_3_3_3(*args, **kw):
    """particle_pusher_manager_3d.F90:1820."""
    _fgp(3, *args, **kw)


def geteb3d_energy_conserving(np_, xp, yp, zp, ex, ey, ez, bx, by, bz, xmin, ymin, zmin, dx,
                              dy, dz, nx, ny, nz, nxguard, nyguard, nzguard, nox, noy, noz,
                              exg, eyg, ezg, bxg, byg, bzg, ll4symtry, l_lower_order_in_v,
                              lvect, field_gathe_algo, l_nodal=False):
    """field_gathering_manager_3d.F90:295-323 (l_nodal = module l_nodalgrid)."""
    parts = [_ptr(a) for a in (xp, yp, zp, ex, ey, ez, bx, by, bz)]
    grids = [_ptr(a, grid=True) for a in (exg, eyg, ezg, bxg, byg, bzg)]
    _lib.call("pxrb_geteb3d_energy_conserving", int(np_), *parts, float(xmin), float(ymin),
              float(zmin), float(dx), float(dy), float(dz), int(nx), int(ny), int(nz),
              int(nxguard), int(nyguard), int(nzguard), int(nox), int(noy), int(noz), *grids,
              int(bool(ll4symtry)), int(bool(l_lower_order_in_v)), int(lvect),
              int(field_gathe_algo), int(bool(l_nodal)), _stream())


def pxr_boris_push_u_3d(np_, uxp, uyp, uzp, gaminv, ex, ey, ez, bx, by, bz, q, m, dt,
                        clight=None):
    """boris_3d.F90:51."""
    cl = _DEFAULT_MODULE["clight"] if clight is None else clight
    _lib.call("pxrb_boris_push_u_3d", int(np_),
              *[_ptr(a) for a in (uxp, uyp, uzp, gaminv, ex, ey, ez, bx, by, bz)],
              float(q), float(m), float(dt), float(cl), _stream())


def pxr_ebcancelpush3d(np_, uxp, uyp, uzp, gi, ex, ey, ez, bx, by, bz, q, m, dt, which,
                       clight=None):
    """vay_3d.F90:56."""
    cl = _DEFAULT_MODULE["clight"] if clight is None else clight
    _lib.call("pxrb_ebcancelpush3d", int(np_),
              *[_ptr(a) for a in (uxp, uyp, uzp, gi, ex, ey, ez, bx, by, bz)],
              float(q), float(m), float(dt), int(which), float(cl), _stream())


def pxr_set_gamma(np_, uxp, uyp, uzp, gaminv, clight=None):
    """boris_3d.F90:1059."""
    cl = _DEFAULT_MODULE["clight"] if clight is None else clight
    _lib.call("pxrb_set_gamma", int(np_), *[_ptr(a) for a in (uxp, uyp, uzp, gaminv)],
              float(cl), _stream())


def pxr_pushxyz(np_, xp, yp, zp, uxp, uyp, uzp, gaminv, dt):
    """boris_3d.F90:849."""
    _lib.call("pxrb_pushxyz", int(np_), *[_ptr(a) for a in (xp, yp, zp, uxp, uyp, uzp, gaminv)],
              float(dt), _stream())


def depose_jxjyjz(jx, jy, jz, np_, xp, yp, zp, uxp, uyp, uzp, gaminv, w, q, xmin, ymin, zmin,
                  dt, dx, dy, dz, nx, ny, nz, nxguard, nyguard, nzguard, nox, noy, noz,
                  current_depo_algo=0, err_flag=None):
    """current_deposition_manager_3d.F90:47 (current_depo_algo 0: specialised
    Esirkepov, 1: arbitrary-order form)."""
    own = err_flag is None
    if own:
        err_flag = torch.zeros(1, dtype=torch.int32, device=jx.device)
    _lib.call("pxrb_depose_jxjyjz", *[_ptr(a, grid=True) for a in (jx, jy, jz)], int(np_),
              *[_ptr(a) for a in (xp, yp, zp, uxp, uyp, uzp, gaminv, w)], float(q),
              float(xmin), float(ymin), float(zmin), float(dt), float(dx), float(dy), float(dz),
              int(nx), int(ny), int(nz), int(nxguard), int(nyguard), int(nzguard), int(nox),
              int(noy), int(noz), int(current_depo_algo),
              _ptr(err_flag, "err_flag", dtype=torch.int32), _stream())


def depose_jxjyjz_esirkepov(jx, jy, jz, np_, xp, yp, zp, uxp, uyp, uzp, gaminv, w, q, xmin,
                            ymin, zmin, dt, dx, dy, dz, nx, ny, nz, nxguard, nyguard, nzguard,
                            nox, noy, noz):
    """current_deposition_manager_3d.F90:75 (arbitrary-order Esirkepov)."""
    depose_jxjyjz(jx, jy, jz, np_, xp, yp, zp, uxp, uyp, uzp, gaminv, w, q, xmin, ymin, zmin,
                  dt, dx, dy, dz, nx, ny, nz, nxguard, nyguard, nzguard, nox, noy, noz, 1)


def _b3(v):
    a = np.ascontiguousarray(np.asarray(v, dtype=np.int64).reshape(3))
    return a, a.ctypes.data


def pxrpush_em3d_evec(xlo, xhi, ylo, yhi, zlo, zhi, ex, exlo, exhi, ey, eylo, eyhi, ez, ezlo,
                      ezhi, bx, bxlo, bxhi, by, bylo, byhi, bz, bzlo, bzhi, jx, jxlo, jxhi, jy,
                      jylo, jyhi, jz, jzlo, jzhi, mudt, dtsdx, dtsdy, dtsdz):
    """yee.F90:637-740."""
    keep, args = [], []
    for v in (xlo, xhi, ylo, yhi, zlo, zhi):
        a, p = _b3(v); keep.append(a); args.append(p)
    for arr, lo, hi in ((ex, exlo, exhi), (ey, eylo, eyhi), (ez, ezlo, ezhi), (bx, bxlo, bxhi),
                        (by, bylo, byhi), (bz, bzlo, bzhi), (jx, jxlo, jxhi), (jy, jylo, jyhi),
                        (jz, jzlo, jzhi)):
        a1, p1 = _b3(lo); a2, p2 = _b3(hi); keep += [a1, a2]
        _check_bounds(arr, a1, a2)
        args += [_ptr(arr, grid=True), p1, p2]
    _lib.call("pxrb_push_em3d_evec", *args, float(mudt), float(dtsdx), float(dtsdy),
              float(dtsdz), _stream())


def pxrpush_em3d_bvec(xlo, xhi, ylo, yhi, zlo, zhi, ex, exlo, exhi, ey, eylo, eyhi, ez, ezlo,
                      ezhi, bx, bxlo, bxhi, by, bylo, byhi, bz, bzlo, bzhi, dtsdx, dtsdy,
                      dtsdz):
    """yee.F90:1258-1347."""
    keep, args = [], []
    for v in (xlo, xhi, ylo, yhi, zlo, zhi):
        a, p = _b3(v); keep.append(a); args.append(p)
    for arr, lo, hi in ((ex, exlo, exhi), (ey, eylo, eyhi), (ez, ezlo, ezhi), (bx, bxlo, bxhi),
                        (by, bylo, byhi), (bz, bzlo, bzhi)):
        a1, p1 = _b3(lo); a2, p2 = _b3(hi); keep += [a1, a2]
        _check_bounds(arr, a1, a2)
        args += [_ptr(arr, grid=True), p1, p2]
    _lib.call("pxrb_push_em3d_bvec", *args, float(dtsdx), float(dtsdy), float(dtsdz),
              _stream())


def _check_bounds(arr, lo, hi):
    ext = tuple(int(h - l + 1) for l, h in zip(lo, hi))
    if tuple(arr.shape) != ext:
        raise ValueError(f"array shape {tuple(arr.shape)} does not match bounds {ext}")
