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
  ``particle_bcs``, ``pxr_particle_sorting``,
  ``pxrdepose_currents_on_grid_jxjyjz``, ``current_bcs``, ``push_bfield``,
  ``bfield_bcs``, ``push_efield``, ``efield_bcs``, ``calc_diags``, ``step``),
  the step loop of src/submain.F90:104-195, on one of two engines:

  - ``engine="plain"``: PICSAR's own arrays in FP64, one kernel per routine
    (the comparison baseline);
  - ``engine="tiled"``: the B200 tiled engine (``picsar_b200.tiled``) in FP64
    or FP32 mixed precision.  The state lives in the engine's layout; the
    module arrays and the species' ``part_*`` arrays are PICSAR-layout FP64
    views filled when they are read, and a view that was handed out is
    written back into the engine before the next engine operation, so code
    that reads or edits module arrays between driver calls sees the
    reference's behaviour.  Gather, push, periodic wrap and deposition are
    one fused kernel, launched by ``field_gathering_plus_particle_pusher``;
    ``pxrdepose_currents_on_grid_jxjyjz`` then finds J deposited, and the
    boundary routines have nothing left to do (the engine writes periodic
    guards itself).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from . import psatd as _psatd
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
    """A 2-D or 3-D tensor in Fortran (column-major) layout."""
    if t.dim() == 2:
        return t.stride() == (1, t.shape[0])
    if t.dim() != 3:
        return False
    s0, s1, s2 = t.shape
    return t.stride() == (1, s0, s0 * s1)


def grid2d_zeros(nx, nz, g, dtype=torch.float64, device="cuda"):
    """A PICSAR x-z grid array (-g:n+g per axis) as a Fortran-ordered tensor."""
    return fortran_zeros((nx + 1 + 2 * g, nz + 1 + 2 * g), dtype, device)


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


_GRIDS = ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz", "rho", "dive")


def _grid_property(name):
    def get(self):
        if self._tiled is not None:
            return self._tiled.grid(name)
        return self._grids[name]

    def set_(self, value):
        if self._tiled is not None:
            self._tiled.set_grid(name, value)
        else:
            self._grids[name] = value
    return property(get, set_, doc=f"module array {name} (PICSAR layout, FP64)")


class PicsarModule:
    """Module variables and global drivers of PICSAR's step loop.

    engine: "plain" (PICSAR arrays, FP64) or "tiled" (the B200 tiled engine;
    precision "fp64" or "fp32" mixed, tuning ``tiled_config``, one pushed
    species)."""

    def __init__(self, nx, ny, nz, nguards=3, dx=1.0, dy=1.0, dz=1.0, xmin=0.0, ymin=0.0,
                 zmin=0.0, dtcoef=0.95, dt=None, nox=1, particle_pusher=0, clight=1.0,
                 mu0=1.0, eps0=1.0, device="cuda", engine="plain", precision="fp64",
                 tiled_config=None):
        if engine not in ("plain", "tiled"):
            raise ValueError("engine must be 'plain' or 'tiled'")
        if engine == "plain" and precision != "fp64":
            raise ValueError("the plain engine computes in FP64 only")
        self._tiled = None
        self._grids = {}
        self.engine, self.precision = engine, precision
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
        # Maxwell solver (modules.F90 fields): FDTD order per axis, nodal grid
        self.norderx = self.nordery = self.norderz = 2
        self.l_nodalgrid = False
        # spectral (PSATD) solver instead of Yee (fields: l_spectral,
        # l_staggered); norderx.. then give its stencil orders (0: infinite)
        self.l_spectral = False
        self.l_staggered = True
        self._psatd = None
        self.nxs = self.nys = self.nzs = 0
        self.particle_pusher = int(particle_pusher)
        self.l_lower_order_in_v = True
        self.currdepo = 0
        self.it = 0
        # particle sorting (shared_data, modules.F90:1491-1503): off by default
        # (control_file.F90:160-166); bin sizes in physical units, as after
        # the scaling by dx at start-up (submain.F90:601)
        # particle boundaries per side (shared_data pbound_*): 0 periodic,
        # 1 absorbing, 2 reflecting, 3 reinjecting
        self.pbound_x_min = self.pbound_x_max = 0
        self.pbound_y_min = self.pbound_y_max = 0
        self.pbound_z_min = self.pbound_z_max = 0
        self._bc_scratch = None
        self.sorting_activated = 0
        self.sorting_dx, self.sorting_dy, self.sorting_dz = self.dx, self.dy, self.dz
        self.sorting_shiftx = self.sorting_shifty = self.sorting_shiftz = 0.0
        self._sort_scratch = None
        self.species = []
        self._err = torch.zeros(1, dtype=torch.int32, device=self.device)
        g = self.nxguards
        if engine == "tiled":
            self._tiled = _TiledState(self, precision, tiled_config)
        else:
            for name in _GRIDS:
                self._grids[name] = grid_zeros(self.nx, self.ny, self.nz, g, device=self.device)

    # -- particles ----------------------------------------------------------
    def add_species(self, name, charge, mass, x, y, z, ux, uy, uz, w, pid=None,
                    sorting_period=0, sorting_start=0):
        if self._tiled is not None:
            sp = self._tiled.add_species(name, charge, mass, x, y, z, ux, uy, uz, w, pid)
            sp.sorting_period, sp.sorting_start = int(sorting_period), int(sorting_start)
            self.species.append(sp)
            return sp
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
        sp.sorting_period, sp.sorting_start = int(sorting_period), int(sorting_start)
        self.species.append(sp)
        return sp

    # -- drivers (module-level routines) -----------------------------------
    def field_gathering_plus_particle_pusher(self):
        """particle_pusher_manager_3d.F90:50-112 with one tile spanning the
        domain: zero the particle fields, fused gather + push.  Tiled engine:
        the fused gather + push + periodic wrap + Esirkepov deposition."""
        if self._tiled is not None:
            self._tiled.particle_step()
            return
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

    def _particle_bcs_general(self, sp, pb):
        n = sp.np
        need = _lib.query("pxrb_particle_bcs_scratch", n)
        if self._bc_scratch is None or self._bc_scratch.numel() < need:
            self._bc_scratch = torch.empty(need, dtype=torch.uint8, device=self.device)
        nout = torch.empty(1, dtype=torch.int64, device=self.device)
        pbh = np.ascontiguousarray(pb, dtype=np.int64)
        # one tile spanning the domain: particle region [min - d/2, max)
        # (tiling.F90:154-185), the bounds of the reinjection clamps
        tlo = np.array([self.xmin - self.dx / 2, self.ymin - self.dy / 2,
                        self.zmin - self.dz / 2])
        thi = np.array([self.xmax, self.ymax, self.zmax])
        _lib.call("pxrb_particle_bcs", n, _ptr(sp.part_x), _ptr(sp.part_y), _ptr(sp.part_z),
                  _ptr(sp.part_ux), _ptr(sp.part_uy), _ptr(sp.part_uz), _ptr(sp.part_gaminv),
                  _ptr(sp.pid_w), _ptr(sp.pid_id), self.xmin, self.ymin, self.zmin, self.xmax,
                  self.ymax, self.zmax, self.dx, self.dy, self.dz, pbh.ctypes.data,
                  tlo.ctypes.data, thi.ctypes.data, self._bc_scratch.data_ptr(),
                  self._bc_scratch.numel(), nout.data_ptr(), _stream())
        m = int(nout.item())
        if m != n:
            for c in ("part_x", "part_y", "part_z", "part_ux", "part_uy", "part_uz",
                      "part_gaminv", "part_ex", "part_ey", "part_ez", "part_bx", "part_by",
                      "part_bz", "pid_w", "pid_id"):
                setattr(sp, c, getattr(sp, c)[:m])

    def _pbounds(self):
        return (self.pbound_x_min, self.pbound_x_max, self.pbound_y_min, self.pbound_y_max,
                self.pbound_z_min, self.pbound_z_max)

    def particle_bcs(self):
        """Particle boundaries of every species (particle_boundaries.F90:
        1098-1300): the periodic wrap, or per side absorbing (removed),
        reflecting or reinjecting particles.  Tiled engine: periodic only,
        done by the fused particle kernel."""
        pb = self._pbounds()
        if self._tiled is not None:
            if any(pb):
                raise PicsarB200Error("the tiled engine wraps particles periodically only; "
                                      "use engine='plain' for other particle boundaries")
            return
        if any(pb):
            for sp in self.species:
                if sp.np:
                    self._particle_bcs_general(sp, pb)
            return
        for sp in self.species:
            if sp.np == 0:
                continue
            _lib.call("pxrb_particle_bcs_periodic", sp.np, _ptr(sp.part_x), _ptr(sp.part_y),
                      _ptr(sp.part_z), self.xmin, self.ymin, self.zmin, self.xmax, self.ymax,
                      self.zmax, _stream())

    def pxr_particle_sorting(self):
        """sorting.F90:67-215: when sorting_activated, every species whose
        sorting_period divides `it` (from sorting_start on) is sorted by
        cell bin (bins sorting_dx x sorting_dy x sorting_dz from the domain
        start plus the shifts; one tile spanning the domain).  Tiled engine:
        the engine's own counting sort by cell tile and bank order."""
        if self.sorting_activated <= 0:
            return
        for sp in self.species:
            if not (self.it >= sp.sorting_start and sp.sorting_period > 0
                    and self.it % sp.sorting_period == 0) or sp.np == 0:
                continue
            if self._tiled is not None:
                self._tiled.sort()
                continue
            # one tile per axis takes both the first- and the last-tile branch of
            # the reference's tile split (tiling.F90:154-185): its particle
            # region, where the bins start, is [min - d/2, max)
            lo = (self.xmin - self.dx / 2 + self.sorting_shiftx,
                  self.ymin - self.dy / 2 + self.sorting_shifty,
                  self.zmin - self.dz / 2 + self.sorting_shiftz)
            hi = (self.xmax + self.sorting_dx, self.ymax + self.sorting_dy,
                  self.zmax + self.sorting_dz)
            pxr_particle_bin_sorting(sp.np, sp.part_x, sp.part_y, sp.part_z, sp.part_ux,
                                     sp.part_uy, sp.part_uz, sp.part_gaminv, sp.pid_w,
                                     *lo, *hi, self.sorting_dx, self.sorting_dy,
                                     self.sorting_dz, module=self)

    def pxrdepose_currents_on_grid_jxjyjz(self):
        """J = 0, then Esirkepov deposition of every species
        (current_deposition_manager_3d.F90:224-494, currdepo = 0).  Tiled
        engine: J was deposited by the fused particle kernel."""
        if self._tiled is not None:
            self._tiled.check_deposited()
            return
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
        if self._tiled is not None:
            return                  # the engine deposits J with periodic wrapping
        _summation_bcs(self.jx, self.jy, self.jz, self.nx, self.ny, self.nz, self.nxjguards)

    def charge_bcs(self):
        if self._tiled is not None:
            return
        _summation_bcs(self.rho, None, None, self.nx, self.ny, self.nz, self.nxjguards)

    def _norder(self):
        return (self.norderx, self.nordery, self.norderz) != (2, 2, 2)

    def _fd_coeffs(self):
        """xcoeffs, ycoeffs, zcoeffs of FD_weights (submain.F90:899-906)."""
        return [FD_weights(np.zeros(o // 2), o, self.l_nodalgrid)
                for o in (self.norderx, self.nordery, self.norderz)]

    def push_bfield(self):
        """B half step (maxwell_solver_manager.F90:44-85): order-2 Yee, or the
        arbitrary-order stencil when an norder is not 2."""
        if self._tiled is not None:
            if self._norder():
                raise PicsarB200Error("the tiled engine's Yee solver is order 2")
            self._tiled.push_b()
            return
        if self._norder():
            cx, cy, cz = self._fd_coeffs()
            pxrpush_em3d_bvec_norder(self.ex, self.ey, self.ez, self.bx, self.by, self.bz,
                                     0.5 * self.dt / self.dx * cx, 0.5 * self.dt / self.dy * cy,
                                     0.5 * self.dt / self.dz * cz, self.nx, self.ny, self.nz,
                                     self.norderx, self.nordery, self.norderz, self.nxguards,
                                     self.nyguards, self.nzguards, self.nxs, self.nys, self.nzs,
                                     self.l_nodalgrid)
            return
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
        if self._tiled is not None:
            if self._norder():
                raise PicsarB200Error("the tiled engine's Yee solver is order 2")
            self._tiled.push_e()
            return
        if self._norder():
            cx, cy, cz = self._fd_coeffs()
            c2 = self.clight ** 2
            pxrpush_em3d_evec_norder(self.ex, self.ey, self.ez, self.bx, self.by, self.bz,
                                     self.jx, self.jy, self.jz, c2 * self.mu0 * self.dt,
                                     c2 * self.dt / self.dx * cx, c2 * self.dt / self.dy * cy,
                                     c2 * self.dt / self.dz * cz, self.nx, self.ny, self.nz,
                                     self.norderx, self.nordery, self.norderz, self.nxguards,
                                     self.nyguards, self.nzguards, self.nxs, self.nys, self.nzs,
                                     self.l_nodalgrid)
            return
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
        if self._tiled is not None:
            return                  # guards written by the engine's Yee kernels
        _field_bc(self.ex, self.ey, self.ez, self.nx, self.ny, self.nz, self.nxguards)

    def bfield_bcs(self):
        if self._tiled is not None:
            return
        _field_bc(self.bx, self.by, self.bz, self.nx, self.ny, self.nz, self.nxguards)

    def pxrdepose_rho_on_grid(self):
        if self._tiled is not None:
            self._tiled.deposit_rho()
            return
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

    def push_psatd_ebfield(self):
        """The spectral field push (maxwell_solver_manager.F90:574-642, local
        FFT): E and B over the FFT region advanced by one analytical step
        from J, rho and rho_old (picsar_b200.psatd)."""
        if self._tiled is not None:
            raise PicsarB200Error("the spectral solver runs on the plain engine")
        key = (self.dx, self.dy, self.dz, self.dt, self.norderx, self.nordery, self.norderz,
               bool(self.l_staggered), self.clight, self.eps0, self.mu0)
        if self._psatd is None or self._psatd[0] != key:
            g = (self.nxguards, self.nyguards, self.nzguards)
            solver = _psatd.PsatdSolver((self.nx, self.ny, self.nz), g,
                                        (self.dx, self.dy, self.dz), self.dt,
                                        (self.norderx, self.nordery, self.norderz),
                                        bool(self.l_staggered), self.clight, self.eps0,
                                        self.mu0, device=self.device)
            self._psatd = (key, solver)
        if "rhoold" not in self._grids:
            self._grids["rhoold"] = torch.zeros_like(self.rho)
        self._psatd[1].push(self.ex, self.ey, self.ez, self.bx, self.by, self.bz, self.jx,
                            self.jy, self.jz, self.rho, self._grids["rhoold"],
                            stream=_stream())

    @property
    def rhoold(self):
        """rho of the previous step (spectral solver)."""
        if "rhoold" not in self._grids:
            self._grids["rhoold"] = torch.zeros_like(self.rho)
        return self._grids["rhoold"]

    def _step_spectral(self, nst, diags):
        """PIC loop of src/submain.F90:101-150 with l_spectral: rho and
        rho_old start at zero; per step rho_old = rho and rho is deposited
        before the sort and the current deposition, then the PSATD push."""
        self.rho.zero_()
        self.rhoold.zero_()
        for _ in range(nst):
            self.field_gathering_plus_particle_pusher()
            self.particle_bcs()
            self.rhoold.copy_(self.rho)
            self.pxrdepose_rho_on_grid()
            self.charge_bcs()
            self.pxr_particle_sorting()
            self.pxrdepose_currents_on_grid_jxjyjz()
            self.current_bcs()
            self.push_psatd_ebfield()
            self.efield_bcs()
            self.bfield_bcs()
            if diags:
                self.calc_diags()
            self.it += 1

    def step(self, nst=1, diags=False):
        """PIC loop of src/submain.F90:104-195 (Yee solver, or the spectral
        solver when l_spectral, l_plasma).  Tiled engine: one fused particle
        kernel and three Yee launches per step, with the engine's own sort and
        re-layout schedule."""
        if self.l_spectral:
            if self._tiled is not None:
                raise PicsarB200Error("the spectral solver runs on the plain engine")
            self._step_spectral(nst, diags)
            return
        if self._tiled is not None:
            for _ in range(nst):
                self._tiled.step()
                if self.sorting_activated > 0:
                    self.pxr_particle_sorting()
                if diags:
                    self.calc_diags()
                self.it += 1
            return
        for _ in range(nst):
            self.field_gathering_plus_particle_pusher()
            self.particle_bcs()
            self.pxr_particle_sorting()
            self.pxrdepose_currents_on_grid_jxjyjz()
            self.current_bcs()
            self.push_bfield(); self.bfield_bcs()
            self.push_efield(); self.efield_bcs()
            self.push_bfield(); self.bfield_bcs()
            if diags:
                self.calc_diags()
            self.it += 1

    def check_errors(self):
        if self._tiled is not None:
            self._tiled.check_errors()
        if int(self._err.item()) != 0:
            raise PicsarB200Error("a particle moved more than one cell in one step")

    def diagnostics(self, gauss=True, to_host=True):
        """FP64 energies (kinetic, E, B) and the Gauss-law residual of the
        current state (diags.F90:847-1358); tiled engine only.  to_host=False
        leaves the 9 sums on the device (see TiledSim.diagnostics)."""
        if self._tiled is None:
            raise PicsarB200Error("diagnostics() reads the tiled engine's FP64 sums")
        self._tiled.flush()
        return self._tiled.sim.diagnostics(gauss=gauss, to_host=to_host)


for _name in _GRIDS:
    setattr(PicsarModule, _name, _grid_property(_name))
del _name


class _TiledSpecies:
    """A species of a tiled-engine PicsarModule: ``part_x`` ... ``part_gaminv``,
    ``pid_w`` (weight) and ``pid_id`` read as PICSAR FP64 arrays in the
    order the particles were added (the engine sorts internally and tracks
    ids).  Arrays that were read are written back into the engine before its
    next operation, so they may be edited in place; the engine recomputes
    gamma from u, so edits of ``part_gaminv`` alone have no effect."""

    _COLS = {"part_x": "x", "part_y": "y", "part_z": "z", "part_ux": "ux", "part_uy": "uy",
             "part_uz": "uz", "part_gaminv": "gaminv", "pid_w": "w", "pid_id": "id"}

    def __init__(self, state, name, charge, mass):
        self._state = state
        self.name, self.charge, self.mass = name, float(charge), float(mass)
        self.ldodepos = True
        self.sorting_period = self.sorting_start = 0

    @property
    def np(self):
        return self._state.sim.np

    def __getattr__(self, attr):
        if attr in _TiledSpecies._COLS:
            return self._state.particle_views()[_TiledSpecies._COLS[attr]]
        if attr in ("part_ex", "part_ey", "part_ez", "part_bx", "part_by", "part_bz"):
            raise AttributeError(
                f"{attr}: the tiled engine gathers E and B inside its fused particle kernel "
                "and keeps no per-particle field arrays (use engine='plain')")
        raise AttributeError(attr)


class _TiledState:
    """The tiled engine behind a PicsarModule: the simulation in the engine's
    layout, plus PICSAR-layout views of the module arrays and particles.

    A view is valid while the engine has not changed what it shows; reading
    a module array exports it if needed.  Views handed out (read or set)
    since the last engine operation are imported back before the next one."""

    _WHICH = {"ex": 0, "ey": 1, "ez": 2, "bx": 3, "by": 4, "bz": 5, "jx": 6, "jy": 7, "jz": 8}

    def __init__(self, m, precision, config):
        from .tiled import TiledConfig, TiledSim
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        if not (m.nxguards == m.nyguards == m.nzguards):
            raise ValueError("the tiled engine takes equal guard counts on all axes")
        self.m = m
        cfg = config or TiledConfig(tile=(8, 8, 8))
        self.sim = TiledSim((m.nx, m.ny, m.nz), order=m.nox, pusher=m.particle_pusher,
                            precision=precision, d=(m.dx, m.dy, m.dz),
                            xmin=(m.xmin, m.ymin, m.zmin), dt=m.dt, clight=m.clight,
                            mu0=m.mu0, eps0=m.eps0, config=cfg, track_ids=True,
                            device=m.device)
        self.ng = m.nxguards
        self.views, self.valid, self.out = {}, set(), set()
        self.pviews, self.pvalid, self.pout = None, False, False
        self.species = None
        self.deposited = False

    # -- module arrays --------------------------------------------------------
    def _view(self, name):
        v = self.views.get(name)
        if v is None:
            m = self.m
            v = grid_zeros(m.nx, m.ny, m.nz, self.ng, device=m.device)
            self.views[name] = v
        return v

    def grid(self, name):
        v = self._view(name)
        if name not in self.valid:
            if name in self._WHICH:
                _lib.call("pxrb_tiled_field_export", self.sim._jp(), self._WHICH[name],
                          v.data_ptr(), self.ng, _stream())
            elif name == "rho":
                self._export_rho(v)
            self.valid.add(name)
        self.out.add(name)
        return v

    def set_grid(self, name, value):
        v = self._view(name)
        if value is not v:
            v.copy_(torch.as_tensor(value).to(v.device, torch.float64))
        self.valid.add(name)
        self.out.add(name)

    def _export_rho(self, v):
        m, g = self.m, self.ng
        idx = lambda n: torch.remainder(torch.arange(-g, n + g + 1, device=m.device), n)
        r = self.sim.rho.view(m.nz, m.ny, m.nx)
        v.copy_(r[idx(m.nz)][:, idx(m.ny)][:, :, idx(m.nx)].permute(2, 1, 0))

    # -- particles ------------------------------------------------------------
    def add_species(self, name, charge, mass, x, y, z, ux, uy, uz, w, pid):
        if self.species is not None:
            raise NotImplementedError("the tiled engine pushes one species per module; use "
                                      "engine='plain' for several")
        sim = self.sim
        sim.q, sim.m = float(charge), float(mass)
        sim._fill_job()
        self.flush()
        sim.load_particles(x, y, z, ux, uy, uz, w, ids=pid)
        self.species = _TiledSpecies(self, name, charge, mass)
        self.pvalid = False
        return self.species

    def particle_views(self):
        if not self.pvalid:
            p = self.sim.particles()
            p["id"] = p["id"].to(torch.float64)
            self.pviews = p
            self.pvalid = True
        self.pout = True
        return self.pviews

    # -- engine operations ----------------------------------------------------
    def flush(self):
        """Write handed-out views back and follow changed module variables."""
        m, sim = self.m, self.sim
        if m.nox != sim.order:
            raise PicsarB200Error("nox changed after the tiled engine was built; build a new "
                                  "PicsarModule for another shape order")
        if m.particle_pusher != sim.pusher or m.dt != sim.dt:
            sim._pull_job()
            sim.pusher, sim.dt = int(m.particle_pusher), float(m.dt)
            sim.job.pusher, sim.job.dt = sim.pusher, sim.dt
            sim._push_job()
        for name in sorted(self.out):
            if name in self._WHICH:
                _lib.call("pxrb_tiled_field_import", sim._jp(), self._WHICH[name],
                          self.views[name].data_ptr(), self.ng, _stream())
        self.out.clear()
        if self.pout and self.pviews is not None:
            p = self.pviews
            sim.load_particles(p["x"], p["y"], p["z"], p["ux"], p["uy"], p["uz"], p["w"],
                               ids=p["id"].to(torch.int32),
                               ids_dense=getattr(sim, "_ids_dense", False))
            self.pvalid = False
        self.pout = False

    def particle_step(self):
        self.flush()
        sim = self.sim
        if getattr(sim, "_j_dirty", False):
            for t in sim.J:
                t.zero_()
            sim._j_dirty = False
        sim.particle_step()
        sim.it += 1
        sim.housekeeping()
        self.deposited = True
        self.valid -= {"jx", "jy", "jz", "rho"}
        self.pvalid = False

    def check_deposited(self):
        if not self.deposited:
            raise PicsarB200Error("tiled engine: the current is deposited by the fused "
                                  "particle kernel; call field_gathering_plus_particle_pusher "
                                  "first")

    def push_b(self):
        self.flush()
        self.sim.push_b(0.5)
        self.valid -= {"bx", "by", "bz"}

    def push_e(self):
        self.flush()
        self.sim.push_e(zero_j=False)
        self.sim._j_dirty = True          # the next particle kernel starts from J = 0
        self.deposited = False
        self.valid -= {"ex", "ey", "ez"}

    def step(self):
        self.flush()
        self.sim.step(1, keep_j=True)
        self.deposited = False
        self.valid.clear()
        self.pvalid = False

    def sort(self):
        self.flush()
        self.sim.sort()
        self.pvalid = False

    def deposit_rho(self):
        self.flush()
        self.sim.diagnostics(gauss=True, to_host=False)
        self.valid.discard("rho")

    def check_errors(self):
        if self.sim.error_flag():
            raise PicsarB200Error("a particle moved more than one cell in one step")


def pxr_particle_bin_sorting(np2, xp, yp, zp, ux, uy, uz, gam, pid, xmin2, ymin2, zmin2,
                             xmax2, ymax2, zmax2, dxf, dyf, dzf, wpid=1, module=None):
    """sorting.F90:247: stable sort of the particle arrays by cell bin, in
    place.  pid: the weight column (1-D), the only pid column the reference
    carries along, or None.  Scratch comes from torch (kept on ``module``
    when given)."""
    n = int(np2)
    if n == 0:
        return
    need = _lib.query("pxrb_particle_bin_sorting_scratch", n)
    scr = getattr(module, "_sort_scratch", None) if module is not None else None
    if scr is None or scr.numel() < need:
        scr = torch.empty(need, dtype=torch.uint8, device=xp.device)
        if module is not None:
            module._sort_scratch = scr
    _lib.call("pxrb_particle_bin_sorting", n,
              *[_ptr(a) for a in (xp, yp, zp, ux, uy, uz, gam)],
              None if pid is None else _ptr(pid, "pid"), float(xmin2), float(ymin2),
              float(zmin2), float(xmax2), float(ymax2), float(zmax2), float(dxf), float(dyf),
              float(dzf), scr.data_ptr(), scr.numel(), _stream())


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


def _host_f64(a, n, name):
    v = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
    if v.size < n:
        raise ValueError(f"{name}: needs {n} weights")
    return v


def pxrpush_em3d_evec_norder(ex, ey, ez, bx, by, bz, jx, jy, jz, mudt, dtsdx, dtsdy, dtsdz, nx,
                             ny, nz, norderx, nordery, norderz, nxguard, nyguard, nzguard, nxs,
                             nys, nzs, l_nodalgrid):
    """yee.F90:46-123 (dtsdx ... host arrays of norder/2 weights)."""
    w = [_host_f64(c, o // 2, nm) for c, o, nm in
         ((dtsdx, norderx, "dtsdx"), (dtsdy, nordery, "dtsdy"), (dtsdz, norderz, "dtsdz"))]
    _lib.call("pxrb_push_em3d_evec_norder",
              *[_ptr(a, n, grid=True) for a, n in zip((ex, ey, ez, bx, by, bz, jx, jy, jz),
                                                       ("ex", "ey", "ez", "bx", "by", "bz",
                                                        "jx", "jy", "jz"))],
              float(mudt), *[c.ctypes.data for c in w], int(nx), int(ny), int(nz),
              int(norderx), int(nordery), int(norderz), int(nxguard), int(nyguard),
              int(nzguard), int(nxs), int(nys), int(nzs), int(bool(l_nodalgrid)), _stream())


def pxrpush_em3d_bvec_norder(ex, ey, ez, bx, by, bz, dtsdx, dtsdy, dtsdz, nx, ny, nz, norderx,
                             nordery, norderz, nxguard, nyguard, nzguard, nxs, nys, nzs,
                             l_nodalgrid):
    """yee.F90:752-821 (dtsdx ... host arrays of norder/2 weights)."""
    w = [_host_f64(c, o // 2, nm) for c, o, nm in
         ((dtsdx, norderx, "dtsdx"), (dtsdy, nordery, "dtsdy"), (dtsdz, norderz, "dtsdz"))]
    _lib.call("pxrb_push_em3d_bvec_norder",
              *[_ptr(a, n, grid=True) for a, n in zip((ex, ey, ez, bx, by, bz),
                                                       ("ex", "ey", "ez", "bx", "by", "bz"))],
              *[c.ctypes.data for c in w], int(nx), int(ny), int(nz), int(norderx),
              int(nordery), int(norderz), int(nxguard), int(nyguard), int(nzguard), int(nxs),
              int(nys), int(nzs), int(bool(l_nodalgrid)), _stream())


def FD_weights(coeffs, norder, l_nodal):
    """submain.F90:927: fills coeffs (numpy float64, norder/2) in place and
    returns it."""
    c = np.asarray(coeffs)
    if c.dtype != np.float64 or not c.flags.c_contiguous or c.size < norder // 2:
        raise ValueError("coeffs: contiguous float64 array of norder/2 values")
    _lib.call("pxrb_fd_weights", c.ctypes.data, int(norder), int(bool(l_nodal)))
    return c


# ---------------------------------------------------------------------------
# 2D (x-z) routines (Forthon names and argument order)
# ---------------------------------------------------------------------------
def geteb2dxz_energy_conserving(np_, xp, yp, zp, ex, ey, ez, bx, by, bz, xmin, ymin, zmin, dx,
                                dy, dz, nx, ny, nz, nxguard, nyguard, nzguard, nox, noy, noz,
                                exg, eyg, ezg, bxg, byg, bzg, l4symtry, l_lower_order_in_v,
                                lvect, field_gathe_algo, l_nodal=False):
    """field_gathering_manager_2d.F90:61 (grids: 2-D x-z Fortran tensors;
    l_nodal = module l_nodalgrid)."""
    parts = [_ptr(a) for a in (xp, zp, ex, ey, ez, bx, by, bz)]
    grids = [_ptr(a, grid=True) for a in (exg, eyg, ezg, bxg, byg, bzg)]
    _lib.call("pxrb_geteb2dxz_energy_conserving", int(np_), parts[0],
              None if yp is None else _ptr(yp), parts[1], *parts[2:], float(xmin),
              float(ymin), float(zmin), float(dx), float(dy), float(dz), int(nx), int(ny),
              int(nz), int(nxguard), int(nyguard), int(nzguard), int(nox), int(noy), int(noz),
              *grids, int(bool(l4symtry)), int(bool(l_lower_order_in_v)), int(lvect),
              int(field_gathe_algo), int(bool(l_nodal)), _stream())


def depose_jxjyjz_2d(jx, jy, jz, np_, xp, yp, zp, uxp, uyp, uzp, gaminv, w, q, xmin, zmin, dt,
                     dx, dz, nx, nz, nxguard, nzguard, nox, noz, lvect):
    """current_deposition_manager_2d.F90:42 (2-D Esirkepov, accumulating)."""
    _lib.call("pxrb_depose_jxjyjz_2d", *[_ptr(a, grid=True) for a in (jx, jy, jz)], int(np_),
              _ptr(xp), None if yp is None else _ptr(yp), _ptr(zp),
              *[_ptr(a) for a in (uxp, uyp, uzp, gaminv, w)], float(q), float(xmin),
              float(zmin), float(dt), float(dx), float(dz), int(nx), int(nz), int(nxguard),
              int(nzguard), int(nox), int(noz), int(lvect), _stream())


def _b2(v):
    a = np.ascontiguousarray(np.asarray(v, dtype=np.int64).reshape(2))
    return a, a.ctypes.data


def _yee2d(name, bounds, arrays, scalars):
    keep, args = [], []
    for v in bounds:
        a, p = _b2(v); keep.append(a); args.append(p)
    for arr, lo, hi in arrays:
        a1, p1 = _b2(lo); a2, p2 = _b2(hi); keep += [a1, a2]
        if tuple(arr.shape) != tuple(int(h - l + 1) for l, h in zip(a1, a2)):
            raise ValueError(f"array shape {tuple(arr.shape)} does not match its bounds")
        args += [_ptr(arr, grid=True), p1, p2]
    _lib.call(name, *args, *[float(v) for v in scalars], _stream())


def pxrpush_em2d_evec(xlo, xhi, ylo, yhi, zlo, zhi, ex, exlo, exhi, ey, eylo, eyhi, ez, ezlo,
                      ezhi, bx, bxlo, bxhi, by, bylo, byhi, bz, bzlo, bzhi, jx, jxlo, jxhi, jy,
                      jylo, jyhi, jz, jzlo, jzhi, mudt, dtsdx, dtsdy, dtsdz):
    """yee.F90:216-310 (bounds of 2 values: x, z)."""
    _yee2d("pxrb_push_em2d_evec", (xlo, xhi, ylo, yhi, zlo, zhi),
           ((ex, exlo, exhi), (ey, eylo, eyhi), (ez, ezlo, ezhi), (bx, bxlo, bxhi),
            (by, bylo, byhi), (bz, bzlo, bzhi), (jx, jxlo, jxhi), (jy, jylo, jyhi),
            (jz, jzlo, jzhi)), (mudt, dtsdx, dtsdy, dtsdz))


def pxrpush_em2d_bvec(xlo, xhi, ylo, yhi, zlo, zhi, ex, exlo, exhi, ey, eylo, eyhi, ez, ezlo,
                      ezhi, bx, bxlo, bxhi, by, bylo, byhi, bz, bzlo, bzhi, dtsdx, dtsdy, dtsdz):
    """yee.F90:912-994 (bounds of 2 values: x, z)."""
    _yee2d("pxrb_push_em2d_bvec", (xlo, xhi, ylo, yhi, zlo, zhi),
           ((ex, exlo, exhi), (ey, eylo, eyhi), (ez, ezlo, ezhi), (bx, bxlo, bxhi),
            (by, bylo, byhi), (bz, bzlo, bzhi)), (dtsdx, dtsdy, dtsdz))


def pxr_pushxz(np_, xp, zp, uxp, uzp, gaminv, dt):
    """boris_2d.F90:42."""
    _lib.call("pxrb_pushxz", int(np_), *[_ptr(a) for a in (xp, zp, uxp, uzp, gaminv)],
              float(dt), _stream())


class PicsarModule2D:
    """Module variables and drivers of PICSAR's 2D (x-z) step loop on the
    plain FP64 path (submain.F90, c_dim = 2): grids are x-z Fortran arrays
    (-g:n+g) per axis; particles keep a y coordinate that is not pushed."""

    def __init__(self, nx, nz, nguards=3, dx=1.0, dz=1.0, xmin=0.0, zmin=0.0, dtcoef=0.95,
                 dt=None, nox=1, particle_pusher=0, clight=1.0, mu0=1.0, eps0=1.0,
                 device="cuda"):
        self.device = torch.device(device)
        self.nx, self.nz = int(nx), int(nz)
        self.ny = 0
        self.nxguards = self.nzguards = int(nguards)
        self.dx, self.dz = float(dx), float(dz)
        self.xmin, self.zmin = float(xmin), float(zmin)
        self.xmax, self.zmax = self.xmin + self.nx * self.dx, self.zmin + self.nz * self.dz
        self.clight, self.mu0, self.eps0 = float(clight), float(mu0), float(eps0)
        if dt is None:
            # submain.F90:587
            dt = dtcoef / (self.clight * math.sqrt(1.0 / self.dx ** 2 + 1.0 / self.dz ** 2))
        self.dt = float(dt)
        self.nox = self.noz = int(nox)
        self.particle_pusher = int(particle_pusher)
        self.l_nodalgrid = False
        self.it = 0
        g = self.nxguards
        for name in ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz"):
            setattr(self, name, grid2d_zeros(self.nx, self.nz, g, device=self.device))
        self.species = []

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

    def field_gathering_plus_particle_pusher(self):
        """particle_pusher_manager_2d.F90:57-278: zero the particle fields,
        gather (l_lower_order_in_v = .TRUE.), push u (Vay or Boris), push x, z."""
        for sp in self.species:
            if sp.np == 0:
                continue
            for c in ("ex", "ey", "ez", "bx", "by", "bz"):
                getattr(sp, "part_" + c).zero_()
            geteb2dxz_energy_conserving(
                sp.np, sp.part_x, sp.part_y, sp.part_z, sp.part_ex, sp.part_ey, sp.part_ez,
                sp.part_bx, sp.part_by, sp.part_bz, self.xmin, 0.0, self.zmin, self.dx, 1.0,
                self.dz, self.nx, 0, self.nz, self.nxguards, 0, self.nzguards, self.nox,
                self.nox, self.noz, self.ex, self.ey, self.ez, self.bx, self.by, self.bz, False,
                True, 256, 0, l_nodal=self.l_nodalgrid)
            fields = (sp.part_ex, sp.part_ey, sp.part_ez, sp.part_bx, sp.part_by, sp.part_bz)
            if self.particle_pusher == 1:
                pxr_ebcancelpush3d(sp.np, sp.part_ux, sp.part_uy, sp.part_uz, sp.part_gaminv,
                                   *fields, sp.charge, sp.mass, self.dt, 0, clight=self.clight)
            else:
                pxr_boris_push_u_3d(sp.np, sp.part_ux, sp.part_uy, sp.part_uz, sp.part_gaminv,
                                    *fields, sp.charge, sp.mass, self.dt, clight=self.clight)
            pxr_pushxz(sp.np, sp.part_x, sp.part_z, sp.part_ux, sp.part_uz, sp.part_gaminv,
                       self.dt)

    def particle_bcs(self):
        """Periodic wrap in x and z (particle_boundaries.F90, 2D branch)."""
        for sp in self.species:
            if sp.np:
                _lib.call("pxrb_particle_bcs_periodic", sp.np, _ptr(sp.part_x),
                          _ptr(sp.part_y), _ptr(sp.part_z), self.xmin, -math.inf, self.zmin,
                          self.xmax, math.inf, self.zmax, _stream())

    def pxrdepose_currents_on_grid_jxjyjz(self):
        """J = 0, then the 2-D Esirkepov deposition of every species
        (current_deposition_manager_2d.F90:334)."""
        self.jx.zero_(); self.jy.zero_(); self.jz.zero_()
        for sp in self.species:
            if sp.np == 0 or not sp.ldodepos:
                continue
            depose_jxjyjz_2d(self.jx, self.jy, self.jz, sp.np, sp.part_x, sp.part_y, sp.part_z,
                             sp.part_ux, sp.part_uy, sp.part_uz, sp.part_gaminv, sp.pid_w,
                             sp.charge, self.xmin, self.zmin, self.dt, self.dx, self.dz, self.nx,
                             self.nz, self.nxguards, self.nzguards, self.nox, self.noz, 256)

    def _bc(self, arrs, fold):
        name = "pxrb_summation_bcs_periodic" if fold else "pxrb_field_bc_periodic"
        _lib.call(name, *[_ptr(a, grid=True) for a in arrs], self.nx, 0, self.nz, self.nxguards,
                  0, self.nzguards, _stream())

    def current_bcs(self):
        self._bc((self.jx, self.jy, self.jz), True)

    def efield_bcs(self):
        self._bc((self.ex, self.ey, self.ez), False)

    def bfield_bcs(self):
        self._bc((self.bx, self.by, self.bz), False)

    def _bounds(self):
        g = self.nxguards
        lo, hi = (-g, -g), (self.nx + g, self.nz + g)
        rng = ((0, 0), (self.nx, self.nz))
        return lo, hi, rng

    def push_bfield(self):
        """B half step (maxwell_solver_manager.F90:453-500, order 2)."""
        lo, hi, (a, b) = self._bounds()
        pxrpush_em2d_bvec(a, b, a, b, a, b, self.ex, lo, hi, self.ey, lo, hi, self.ez, lo, hi,
                          self.bx, lo, hi, self.by, lo, hi, self.bz, lo, hi,
                          0.5 * self.dt / self.dx, 0.0, 0.5 * self.dt / self.dz)

    def push_efield(self):
        """E full step (maxwell_solver_manager.F90:510-560, order 2)."""
        lo, hi, (a, b) = self._bounds()
        c2 = self.clight ** 2
        pxrpush_em2d_evec(a, b, a, b, a, b, self.ex, lo, hi, self.ey, lo, hi, self.ez, lo, hi,
                          self.bx, lo, hi, self.by, lo, hi, self.bz, lo, hi, self.jx, lo, hi,
                          self.jy, lo, hi, self.jz, lo, hi, c2 * self.mu0 * self.dt,
                          c2 * self.dt / self.dx, 0.0, c2 * self.dt / self.dz)

    def step(self, nst=1):
        """2D PIC loop (submain.F90, c_dim = 2, Yee solver)."""
        for _ in range(nst):
            self.field_gathering_plus_particle_pusher()
            self.particle_bcs()
            self.pxrdepose_currents_on_grid_jxjyjz()
            self.current_bcs()
            self.push_bfield(); self.bfield_bcs()
            self.push_efield(); self.efield_bcs()
            self.push_bfield(); self.bfield_bcs()
            self.it += 1


def _check_bounds(arr, lo, hi):
    ext = tuple(int(h - l + 1) for l, h in zip(lo, hi))
    if tuple(arr.shape) != ext:
        raise ValueError(f"array shape {tuple(arr.shape)} does not match bounds {ext}")
