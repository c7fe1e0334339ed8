"""PICSAR input decks (``.pixr``) and field dumps (``.pxr``) on the B200 engines.

``read_input_file(path)`` restates the reference's deck reader
(src/initialization/control_file.F90:77-1311) with the rules that decide
what a deck means:

  * a line that holds ``section::<name>`` anywhere opens that section (the
    header line itself is not checked for ``#``); inside a section every
    line that contains ``#`` anywhere is skipped;
  * keys are matched as substrings, in the reference's order, the first
    match wins;
  * integer values are read with the ``(i10)`` edit: only the 10 characters
    after the ``=`` count, blanks ignored; reals, logicals and names are
    read list-directed (first value, ``d`` exponents accepted);
  * the readers of the cpusplit, plasma, solver, sorting, timestat, main and
    output sections keep their end flag between calls (a saved initial
    value), so a second section of those kinds is not read;
  * the temporal section has no end marker: it reads to the end of the file,
    so keys of later sections that contain its keys (``output_frequency``
    contains ``frequency``) set its values.

``Deck.derived()`` applies what the reference's initialisation does after
reading (src/parallelization/mpi/mpi_routines.F90:1514-1528,
src/submain.F90:549-610): ``nx`` in a deck counts grid points, cells are
``nx - 1`` and ``dx = (xmax - xmin) / cells`` (a deck's ``dx`` is
overwritten); ``dt`` from ``dtcoef``; ``nsteps`` from ``t_max`` in units of
the plasma period ``1/w0``; sorting lengths in cells.

``load_particles(deck)`` restates the reference's loader
(src/parallelization/tiling/tiling.F90:876-1003, ``pdistr`` 1 and 2, 3D and
2D).  Positions follow it exactly for ``pdistr = 1``; the random numbers
(gfortran's ``RANDOM_NUMBER``) come from a seeded NumPy generator instead,
so thermal velocities and ``pdistr = 2`` positions have the reference's
distribution, not its values.

``run_deck(path)`` runs a deck the way the mini-app's main program does
(src/submain.F90:104-205): per iteration one PIC step, the charge
deposition (``calc_diags``) and ``output_routines``: field dumps in the
``.pxr`` format (src/ios/simple_io.F90:493-588) and the temporal
diagnostics (src/ios/simple_io.F90:236-455, src/diags/diags.F90:253-420,
847-1300), all under ``<out_dir>/`` (the reference writes ``./RESULTS/``).

Physical constants are the reference's SI values (src/modules/modules.F90:
57-81).  ``l_spectral`` decks run the PSATD push of ``picsar_b200.psatd``
(3D, plain engine, ``dt = min(dx, dy, dz) / c`` as submain.F90:578-586
sets it).  Not supported (a deck that asks raises ``DeckError``): the laser
antenna, the matrix form of the spectral solver (``g_spectral``) and
distributed FFTs, PML / absorbing boundaries, different shape orders per
axis, and (tiled engine) more than one species.
"""
from __future__ import annotations

import math
import os
import re
import struct
from dataclasses import dataclass, field

import numpy as np

EMASS = 9.10938291e-31
PMASS = 1.6726231000000001e-27
ECHARGE = 1.6021764620000001e-19
CLIGHT = 2.99792458e8
MU0 = 1.2566370614359173e-06
EPS0 = 8.854187817620389e-12
IMU0 = 795774.715459
PI = 3.14159265358979323
STRING_LENGTH = 264          # length of the reader's line buffer (constants: string_length)
HUGE = float(np.finfo(np.float64).max)


class DeckError(ValueError):
    """A deck the reference reader would reject, or one this runner cannot run."""


# ----------------------------------------------------------------- values
_REAL = re.compile(r"^([+-]?(?:\d+\.?\d*|\.\d+))(?:([eEdDqQ])([+-]?\d+)|([+-]\d+))?$")


def _token(s):
    """First list-directed value of s: up to a blank, comma or slash."""
    s = s.lstrip(" \t")
    if not s:
        raise DeckError("missing value")
    if s[0] in "'\"":
        end = s.find(s[0], 1)
        return s[1:end if end > 0 else len(s)]
    m = re.match(r"[^ \t,/]*", s)
    return m.group(0)


def read_i10(rest):
    """``READ(rest, '(i10)')``: the first 10 characters, blanks ignored."""
    f = rest[:10].replace(" ", "").replace("\t", "")
    if f == "":
        return 0
    if not re.fullmatch(r"[+-]?\d+", f):
        raise DeckError(f"bad integer field {rest[:10]!r}")
    return int(f)


def read_real(rest):
    """List-directed real."""
    t = _token(rest)
    m = _REAL.match(t)
    if not m:
        raise DeckError(f"bad real value {t!r}")
    mant, _, e1, e2 = m.groups()
    exp = e1 if e1 is not None else e2
    # correctly rounded conversion of the whole decimal string
    return float(mant + ("e" + exp if exp is not None else ""))


def read_int(rest):
    """List-directed integer."""
    t = _token(rest)
    if not re.fullmatch(r"[+-]?\d+", t):
        raise DeckError(f"bad integer value {t!r}")
    return int(t)


def read_logical(rest):
    """List-directed logical: optional '.', then T or F."""
    t = _token(rest)
    u = t[1:] if t.startswith(".") else t
    if u[:1].upper() == "T":
        return True
    if u[:1].upper() == "F":
        return False
    raise DeckError(f"bad logical value {t!r}")


def read_name(rest):
    """List-directed character value."""
    return _token(rest)


# ------------------------------------------------------------------ deck
@dataclass
class Species:
    """One ``section::species`` (defaults as read_species_section sets
    them); mass and charge in kg and C, velocities in m/s."""
    name: str = ""
    charge: float = -ECHARGE
    mass: float = EMASS
    nppcell: int = 0
    x_min: float = 0.0
    x_max: float = 0.0
    y_min: float = 0.0
    y_max: float = 0.0
    z_min: float = 0.0
    z_max: float = 0.0
    vdrift_x: float = 0.0
    vdrift_y: float = 0.0
    vdrift_z: float = 0.0
    vth_x: float = 0.0
    vth_y: float = 0.0
    vth_z: float = 0.0
    sorting_period: int = 0
    sorting_start: int = 0


@dataclass
class ParticleDump:
    """One ``section::particle_dump``: every diag_period iterations the
    particles of one species inside the (strict) position and momentum
    ranges are written (write_particles_to_file)."""
    ispecies: int = -1
    dump_x_min: float = 0.0
    dump_x_max: float = 0.0
    dump_y_min: float = 0.0
    dump_y_max: float = 0.0
    dump_z_min: float = 0.0
    dump_z_max: float = 0.0
    dump_ux_min: float = 1e7
    dump_ux_max: float = 1e9
    dump_uy_min: float = 1e7
    dump_uy_max: float = 1e9
    dump_uz_min: float = 1e7
    dump_uz_max: float = 1e9
    diag_period: int = -1


_TEMPORAL_NAMES = ("kinE", "exE", "eyE", "ezE", "bxE", "byE", "bzE", "divE-rho", "rho", "divE")
_OUTPUT_FIELDS = ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz", "rho", "dive", "divj",
                  "divb")


@dataclass
class Deck:
    """Every variable the reader sets, with the values default_init and the
    module declarations give them."""
    c_dim: int = 3
    ntilex: int = 1
    ntiley: int = 1
    ntilez: int = 1
    norderx: int = 2
    nordery: int = 2
    norderz: int = 2
    nx_pml: int = 0
    ny_pml: int = 0
    nz_pml: int = 0
    absorbing_bcs_x: bool = False
    absorbing_bcs_y: bool = False
    absorbing_bcs_z: bool = False
    l_nodalgrid: bool = False
    l_spectral: bool = False
    g_spectral: bool = False
    l_staggered: bool = True
    nox: int = 1
    noy: int = 1
    noz: int = 1
    nxguards: int = 2
    nyguards: int = 2
    nzguards: int = 2
    nxjguards: int = 2
    nyjguards: int = 2
    nzjguards: int = 2
    topology: int = 0
    mpicom_curr: int = 1
    currdepo: int = 0
    rhodepo: int = 0
    fieldgathe: int = 0
    partcom: int = 0
    particle_pusher: int = 0
    fg_p_pp_separated: int = 0
    lvec_curr_depo: int = 8
    lvec_charge_depo: int = 64
    lvec_fieldgathe: int = 256
    mpi_buf_size: int = 2000
    nprocx: int = 0
    nprocy: int = 0
    nprocz: int = 0
    sorting_activated: int = 0
    sorting_dx: float = 1.0
    sorting_dy: float = 1.0
    sorting_dz: float = 1.0
    sorting_shiftx: float = 0.0
    sorting_shifty: float = 0.0
    sorting_shiftz: float = 0.0
    sorting_verbose: bool = True
    timestat_activated: int = 0
    timestat_period: int = 0
    timestat_itstart: int = 0
    timestat_perit: int = 0
    nbuffertimestat: int = 1
    l_lower_order_in_v: bool = True
    dtcoef: float = 0.7
    tmax: float = 0.0
    nsteps: int = 0
    nlab: float = 1e23
    g0: float = 1.0
    l_plasma: bool = True
    pdistr: int = 1
    fftw_with_mpi: bool = False
    fftw_hybrid: bool = False
    fftw_mpi_transpose: bool = False
    p3dfft_flag: bool = False
    p3dfft_stride: bool = False
    # main section grid (nx etc. count grid points as read; 0: not given)
    nx_global_grid: int = 0
    ny_global_grid: int = 0
    nz_global_grid: int = 0
    dx: float = 0.0
    dy: float = 0.0
    dz: float = 0.0
    xmin: float = 0.0
    ymin: float = 0.0
    zmin: float = 0.0
    xmax: float = 0.0
    ymax: float = 0.0
    zmax: float = 0.0
    # output
    output_frequency: int = -1
    output_step_min: int = 0
    output_step_max: int = 0
    c_output: dict = field(default_factory=lambda: {k: 0 for k in _OUTPUT_FIELDS})
    temdiag_frequency: int = 0
    temdiag_format: int = 0
    temdiag_act_list: list = field(default_factory=lambda: [0] * 10)
    species: list = field(default_factory=list)
    particle_dumps: list = field(default_factory=list)
    antenna: bool = False
    sections: list = field(default_factory=list)   # section headers met, in order

    # ---------------------------------------------------------- derived
    def derived(self):
        """The quantities the reference's initialisation computes from the
        deck for one domain: a dict with cells per axis, dx, dy, dz, dt,
        nsteps, tmax, nc, w0_l and the sorting lengths in metres."""
        nxc = self.nx_global_grid - 1
        nyc = self.ny_global_grid - 1
        nzc = self.nz_global_grid - 1
        if self.c_dim == 2:
            nyc = 1
        if nxc < 1 or nzc < 1 or (self.c_dim == 3 and nyc < 1):
            raise DeckError(f"grid of {self.nx_global_grid} x {self.ny_global_grid} x "
                            f"{self.nz_global_grid} points")
        dx = (self.xmax - self.xmin) / nxc
        dz = (self.zmax - self.zmin) / nzc
        if self.c_dim == 2:
            dy = HUGE
            if self.l_spectral:
                dt = min(dx, dz) / CLIGHT
            else:
                dt = self.dtcoef / (CLIGHT * math.sqrt(1.0 / dx ** 2 + 1.0 / dz ** 2))
        else:
            dy = (self.ymax - self.ymin) / nyc
            if self.l_spectral:
                dt = min(dx, dy, dz) / CLIGHT
            else:
                dt = self.dtcoef / (CLIGHT * math.sqrt(1.0 / dx ** 2 + 1.0 / dy ** 2 +
                                                       1.0 / dz ** 2))
        nc = self.nlab * self.g0
        w0_l = ECHARGE * math.sqrt(nc / (self.g0 * EMASS * EPS0))
        if self.nsteps == 0:
            nsteps = int(np.rint(self.tmax / (w0_l * dt)))
            tmax = self.tmax
        else:
            nsteps = self.nsteps
            tmax = nsteps * w0_l * dt
        return {"n": (nxc, nyc, nzc), "dx": dx, "dy": dy, "dz": dz, "dt": dt,
                "nsteps": nsteps, "tmax": tmax, "nc": nc, "w0_l": w0_l,
                "sorting_d": (self.sorting_dx * dx, self.sorting_dy * dy,
                              self.sorting_dz * dz),
                "sorting_shift": (self.sorting_shiftx * dx, self.sorting_shifty * dy,
                                  self.sorting_shiftz * dz)}


# ---------------------------------------------------------------- reader
# (key, attribute, reader) per section, in the reference's order
_I, _R, _L, _N, _IL = read_i10, read_real, read_logical, read_name, read_int
_CPUSPLIT = [("nprocx", "nprocx", _I), ("nprocy", "nprocy", _I), ("nprocz", "nprocz", _I),
             ("topology", "topology", _I), ("mpicom_curr", "mpicom_curr", _I),
             ("partcom", "partcom", _I), ("fg_p_pp_separated", "fg_p_pp_separated", _I),
             ("particle_pusher", "particle_pusher", _I),
             ("lvec_curr_depo", "lvec_curr_depo", _I),
             ("lvec_charge_depo", "lvec_charge_depo", _I),
             ("lvec_fieldgathe", "lvec_fieldgathe", _I), ("mpi_buf_size", "mpi_buf_size", _I),
             ("c_dim", "c_dim", _I)]
_PLASMA = [("nlab", "nlab", _R), ("gamma0", "g0", _R), ("pdistr", "pdistr", _IL),
           ("particle_pusher", "particle_pusher", _I)]
_SOLVER = [("norderx", "norderx", _I), ("nordery", "nordery", _I), ("norderz", "norderz", _I),
           ("nox", "nox", _I), ("nx_pml", "nx_pml", _I), ("ny_pml", "ny_pml", _I),
           ("nz_pml", "nz_pml", _I), ("noy", "noy", _I), ("noz", "noz", _I),
           ("currdepo", "currdepo", _I), ("fieldgathe", "fieldgathe", _I),
           ("rhodepo", "rhodepo", _I), ("partcom", "partcom", _I),
           ("mpi_buf_size", None, None), ("l_spectral", "l_spectral", _L),
           ("absorbing_bcs_x", "absorbing_bcs_x", _L),
           ("absorbing_bcs_y", "absorbing_bcs_y", _L),
           ("absorbing_bcs_z", "absorbing_bcs_z", _L), ("g_spectral", "g_spectral", _L),
           ("l_staggered", "l_staggered", _L), ("fftw_with_mpi", "fftw_with_mpi", _L),
           ("fftw_mpi_tr", "fftw_mpi_transpose", _L), ("fftw_hybrid", "fftw_hybrid", _L),
           ("p3dfft_flag", "p3dfft_flag", _L), ("p3dfft_stride", "p3dfft_stride", _L),
           ("fg_p_pp_separated", "fg_p_pp_separated", _I)]
_SORTING = [("activation", "sorting_activated", _I), ("dx", "sorting_dx", _R),
            ("dy", "sorting_dy", _R), ("dz", "sorting_dz", _R),
            ("shiftx", "sorting_shiftx", _R), ("shifty", "sorting_shifty", _R),
            ("shiftz", "sorting_shiftz", _R), ("verbose", "sorting_verbose", _L)]
_TIMESTAT = [("activation", "timestat_activated", _I), ("period", "timestat_period", _I),
             ("it_start", "timestat_itstart", _I), ("per_it", "timestat_perit", _I),
             ("buffersize", "nbuffertimestat", _I)]
_MAIN = [("c_dim", "c_dim", _I), ("nx", "nx_global_grid", _I), ("ny", "ny_global_grid", _I),
         ("nz", "nz_global_grid", _I), ("ntilex", "ntilex", _I), ("ntiley", "ntiley", _I),
         ("ntilez", "ntilez", _I), ("dx", "dx", _R), ("dy", "dy", _R), ("dz", "dz", _R),
         ("xmin", "xmin", _R), ("ymin", "ymin", _R), ("zmin", "zmin", _R),
         ("xmax", "xmax", _R), ("ymax", "ymax", _R), ("zmax", "zmax", _R),
         ("t_max", "tmax", _R), ("nsteps", "nsteps", _IL), ("dtcoef", "dtcoef", _R),
         ("nguardsx", "nxguards", _I), ("nguardsy", "nyguards", _I),
         ("nguardsz", "nzguards", _I), ("njguardsx", "nxjguards", _I),
         ("njguardsy", "nyjguards", _I), ("njguardsz", "nzjguards", _I),
         ("l_plasma", "l_plasma", _L)]
_OUTPUT = ([("output_frequency", "output_frequency", _I),
            ("output_step_min", "output_step_min", _I),
            ("output_step_max", "output_step_max", _I)]
           + [(k, "c_output:" + k, _I) for k in _OUTPUT_FIELDS])
_TEMPORAL = ([("frequency", "temdiag_frequency", _I), ("format", "temdiag_format", _I)]
             + [(k, f"temdiag:{i}", _I) for i, k in enumerate(_TEMPORAL_NAMES)])
_SPECIES = [("name", "name", _N), ("mass", "mass", _R), ("charge", "charge", _R),
            ("nppcell", "nppcell", _I), ("x_min", "x_min", _R), ("x_max", "x_max", _R),
            ("y_min", "y_min", _R), ("y_max", "y_max", _R), ("z_min", "z_min", _R),
            ("z_max", "z_max", _R), ("vdrift_x", "vdrift_x", _R),
            ("vdrift_y", "vdrift_y", _R), ("vdrift_z", "vdrift_z", _R),
            ("vth_x", "vth_x", _R), ("vth_y", "vth_y", _R), ("vth_z", "vth_z", _R),
            ("sorting_period", "sorting_period", _IL),
            ("sorting_start", "sorting_start", _IL)]
_DUMP = [("dump_x_min", "dump_x_min", _R), ("dump_x_max", "dump_x_max", _R),
         ("species_name", None, _N), ("dump_y_min", "dump_y_min", _R),
         ("dump_y_max", "dump_y_max", _R), ("dump_z_min", "dump_z_min", _R),
         ("dump_z_max", "dump_z_max", _R), ("dump_ux_min", "dump_ux_min", _R),
         ("dump_ux_max", "dump_ux_max", _R), ("dump_uy_min", "dump_uy_min", _R),
         ("dump_uy_max", "dump_uy_max", _R), ("dump_uz_min", "dump_uz_min", _R),
         ("dump_uz_max", "dump_uz_max", _R), ("diag_period", "diag_period", _I)]
# sections whose reader keeps its end flag from one call to the next
_SAVED = {"cpusplit", "plasma", "solver", "sorting", "timestat", "main", "output"}
_KEYS = {"cpusplit": _CPUSPLIT, "plasma": _PLASMA, "solver": _SOLVER, "sorting": _SORTING,
         "timestat": _TIMESTAT, "main": _MAIN, "output": _OUTPUT, "temporal": _TEMPORAL}


class _Lines:
    def __init__(self, text):
        self.lines = [ln[:STRING_LENGTH] for ln in text.split("\n")]
        if self.lines and self.lines[-1] == "":
            self.lines.pop()
        self.i = 0

    def next(self):
        """The next line, or None at the end of the file."""
        if self.i >= len(self.lines):
            return None
        ln = self.lines[self.i]
        self.i += 1
        return ln


def _set(deck, target, attr, value):
    if attr.startswith("c_output:"):
        deck.c_output[attr.split(":", 1)[1]] = value
    elif attr.startswith("temdiag:"):
        deck.temdiag_act_list[int(attr.split(":", 1)[1])] = value
    else:
        setattr(target, attr, value)


def _value(line):
    """Text after the first '=' (the whole line when there is none, as the
    reference's INDEX returns 0 then)."""
    ix = line.find("=")
    return line[ix + 1:] if ix >= 0 else line


def _read_section(deck, src, name):
    """One section reader: lines until its end marker (or the end of the
    file); returns True when the end marker was met."""
    keys = _KEYS[name]
    end = f"end::{name}"
    while True:
        ln = src.next()
        if ln is None:
            return False
        if "#" in ln:
            continue
        for key, attr, reader in keys:
            if key in ln:
                if attr is not None:
                    _set(deck, deck, attr, reader(_value(ln)))
                break
        else:
            if name != "temporal" and end in ln:
                return True


def _read_species(deck, src):
    sp = Species()
    deck.species.append(sp)
    while True:
        ln = src.next()
        if ln is None:
            return
        if "#" in ln:
            continue
        for key, attr, reader in _SPECIES:
            if key in ln:
                v = reader(_value(ln))
                if attr == "mass":
                    v *= EMASS
                elif attr == "charge":
                    v *= ECHARGE
                elif attr.startswith("vdrift_") or attr.startswith("vth_"):
                    v *= CLIGHT
                setattr(sp, attr, v)
                break
        else:
            if "end::species" in ln:
                return


def _read_dump(deck, src):
    dp = ParticleDump(dump_x_min=deck.xmin, dump_x_max=deck.xmax, dump_y_min=deck.ymin,
                      dump_y_max=deck.ymax, dump_z_min=deck.zmin, dump_z_max=deck.zmax)
    deck.particle_dumps.append(dp)
    while True:
        ln = src.next()
        if ln is None:
            return
        if "#" in ln:
            continue
        for key, attr, reader in _DUMP:
            if key in ln:
                v = reader(_value(ln))
                if attr is None:            # species_name: first species whose name it holds
                    for i, sp in enumerate(deck.species):
                        if sp.name in v:
                            dp.ispecies = i
                            break
                else:
                    setattr(dp, attr, v)
                break
        else:
            if "end::particle_dump" in ln:
                return


def _skip_antenna(deck, src):
    deck.antenna = True
    while True:
        ln = src.next()
        if ln is None or "end::antenna" in ln:
            return


def read_input_text(text):
    """A Deck from the text of a ``.pixr`` file (see the module docstring)."""
    deck = Deck()
    src = _Lines(text)
    ended = set()
    while True:
        ln = src.next()
        if ln is None:
            break
        ix = ln.find("section::")
        if ix < 0:
            continue
        name = ln[ix:].rstrip().lstrip()[len("section::"):]
        deck.sections.append(name)
        if name in _KEYS:
            if name in _SAVED and name in ended:
                continue                     # its end flag is still set: nothing read
            if _read_section(deck, src, name):
                ended.add(name)
            if name == "temporal":
                break                        # read to the end of the file
        elif name == "species":
            _read_species(deck, src)
        elif name == "particle_dump":
            _read_dump(deck, src)
        elif name == "antenna":
            _skip_antenna(deck, src)
    return deck


def read_input_file(path):
    """A Deck from a ``.pixr`` file."""
    with open(path, "r", errors="replace") as f:
        return read_input_text(f.read())


# --------------------------------------------------------------- loading
def _nint(v):
    """Fortran NINT: nearest integer, halves away from zero."""
    return int(math.copysign(math.floor(abs(v) + 0.5), v))


def _box(lo, hi, dom_lo, dom_hi, d):
    """Cell range [a, b) of a species box in the domain (tiling.F90:880-885)."""
    return (_nint(max(lo - dom_lo, 0.0) / d), _nint(min(hi - dom_lo, dom_hi - dom_lo) / d))


def _velocities(sp, r):
    """The loader's thermal draw (tiling.F90:899-913) from uniforms r[:, 0:3]:
    returns ux, uy, uz, gaminv."""
    v = np.maximum(1e-10, r[:, 0])
    th = 2 * PI * r[:, 1]
    phi = 2 * PI * r[:, 2]
    a = np.sqrt(-2.0 * np.log(v))
    vx = sp.vdrift_x + sp.vth_x * a * np.cos(th) * np.cos(phi)
    vy = sp.vdrift_y + sp.vth_y * a * np.cos(th) * np.sin(phi)
    vz = sp.vdrift_z + sp.vth_z * a * np.sin(th)
    gaminv = np.sqrt(1.0 - (vx ** 2 + vy ** 2 + vz ** 2) * (1.0 / CLIGHT ** 2))
    return vx / gaminv, vy / gaminv, vz / gaminv, gaminv


def load_particles(deck, seed=0):
    """Per species a dict of FP64 arrays x, y, z, ux, uy, uz, gaminv, w in the
    reference loader's order (tiling.F90:876-1003; see the module
    docstring for the random numbers)."""
    der = deck.derived()
    dx, dy, dz, nc = der["dx"], der["dy"], der["dz"], der["nc"]
    g = np.random.default_rng(seed)
    out = []
    for sp in deck.species:
        npc = int(sp.nppcell)
        j0, j1 = _box(sp.x_min, sp.x_max, deck.xmin, deck.xmax, dx)
        l0, l1 = _box(sp.z_min, sp.z_max, deck.zmin, deck.zmax, dz)
        if deck.c_dim == 3:
            k0, k1 = _box(sp.y_min, sp.y_max, deck.ymin, deck.ymax, dy)
        else:
            k0, k1 = 0, 1
        nj, nk, nl = max(0, j1 - j0), max(0, k1 - k0), max(0, l1 - l0)
        n = nj * nk * nl * max(npc, 0)
        if n == 0:
            e = np.zeros(0)
            out.append({c: e.copy() for c in ("x", "y", "z", "ux", "uy", "uz", "gaminv", "w")})
            continue
        if deck.pdistr == 1:
            # loop order l, k, j, ipart (ipart fastest)
            L, K, J, P = np.meshgrid(np.arange(l0, l1), np.arange(k0, k1), np.arange(j0, j1),
                                     np.arange(1, npc + 1), indexing="ij")
            J, K, L, P = (a.ravel().astype(np.float64) for a in (J, K, L, P))
            if deck.c_dim == 3:
                x = deck.xmin + J * dx + dx / npc * (P - 0.5)
                y = deck.ymin + K * dy + dy / npc * (P - 0.5)
                z = deck.zmin + L * dz + dz / npc * (P - 0.5)
                w = np.full(n, nc * dx * dy * dz / npc)
            else:
                x = deck.xmin + J * dx + dx / npc * (P - 1)
                y = np.zeros(n)
                z = deck.zmin + L * dz + dz / npc * (P - 1)
                w = np.full(n, nc * dx * dz / npc)
            ux, uy, uz, gi = _velocities(sp, g.random((n, 3)))
        elif deck.pdistr == 2:
            if deck.c_dim != 3:
                raise DeckError("pdistr = 2 is a 3D loader in the reference")
            r = g.random((n, 6))
            x = deck.xmin + np.minimum(r[:, 0], 0.999) * (deck.xmax - deck.xmin)
            y = deck.ymin + np.minimum(r[:, 1], 0.999) * (deck.ymax - deck.ymin)
            z = deck.zmin + np.minimum(r[:, 2], 0.999) * (deck.zmax - deck.zmin)
            w = np.full(n, nc * dx * dy * dz / npc)
            ux, uy, uz, gi = _velocities(sp, r[:, 3:6])
        else:
            raise DeckError(f"pdistr = {deck.pdistr} is not a loader of the reference")
        out.append({"x": x, "y": y, "z": z, "ux": ux, "uy": uy, "uz": uz, "gaminv": gi, "w": w})
    return out


# ----------------------------------------------------------------- dumps
_PXR_HEADER = struct.Struct("<ddiddiddi")


def write_pxr(filename, arr, lo, hi, n_global):
    """A ``.pxr`` field dump (simple_io.F90:493-588, one domain): the header
    (xmin, xmax, nx as int32, then y and z) and the grid's nodes 0..n-1 per
    axis as FP64, x fastest.  arr: array of those nodes, shape (nx, ny, nz)."""
    a = np.asarray(arr, dtype=np.float64)
    if a.shape != tuple(n_global):
        raise DeckError(f"dump shape {a.shape} against the header's {tuple(n_global)}")
    with open(filename, "wb") as f:
        f.write(_PXR_HEADER.pack(lo[0], hi[0], n_global[0], lo[1], hi[1], n_global[1],
                                 lo[2], hi[2], n_global[2]))
        f.write(np.asfortranarray(a).tobytes(order="F"))


def read_pxr(filename):
    """(header dict, array of shape (nx, ny, nz)) of a ``.pxr`` dump."""
    with open(filename, "rb") as f:
        raw = f.read()
    h = _PXR_HEADER.unpack_from(raw, 0)
    n = (h[2], h[5], h[8])
    data = np.frombuffer(raw, dtype=np.float64, offset=_PXR_HEADER.size,
                         count=n[0] * n[1] * n[2])
    hdr = {"xmin": h[0], "xmax": h[1], "nx": n[0], "ymin": h[3], "ymax": h[4], "ny": n[1],
           "zmin": h[6], "zmax": h[7], "nz": n[2]}
    return hdr, data.reshape(n, order="F")


def _step_label(it):
    """``WRITE(strtemp, '(I5)') it`` then trimmed: '*****' past five digits."""
    s = str(it)
    return s if len(s) <= 5 else "*****"


# -------------------------------------------------------------- run state
class _Grids:
    """Node views of a module's grids (device tensors) for the dumps and the
    diagnostics."""

    def __init__(self, m, deck, der):
        self.m, self.deck, self.der = m, deck, der
        self.two_d = deck.c_dim == 2
        self.n = der["n"]
        self.g = m.nxguards

    def _full(self, name):
        """The guarded grid as (x, y, z) FP64 tensor (2D: y extent 1)."""
        import torch
        a = getattr(self.m, name).to(torch.float64)
        return a[:, None, :] if self.two_d else a

    def nodes(self, name, lo=0, hi=None):
        """Nodes lo..hi-1 per axis (hi default n; 2D: the one y plane)."""
        g = self.g
        nx, ny, nz = self.n
        hx, hy, hz = (nx, ny, nz) if hi is None else hi
        a = self._full(name)
        if self.two_d:
            return a[g + lo:g + hx, :, g + lo:g + hz]
        return a[g + lo:g + hx, g + lo:g + hy, g + lo:g + hz]

    def div(self, fx, fy, fz, forward=False):
        """calc_field_div (backward differences, nodes 0..n) or calc_field_divB
        (forward differences, nodes 1..n, node 0 left at zero) over nodes
        0..n, as a device tensor.  2D: the x-z divergence."""
        import torch
        g = self.g
        nx, ny, nz = self.n
        d = self.der
        ax, ay, az = (self._full(c) for c in (fx, fy, fz))
        gy, ey = (0, 1) if self.two_d else (g, ny + 1)
        X = lambda k: slice(g + k, g + nx + 1 + k)
        Y = lambda k: slice(gy + k, gy + ey + k)
        Z = lambda k: slice(g + k, g + nz + 1 + k)
        if not forward:
            out = (1.0 / d["dx"]) * (ax[X(0), Y(0), Z(0)] - ax[X(-1), Y(0), Z(0)])
            if not self.two_d:
                out = out + (1.0 / d["dy"]) * (ay[X(0), Y(0), Z(0)] - ay[X(0), Y(-1), Z(0)])
            return out + (1.0 / d["dz"]) * (az[X(0), Y(0), Z(0)] - az[X(0), Y(0), Z(-1)])
        out = torch.zeros((nx + 1, ey, nz + 1), dtype=torch.float64, device=ax.device)
        X1 = lambda k: slice(g + 1 + k, g + nx + 1 + k)
        Y1 = (lambda k: slice(0, 1)) if self.two_d else (lambda k: slice(g + 1 + k, g + ny + 1 + k))
        Z1 = lambda k: slice(g + 1 + k, g + nz + 1 + k)
        v = (1.0 / d["dx"]) * (ax[X1(1), Y1(0), Z1(0)] - ax[X1(0), Y1(0), Z1(0)])
        if not self.two_d:
            v = v + (1.0 / d["dy"]) * (ay[X1(0), Y1(1), Z1(0)] - ay[X1(0), Y1(0), Z1(0)])
        v = v + (1.0 / d["dz"]) * (az[X1(0), Y1(0), Z1(1)] - az[X1(0), Y1(0), Z1(0)])
        if self.two_d:
            out[1:, :, 1:] = v
        else:
            out[1:, 1:, 1:] = v
        return out


class _Temporal:
    """The temporal diagnostic files (diags.F90:253-420, simple_io.F90:
    236-455): one file per active diagnostic with its header, one record per
    output iteration."""

    def __init__(self, deck, der, out_dir, nspecies):
        self.deck, self.der = deck, der
        self.files = []
        if deck.temdiag_frequency <= 0:
            return
        for i, name in enumerate(_TEMPORAL_NAMES):
            if deck.temdiag_act_list[i] > 0:
                nb = nspecies if i == 0 else 1
                path = os.path.join(out_dir, name)
                val = deck.temdiag_frequency * der["dt"]
                if deck.temdiag_format == 1:
                    with open(path, "w") as f:
                        f.write(f" {nb} {val!r}\n")
                else:
                    with open(path, "wb") as f:
                        f.write(struct.pack("<id", nb, val))
                self.files.append((i, path))

    def due(self, it):
        return bool(self.files) and it % self.deck.temdiag_frequency == 0

    def write(self, values):
        for i, path in self.files:
            v = values[i]
            if self.deck.temdiag_format == 1:
                with open(path, "a") as f:
                    f.write(" " + " ".join(repr(float(x)) for x in v) + "\n")
            else:
                with open(path, "ab") as f:
                    f.write(np.asarray(v, dtype="<f8").tobytes())


def _temporal_values(m, deck, grids, need):
    """The diagnostics of simple_io.F90:236-408 for the active entries (FP64
    sums on the device)."""
    import torch
    der = grids.der
    vals = {}
    if need[0]:
        ke = []
        for sp in m.species:
            gi = sp.part_gaminv.to(torch.float64)
            w = sp.pid_w.to(torch.float64)
            # (reference: the electron mass for every species)
            ke.append(float(((1.0 / gi - 1.0) * w).sum()) * EMASS * CLIGHT ** 2)
        vals[0] = ke
    dv = der["dx"] * der["dz"] * (1.0 if grids.two_d else der["dy"])
    n = grids.n
    hi = (n[0] + 1, n[1] + 1, n[2] + 1)
    for i, name, k in ((1, "ex", EPS0), (2, "ey", EPS0), (3, "ez", EPS0), (4, "bx", IMU0),
                       (5, "by", IMU0), (6, "bz", IMU0)):
        if need[i]:
            a = grids.nodes(name, 1, hi)
            vals[i] = [float((a * a * 0.5).sum()) * dv * k]
    if need[7] or need[8] or need[9]:
        if grids.two_d:
            raise DeckError("the rho diagnostics need the 2D charge deposition, not built")
        dive = grids.div("ex", "ey", "ez")[1:, 1:, 1:]
        rho = grids.nodes("rho", 1, hi)
        if need[7]:
            vals[7] = [math.sqrt(float(((dive * EPS0 - rho) ** 2).sum()))]
        if need[8]:
            vals[8] = [math.sqrt(float((rho ** 2).sum()))]
        if need[9]:
            vals[9] = [math.sqrt(float((dive ** 2).sum()))]
    return vals


def _output_fields(m, deck, grids, it, out_dir):
    """The field dumps of output_routines (simple_io.F90:62-223)."""
    if deck.output_frequency < 1:
        return []
    if not (deck.output_step_min <= it <= deck.output_step_max and
            (it - deck.output_step_min) % deck.output_frequency == 0):
        return []
    n = grids.n
    if grids.two_d:
        lo, hi, ng = (deck.xmin, -HUGE, deck.zmin), (deck.xmax, HUGE, deck.zmax), (n[0], 1, n[2])
    else:
        lo, hi, ng = (deck.xmin, deck.ymin, deck.zmin), (deck.xmax, deck.ymax, deck.zmax), n
    written = []
    lab = _step_label(it)
    for name in _OUTPUT_FIELDS:
        if deck.c_output[name] != 1:
            continue
        if name in ("dive", "divj", "divb"):
            src = {"dive": ("ex", "ey", "ez", False), "divj": ("jx", "jy", "jz", False),
                   "divb": ("bx", "by", "bz", True)}[name]
            arr = grids.div(*src)[:n[0], :ng[1], :n[2]]
        else:
            if name == "rho" and grids.two_d:
                raise DeckError("rho dumps need the 2D charge deposition, not built")
            arr = grids.nodes(name)
        path = os.path.join(out_dir, f"{name}{lab}.pxr")
        write_pxr(path, arr.cpu().numpy(), lo, hi, ng)
        written.append(path)
    return written


def _output_particles(m, deck, it, out_dir):
    """The particle dumps of write_particles_to_file (simple_io.F90:601-697,
    one domain): ``<species>_it_<it>`` holding x, y, z, ux, uy, uz and the
    weight of the selected particles, each as a block of FP64 values.  The
    selection is strict on every bound (get_particles_to_dump,
    :709-761); the reference marks its mask at tile-local indices but reads
    it at global ones, which agree with one tile, the case here."""
    import torch
    written = []
    lab = _step_label(it)
    for dp in deck.particle_dumps:
        if dp.diag_period < 1 or it % dp.diag_period != 0 or dp.ispecies < 0:
            continue
        sp = m.species[dp.ispecies]
        cols = [getattr(sp, c).to(torch.float64) for c in
                ("part_x", "part_y", "part_z", "part_ux", "part_uy", "part_uz", "pid_w")]
        x, y, z, ux, uy, uz, _ = cols
        keep = ((x > dp.dump_x_min) & (x < dp.dump_x_max) & (y > dp.dump_y_min) &
                (y < dp.dump_y_max) & (z > dp.dump_z_min) & (z < dp.dump_z_max) &
                (ux > dp.dump_ux_min) & (ux < dp.dump_ux_max) & (uy > dp.dump_uy_min) &
                (uy < dp.dump_uy_max) & (uz > dp.dump_uz_min) & (uz < dp.dump_uz_max))
        path = os.path.join(out_dir, f"{sp.name}_it_{lab}")
        with open(path, "wb") as f:
            for c in cols:
                f.write(c[keep].cpu().numpy().astype("<f8").tobytes())
        written.append(path)
    return written


def read_particle_dump(path):
    """{x, y, z, ux, uy, uz, w} of a particle dump file."""
    v = np.fromfile(path, dtype="<f8")
    n = v.size // 7
    return {c: v[i * n:(i + 1) * n] for i, c in enumerate(("x", "y", "z", "ux", "uy", "uz",
                                                            "w"))}


def build(deck, engine="plain", precision="fp64", device="cuda", seed=0, tiled_config=None):
    """The deck's simulation: a ``PicsarModule`` (c_dim 3) or ``PicsarModule2D``
    (c_dim 2) in SI units with its species loaded.  Returns (module, derived)."""
    if deck.antenna:
        raise DeckError("the laser antenna is not supported")
    if deck.g_spectral or deck.fftw_with_mpi or deck.p3dfft_flag:
        raise DeckError("spectral variants other than the local-FFT PSATD push are not "
                        "supported (g_spectral, distributed FFTs)")
    if deck.l_spectral and (deck.c_dim != 3 or engine != "plain"):
        raise DeckError("the spectral (PSATD) solver runs 3D decks on the plain engine")
    if deck.absorbing_bcs_x or deck.absorbing_bcs_y or deck.absorbing_bcs_z or \
            deck.nx_pml or deck.ny_pml or deck.nz_pml:
        raise DeckError("PML / absorbing field boundaries are not supported")
    if deck.nox != deck.noz or (deck.c_dim == 3 and deck.nox != deck.noy):
        raise DeckError("different shape orders per axis are not supported")
    if deck.nox not in (1, 2, 3):
        raise DeckError(f"shape order {deck.nox}")
    der = deck.derived()
    nx, ny, nz = der["n"]
    from .picsar import PicsarModule, PicsarModule2D
    parts = load_particles(deck, seed=seed)
    if deck.c_dim == 2:
        if engine != "plain":
            raise DeckError("2D decks run on the plain engine")
        ng = max(deck.nxguards, deck.nzguards, deck.nxjguards, deck.nzjguards, deck.nox + 1)
        m = PicsarModule2D(nx, nz, nguards=ng, dx=der["dx"], dz=der["dz"], xmin=deck.xmin,
                           zmin=deck.zmin, dt=der["dt"], nox=deck.nox,
                           particle_pusher=deck.particle_pusher, clight=CLIGHT, mu0=MU0,
                           eps0=EPS0, device=device)
    else:
        ng = max(deck.nxguards, deck.nyguards, deck.nzguards, deck.nxjguards, deck.nyjguards,
                 deck.nzjguards, deck.nox + 1)
        if engine == "tiled":
            if len(deck.species) > 1:
                raise DeckError("the tiled engine pushes one species; run several species "
                                "with engine='plain'")
            if (deck.norderx, deck.nordery, deck.norderz) != (2, 2, 2):
                raise DeckError("the tiled engine runs the 2nd-order Yee solver")
            ng = 3
        m = PicsarModule(nx, ny, nz, nguards=ng, dx=der["dx"], dy=der["dy"], dz=der["dz"],
                         xmin=deck.xmin, ymin=deck.ymin, zmin=deck.zmin, dt=der["dt"],
                         nox=deck.nox, particle_pusher=deck.particle_pusher, clight=CLIGHT,
                         mu0=MU0, eps0=EPS0, device=device, engine=engine,
                         precision=precision, tiled_config=tiled_config)
        m.norderx, m.nordery, m.norderz = deck.norderx, deck.nordery, deck.norderz
        m.l_lower_order_in_v = deck.l_lower_order_in_v
        m.l_spectral, m.l_staggered = bool(deck.l_spectral), bool(deck.l_staggered)
        if engine == "plain":
            m.sorting_activated = deck.sorting_activated
            m.sorting_dx, m.sorting_dy, m.sorting_dz = der["sorting_d"]
            m.sorting_shiftx, m.sorting_shifty, m.sorting_shiftz = der["sorting_shift"]
    for sp, p in zip(deck.species, parts):
        if deck.c_dim == 2:
            m.add_species(sp.name, sp.charge, sp.mass, p["x"], p["y"], p["z"], p["ux"],
                          p["uy"], p["uz"], p["w"])
        else:
            m.add_species(sp.name, sp.charge, sp.mass, p["x"], p["y"], p["z"], p["ux"],
                          p["uy"], p["uz"], p["w"], sorting_period=sp.sorting_period,
                          sorting_start=sp.sorting_start)
    return m, der


def run_deck(deck, out_dir="RESULTS", engine="plain", precision="fp64", device="cuda", seed=0,
             nsteps=None, tiled_config=None):
    """Run a deck (a Deck or a ``.pixr`` path) for its ``nsteps`` (or the given
    number) of iterations, writing its field dumps and temporal diagnostics
    under out_dir.  Returns (module, {"dumps": [...], "nsteps": n})."""
    if not isinstance(deck, Deck):
        deck = read_input_file(deck)
    m, der = build(deck, engine=engine, precision=precision, device=device, seed=seed,
                   tiled_config=tiled_config)
    os.makedirs(out_dir, exist_ok=True)
    grids = _Grids(m, deck, der)
    temporal = _Temporal(deck, der, out_dir, len(deck.species))
    need = [deck.temdiag_act_list[i] > 0 for i in range(10)]
    dumps = []
    steps = der["nsteps"] if nsteps is None else int(nsteps)
    rho_on = deck.l_plasma and deck.c_dim == 3
    for it in range(steps):
        if deck.c_dim == 2:
            m.step(1)
        else:
            m.step(1, diags=rho_on)          # calc_diags: rho deposition + charge_bcs
        dumps += _output_fields(m, deck, grids, it, out_dir)
        if deck.c_dim == 3:
            dumps += _output_particles(m, deck, it, out_dir)
        if temporal.due(it):
            temporal.write(_temporal_values(m, deck, grids, need))
    return m, {"dumps": dumps, "nsteps": steps, "derived": der}


def main(argv=None):
    """``python -m picsar_b200.deck [deck.pixr] [--engine plain|tiled]
    [--precision fp64|fp32] [--seed N]``: the mini-app executable's use of a
    deck (control_file.F90:452-458: the first argument names the deck when
    it contains '.pixr', else ``input_file.pixr``), outputs under
    ``./RESULTS``."""
    import argparse
    import sys
    argv = sys.argv[1:] if argv is None else argv
    ap = argparse.ArgumentParser(prog="python -m picsar_b200.deck")
    ap.add_argument("deck", nargs="?", default="")
    ap.add_argument("--engine", default="plain", choices=["plain", "tiled"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default="RESULTS")
    a = ap.parse_args(argv)
    path = a.deck if ".pixr" in a.deck else "input_file.pixr"
    if not os.path.exists(path):
        print(f"Error opening input file [{path}]. Check input filename.", file=sys.stderr)
        return 1
    m, info = run_deck(path, out_dir=a.out, engine=a.engine, precision=a.precision,
                       seed=a.seed)
    der = info["derived"]
    print(f"{path}: {info['nsteps']} steps of dt = {der['dt']:.6g} s on the {a.engine} "
          f"engine; {len(info['dumps'])} field dumps in {a.out}/")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
