"""Host side of the tiled engine (FP32 mixed precision or FP64).

``TiledSim`` owns one periodic simulation in the B200-native layout (see
``pxrb_tiled_job`` in include/picsar_b200.h) and runs the per-step loop of
src/submain.F90:104-195 as four launches:

  1. fused particle kernel: gather + push + position push + periodic wrap +
     Esirkepov deposition into J (FP64, flushed once per tile);
  2. B half push; 3. E push (J consumed and zeroed); 4. B half push;

plus a counting sort by cell tile every ``sort_interval`` steps (the
reference's pxr_particle_sorting).  Guard cells of E/B are refreshed by the
Yee kernels themselves, and J is deposited with periodic wrapping, so the
reference's field_bc / current_bcs exchanges have no separate launches.

All device work goes through the C ABI of libpicsar_b200.so; torch only
allocates memory and provides the stream.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import PicsarB200Error

_P = C.c_void_p


class TiledJob(C.Structure):
    """Mirror of ``pxrb_tiled_job`` (include/picsar_b200.h)."""
    _fields_ = (
        [(n, C.c_int32) for n in ("nx", "ny", "nz", "tx", "ty", "tz", "ntx", "nty", "ntz", "g",
                                  "pitch_x", "order", "pusher", "drift", "prec", "pitch_y")]
        + [("np", C.c_int64)]
        + [(n, C.c_double) for n in ("dx", "dy", "dz", "dt", "q", "m", "clight", "mu0", "eps0",
                                     "xmin", "ymin", "zmin")]
        + [(n, _P) for n in ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz", "cell", "ox",
                             "oy", "oz", "ux", "uy", "uz", "w", "cell_b", "ox_b", "oy_b", "oz_b",
                             "ux_b", "uy_b", "uz_b", "w_b", "pid", "pid_b", "tile_off",
                             "tile_cnt", "ke_tile", "counters", "cell_cnt", "rank_b", "perm",
                             "tile_stats")]
        + [(n, C.c_int32) for n in ("select_lanes", "cell_order")]
    )


_lib.register({
    "pxrb_tiled_particle_step": "p I I I I I p I p p I I i s",
    "pxrb_tiled_push_b": "p I I p i d s",
    "pxrb_tiled_push_e": "p I I p i I s",
    "pxrb_tiled_sort": "p p s",
    "pxrb_tiled_relayout": "p I I I i s",
    "pxrb_tiled_load_particles": "p p p p p p p p s",
    "pxrb_tiled_store_particles": "p p p p p p p p p s",
    "pxrb_tiled_store_particles_by_id": "p i I p p p p p p p p s",
    "pxrb_tiled_field_import": "p I p i s",
    "pxrb_tiled_field_export": "p I p i s",
    "pxrb_tiled_diagnostics": "p p p i p s",
    "pxrb_tiled_smem_bytes": "=i I I I I I I I",
    "pxrb_tiled_job_size": "=i",
    "pxrb_tiled_max_threads": "I",
    "pxrb_tiled_diag_scratch": "=i p",
    "pxrb_tiled_diagnostics_noalloc": "p I p s",
})


def smem_bytes(order, prec, acc, tile, drift):
    return _lib.query("pxrb_tiled_smem_bytes", order, prec, acc, tile[0], tile[1], tile[2],
                      drift)


def _check_layout():
    n = _lib.query("pxrb_tiled_job_size")
    if n != C.sizeof(TiledJob):
        raise PicsarB200Error(f"pxrb_tiled_job layout mismatch: C {n} B, Python {C.sizeof(TiledJob)} B")


_I32MAX = 2 ** 31 - 1
# (tile edge, window margin) pairs the particle kernel is compiled for
SUPPORTED_SHAPES = {(8, 1), (8, 0), (8, 2), (4, 1), (4, 0)}
# ... and those of the FP64 engine
SUPPORTED_SHAPES_FP64 = {(8, 1), (8, 0), (4, 1), (4, 0)}
# accumulator modes compiled for the FP32 engine per shape (FP64 engine: mode 3)
SUPPORTED_ACC = {(8, 1): (0, 1, 2, 4), (8, 2): (1, 2), (4, 1): (1, 2)}


def launch_threads(cfg, acc):
    """CTA size of the particle kernel for a configuration and accumulator:
    `threads` for the FP32 engine, `fp64_threads` for the FP64 one (mode 3),
    each at most pxrb_tiled_max_threads(acc)."""
    want = cfg.fp64_threads if acc == 3 else cfg.threads
    return min(want, _lib.query("pxrb_tiled_max_threads", acc))


@dataclass
class TiledConfig:
    """Tuning knobs of the tiled engine (chosen by picsar_b200.autotune)."""
    tile: tuple = (8, 8, 8)
    drift: int = 1
    threads: int = 256
    ctas_per_sm: int = 2
    sort_interval: int = 20
    relayout_interval: int = 4  # bank-order re-layout of the tiles between sorts (0: none)
    acc: int = 2                # FP32 engine current accumulator (see picsar_b200.h)
    select_lanes: bool = True   # FP32 engine: distinct bank classes per warp, second pass
    fp64_threads: int = 512     # FP64 engine's CTA size (one CTA per SM; `threads` is FP32's)


def h2d_bytes(buf):
    """Host bytes staged in pinned memory for a non-blocking copy to the
    device (torch keeps the pinned block until the copy has run).  A blocking
    copy from pageable memory would synchronise the stream it is issued on."""
    return torch.frombuffer(bytearray(buf), dtype=torch.uint8).pin_memory()


def h2d(t, device):
    """A host tensor on the device without blocking the host (see h2d_bytes)."""
    return t.pin_memory().to(device, non_blocking=True)


def _stream():
    return torch.cuda.current_stream().cuda_stream


class TiledSim:
    """One periodic PIC simulation in the tiled B200 layout."""

    def __init__(self, n, order=1, pusher=0, precision="fp32", d=(1.0, 1.0, 1.0),
                 xmin=(0.0, 0.0, 0.0), dt=None, q=-1.0, m=1.0, clight=1.0, mu0=1.0, eps0=1.0,
                 config: TiledConfig | None = None, track_ids=False, device="cuda"):
        _check_layout()
        cfg = config or TiledConfig()
        self.cfg = cfg
        self.device = torch.device(device)
        nx, ny, nz = (int(v) for v in n)
        if nx > 2048 or ny > 2048 or nz > 1024:
            raise ValueError("the packed cell index allows nx, ny <= 2048 and nz <= 1024")
        if order not in (1, 2, 3):
            raise ValueError("shape order must be 1, 2 or 3")
        self.n, self.order, self.pusher = (nx, ny, nz), int(order), int(pusher)
        self.prec = 0 if precision in ("fp32", "mixed", torch.float32) else 1
        self.rdtype = torch.float32 if self.prec == 0 else torch.float64
        self.d = tuple(float(v) for v in d)
        self.xmin = tuple(float(v) for v in xmin)
        if dt is None:
            dt = 0.95 / (clight * math.sqrt(sum(1.0 / v ** 2 for v in self.d)))
        self.dt = float(dt)
        self.q, self.m, self.clight, self.mu0, self.eps0 = q, m, clight, mu0, eps0
        tile = tuple(int(t) for t in cfg.tile)
        if not (tile[0] == tile[1] == tile[2]) or (tile[0], cfg.drift) not in SUPPORTED_SHAPES:
            raise ValueError(f"tile {tile} with drift {cfg.drift} not compiled; "
                             f"supported (edge, drift): {sorted(SUPPORTED_SHAPES)}")
        if self.prec == 1 and (tile[0], cfg.drift) not in SUPPORTED_SHAPES_FP64:
            raise ValueError(f"tile {tile} with drift {cfg.drift} not compiled for FP64; "
                             f"supported (edge, drift): {sorted(SUPPORTED_SHAPES_FP64)}")
        self.tile = tile
        self.g = max(3, cfg.drift + 2)
        if min(self.n) < 2 * self.g:
            raise ValueError(f"each axis needs at least {2 * self.g} cells")
        self.nt = tuple(-(-v // t) for v, t in zip(self.n, tile))
        self.ntiles = self.nt[0] * self.nt[1] * self.nt[2]
        al = 4 if self.prec == 0 else 2          # 16-byte rows (TMA-compatible pitch)
        # every tile window fits: pad each axis to whole tiles plus guards
        self.pitch = -(-(self.nt[0] * tile[0] + 2 * self.g) // al) * al
        self.pitch_y = self.nt[1] * tile[1] + 2 * self.g
        fshape = (self.nt[2] * tile[2] + 2 * self.g, self.pitch_y, self.pitch)
        dev, rd = self.device, self.rdtype
        self.E = [torch.zeros(fshape, dtype=rd, device=dev) for _ in range(3)]
        self.B = [torch.zeros(fshape, dtype=rd, device=dev) for _ in range(3)]
        self.J = [torch.zeros(nx * ny * nz, dtype=torch.float64, device=dev) for _ in range(3)]
        self.rho = torch.zeros(nx * ny * nz, dtype=torch.float64, device=dev)
        self.tile_off = torch.zeros(self.ntiles + 1, dtype=torch.int32, device=dev)
        self.tile_cnt = torch.zeros(self.ntiles + 1, dtype=torch.int32, device=dev)
        self.ke_tile = torch.zeros(self.ntiles, dtype=torch.float64, device=dev)
        self.tile_stats = torch.zeros(self.ntiles * 4, dtype=torch.float32, device=dev)
        self.cell_cnt = torch.zeros(self.ntiles * tile[0] * tile[1] * tile[2], dtype=torch.int32,
                                    device=dev)
        self.counters = torch.zeros(4, dtype=torch.int32, device=dev)
        # (built on the device: a blocking host copy would wait for the stream)
        self.work = torch.zeros((self.ntiles, 2), dtype=torch.int32, device=dev)
        self.work[:, 1] = torch.arange(self.ntiles, dtype=torch.int32, device=dev)
        self.ctr = torch.zeros(1, dtype=torch.int32, device=dev)
        ncell = nx * ny * nz
        self.total_cells = -(-ncell // 1024) * 1024
        self.cell_off = torch.zeros(2, dtype=torch.int64, device=dev)
        self.cell_off[1] = self.total_cells
        self.diag_out = torch.zeros(9, dtype=torch.float64, device=dev)
        self.track_ids = track_ids
        self.np = 0
        self.it = 0
        self.launches = 0          # kernels of this library launched so far
        self.acc = 3 if self.prec == 1 else cfg.acc
        if self.prec == 0 and self.acc not in SUPPORTED_ACC.get((tile[0], cfg.drift), (2,)):
            raise ValueError(f"accumulator mode {self.acc} not compiled for this tile shape")
        if self.acc == 4 and self.order == 2:
            raise ValueError("the cell-grouped kernel (mode 4) takes shape orders 1 and 3")
        self.smem = smem_bytes(self.order, self.prec, self.acc, tile, cfg.drift)
        props = torch.cuda.get_device_properties(self.device)
        self.num_sms = props.multi_processor_count
        self.job = TiledJob()
        self.job_dev = torch.zeros(C.sizeof(TiledJob), dtype=torch.uint8, device=dev)
        self._fill_job()

    # ------------------------------------------------------------------ setup
    def _fill_job(self):
        j = self.job
        j.nx, j.ny, j.nz = self.n
        j.tx, j.ty, j.tz = self.tile
        j.ntx, j.nty, j.ntz = self.nt
        j.g, j.pitch_x, j.order, j.pusher = self.g, self.pitch, self.order, self.pusher
        j.pitch_y = self.pitch_y
        j.drift, j.prec, j.np = self.cfg.drift, self.prec, self.np
        j.dx, j.dy, j.dz = self.d
        j.dt, j.q, j.m, j.clight, j.mu0, j.eps0 = (self.dt, self.q, self.m, self.clight,
                                                   self.mu0, self.eps0)
        j.xmin, j.ymin, j.zmin = self.xmin
        for name, t in zip(("ex", "ey", "ez"), self.E):
            setattr(j, name, t.data_ptr())
        for name, t in zip(("bx", "by", "bz"), self.B):
            setattr(j, name, t.data_ptr())
        for name, t in zip(("jx", "jy", "jz"), self.J):
            setattr(j, name, t.data_ptr())
        j.tile_off, j.tile_cnt = self.tile_off.data_ptr(), self.tile_cnt.data_ptr()
        j.ke_tile, j.counters = self.ke_tile.data_ptr(), self.counters.data_ptr()
        j.cell_cnt = self.cell_cnt.data_ptr()
        j.tile_stats = self.tile_stats.data_ptr()
        j.select_lanes = int(bool(self.cfg.select_lanes))
        j.cell_order = int(self.acc == 4)
        self._push_job()

    def _jp(self):
        return C.addressof(self.job)

    def _push_job(self):
        """Copy the host descriptor to the device in stream order, without
        blocking the host."""
        self.job_dev.copy_(h2d_bytes(bytes(self.job)), non_blocking=True)

    def set_job_bytes(self, raw):
        """Replace the host descriptor by `raw` (a host uint8 tensor holding a
        copy of the device descriptor)."""
        if raw.numel() != C.sizeof(TiledJob):
            raise ValueError("descriptor size mismatch")
        C.memmove(C.addressof(self.job), raw.data_ptr(), C.sizeof(TiledJob))

    def _pull_job(self):
        """Refresh the host descriptor from the device (the sort swaps the
        particle array pointers there)."""
        raw = self.job_dev.cpu().numpy().tobytes()
        C.memmove(C.addressof(self.job), raw, len(raw))

    def load_particles(self, x, y, z, ux, uy, uz, w, ids=None, ids_dense=None, sort=True):
        """Load particles given as PICSAR arrays (absolute FP64 positions),
        device tensors or host arrays (pinned host tensors are uploaded
        without blocking the host).  ids (tracked ids only): the particles'
        identifiers, by default 0..N-1; ids_dense: True when ids is a
        permutation of 0..N-1 (then particles() restores the id order by a
        scatter instead of a sort).  sort=False leaves the particles unsorted
        (the caller sorts before stepping); the host descriptor then still
        points at the arrays the device uses."""
        dev = self.device

        def f64(a):
            t = torch.as_tensor(a, dtype=torch.float64)
            return t.to(dev, non_blocking=t.is_pinned()).contiguous()
        x, y, z, ux, uy, uz, w = (f64(a) for a in (x, y, z, ux, uy, uz, w))
        N = int(x.numel())
        if N > _I32MAX:
            raise ValueError("at most 2^31-1 particles per simulation")
        self.np = N
        rd = self.rdtype
        mk = lambda dt=rd: torch.empty(N, dtype=dt, device=dev)
        self.parts = {c: mk() for c in ("ox", "oy", "oz", "ux", "uy", "uz", "w")}
        self.parts_b = {c: mk() for c in ("ox", "oy", "oz", "ux", "uy", "uz", "w")}
        self.cell = torch.empty(N, dtype=torch.int32, device=dev)
        self.cell_b = torch.empty(N, dtype=torch.int32, device=dev)
        self.rank_b = torch.empty(N, dtype=torch.int32, device=dev)
        self.perm = torch.empty(N, dtype=torch.int32, device=dev)
        j = self.job
        j.np = N
        j.cell, j.cell_b = self.cell.data_ptr(), self.cell_b.data_ptr()
        j.rank_b = self.rank_b.data_ptr()
        j.perm = self.perm.data_ptr()
        for c in ("ox", "oy", "oz", "ux", "uy", "uz", "w"):
            setattr(j, c, self.parts[c].data_ptr())
            setattr(j, c + "_b", self.parts_b[c].data_ptr())
        if self.track_ids:
            idt = (torch.arange(N, dtype=torch.int32, device=dev) if ids is None
                   else torch.as_tensor(ids).to(dev, torch.int32))
            self._ids_dense = ids is None or bool(ids_dense)
            self.pid, self.pid_b = idt.contiguous(), torch.empty(N, dtype=torch.int32, device=dev)
            j.pid, j.pid_b = self.pid.data_ptr(), self.pid_b.data_ptr()
        else:
            j.pid = j.pid_b = None
        self._push_job()
        _lib.call("pxrb_tiled_load_particles", self._jp(), x.data_ptr(), y.data_ptr(),
                  z.data_ptr(), ux.data_ptr(), uy.data_ptr(), uz.data_ptr(), w.data_ptr(),
                  _stream())
        if sort:
            self.sort()

    def load_state(self, st):
        """Load a picsar_b200.init.PlasmaState."""
        self.load_particles(st.x, st.y, st.z, st.ux, st.uy, st.uz, st.w)

    def import_field(self, name, arr, nguard):
        """Copy a PICSAR guarded FP64 Fortran grid (ex..bz, jx..jz) in."""
        which = ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz").index(name)
        _lib.call("pxrb_tiled_field_import", self._jp(), which, arr.data_ptr(), nguard,
                  _stream())

    def export_field(self, name, nguard):
        from .picsar import grid_zeros
        which = ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz").index(name)
        out = grid_zeros(*self.n, nguard, device=self.device)
        _lib.call("pxrb_tiled_field_export", self._jp(), which, out.data_ptr(), nguard,
                  _stream())
        return out

    # -------------------------------------------------------------- stepping
    def sort(self):
        # sizes, tile_cnt and tile_off of the host descriptor never change;
        # the particle pointers it holds may be stale (the device swaps them)
        _lib.call("pxrb_tiled_sort", self._jp(), self.job_dev.data_ptr(), _stream())
        self.launches += 7 if self.np > 0 else 1   # the particle arrays now sit in the former *_b buffers

    def arrays(self):
        """The particle arrays the device descriptor currently points at
        (sorts and re-layouts exchange them with their scratch copies):
        {"cell", "ox", "oy", "oz", "ux", "uy", "uz", "w"} tensors, and "pid"
        when ids are tracked."""
        self._pull_job()
        j = self.job
        out = {"cell": self.cell if self.cell.data_ptr() == j.cell else self.cell_b}
        for c in ("ox", "oy", "oz", "ux", "uy", "uz", "w"):
            a, b = self.parts[c], self.parts_b[c]
            out[c] = a if a.data_ptr() == getattr(j, c) else b
        if self.track_ids and j.pid:
            out["pid"] = self.pid if self.pid.data_ptr() == j.pid else self.pid_b
        return out

    def relayout(self):
        """Restore the bank order inside every tile for the particles' current
        cells (particles keep their tiles)."""
        if self.np > 0:
            _lib.call("pxrb_tiled_relayout", self.job_dev.data_ptr(), 1, self.prec, self.ntiles,
                      self.np, _stream())
            self.launches += 3      # the particle arrays now sit in the former *_b buffers

    def particle_step(self):
        ctas = min(self.ntiles, self.num_sms * self.cfg.ctas_per_sm)
        _lib.call("pxrb_tiled_particle_step", self.job_dev.data_ptr(), self.order, self.prec,
                  self.tile[0], self.cfg.drift, self.acc, self.work.data_ptr(), self.ntiles, None, self.ctr.data_ptr(),
                  launch_threads(self.cfg, self.acc), ctas, self.smem, _stream())
        self.launches += 1

    def push_b(self, frac=0.5):
        _lib.call("pxrb_tiled_push_b", self.job_dev.data_ptr(), 1, self.prec,
                  self.cell_off.data_ptr(), self.total_cells, frac, _stream())
        self.launches += 1

    def push_e(self, zero_j=True):
        _lib.call("pxrb_tiled_push_e", self.job_dev.data_ptr(), 1, self.prec,
                  self.cell_off.data_ptr(), self.total_cells, int(zero_j), _stream())
        self.launches += 1

    def step(self, nsteps=1, keep_j=False, events=None):
        """nsteps PIC steps.  keep_j: leave the last step's J in place (it is
        otherwise consumed by the E push); the next step clears it.  events:
        a (start, end) pair of CUDA events recorded around the particle
        kernel (nsteps = 1)."""
        for s in range(nsteps):
            if getattr(self, "_j_dirty", False):
                for t in self.J:
                    t.zero_()
                self._j_dirty = False
            if events is not None:
                events[0].record(torch.cuda.current_stream())
            self.particle_step()
            if events is not None:
                events[1].record(torch.cuda.current_stream())
            self.push_b(0.5)
            last = s == nsteps - 1
            self.push_e(zero_j=not (keep_j and last))
            if keep_j and last:
                self._j_dirty = True
            self.push_b(0.5)
            self.it += 1
            self.housekeeping()

    def housekeeping(self):
        """The engine's particle-order schedule after step `it`: the sort every
        sort_interval steps, the bank re-layout every relayout_interval steps
        between sorts."""
        if self.cfg.sort_interval > 0 and self.it % self.cfg.sort_interval == 0:
            self.sort()
        elif (self.cfg.relayout_interval > 0 and self.acc != 4
              and self.it % self.cfg.relayout_interval == 0):
            self.relayout()      # (the cell-grouped kernel orders particles itself)

    # ----------------------------------------------------------- diagnostics
    def diagnostics(self, gauss=True, to_host=True, pull=True):
        """FP64 energies and (gauss=True) the Gauss-law residual of the current
        state; to_host=False leaves the 9 values in self.diag_out (device).
        pull=False: the host descriptor is known to be current (no sort or
        re-layout since the load), so it is not read back from the device."""
        n_scr = _lib.query("pxrb_tiled_diag_scratch", self._jp())
        if getattr(self, "_scratch", None) is None or self._scratch.numel() < n_scr:
            self._scratch = torch.zeros(n_scr, dtype=torch.float64, device=self.device)
        if gauss and pull:
            self._pull_job()     # rho deposition reads the current particle arrays
        _lib.call("pxrb_tiled_diagnostics", self._jp(),
                  self.rho.data_ptr() if gauss else None, self._scratch.data_ptr(),
                  self._scratch.numel(), self.diag_out.data_ptr(), _stream())
        if not to_host:
            return self.diag_out
        o = self.diag_out.cpu().tolist()
        return {"kinetic": o[0], "ex": o[1], "ey": o[2], "ez": o[3], "bx": o[4], "by": o[5],
                "bz": o[6], "gauss_norm": o[7], "rho_norm": o[8], "field": sum(o[1:7]),
                "total": o[0] + sum(o[1:7])}

    def diagnostics_noalloc(self, gauss=True, out=None):
        """Same values as diagnostics(), computed by the entry point that
        allocates nothing (its scratch is a static device array of the
        library; jobs up to 1,048,576 cells).  out: optional DEVICE float64[9]
        tensor that receives the values."""
        if out is None:
            out = self.diag_out
        if gauss:
            self._pull_job()
        _lib.call("pxrb_tiled_diagnostics_noalloc", self._jp(), int(bool(gauss)),
                  out.data_ptr(), _stream())
        o = out.cpu().tolist()
        return {"kinetic": o[0], "ex": o[1], "ey": o[2], "ez": o[3], "bx": o[4], "by": o[5],
                "bz": o[6], "gauss_norm": o[7], "rho_norm": o[8], "field": sum(o[1:7]),
                "total": o[0] + sum(o[1:7])}

    def slow_path_count(self):
        return int(self.counters[0].item())

    def error_flag(self):
        return int(self.counters[1].item())

    def deferred_count(self):
        """Particle-steps the FP32 particle kernel deferred to its second,
        class-bucketed pass since the simulation was created."""
        return int(self.counters[2].item())

    def particles(self):
        """PICSAR-style FP64 particle arrays (sorted by id when ids are tracked)."""
        N, dev = self.np, self.device
        out = {c: torch.empty(N, dtype=torch.float64, device=dev)
               for c in ("x", "y", "z", "ux", "uy", "uz", "gaminv", "w")}
        if self.track_ids and getattr(self, "_ids_dense", False):
            # ids are the positions of the id order: one pass writes every
            # column in that order, reading the current device descriptor
            _lib.call("pxrb_tiled_store_particles_by_id", self.job_dev.data_ptr(), N, self.prec,
                      *[out[c].data_ptr() for c in ("x", "y", "z", "ux", "uy", "uz", "gaminv",
                                                    "w")], _stream())
            out["id"] = torch.arange(N, dtype=torch.int32, device=dev)
            return out
        self._pull_job()
        _lib.call("pxrb_tiled_store_particles", self._jp(),
                  *[out[c].data_ptr() for c in ("x", "y", "z", "ux", "uy", "uz", "gaminv", "w")],
                  _stream())
        if self.track_ids and self.job.pid:
            C_ptr = self.job.pid
            cur = self.pid if self.pid.data_ptr() == C_ptr else self.pid_b
            order = torch.argsort(cur.long())
            out = {k: v[order] for k, v in out.items()}
            out["id"] = cur[order]
        return out

    def tensors(self):
        """Every device tensor this simulation owns (for stream bookkeeping
        when it was built on another stream than the one that steps it)."""
        out = []
        for v in vars(self).values():
            if torch.is_tensor(v):
                out.append(v)
            elif isinstance(v, (list, tuple)):
                out.extend(t for t in v if torch.is_tensor(t))
            elif isinstance(v, dict):
                out.extend(t for t in v.values() if torch.is_tensor(t))
        return [t for t in out if t.is_cuda]

    def state_bytes(self):
        """Device bytes held by this simulation."""
        tot = 0
        for t in self.E + self.B + self.J + [self.rho, self.tile_off, self.tile_cnt,
                                             self.ke_tile, self.tile_stats]:
            tot += t.numel() * t.element_size()
        if self.np:
            tot += sum(t.numel() * t.element_size() for t in self.parts.values()) * 2
            tot += self.cell.numel() * 12
        return tot


def smoke_check():
    """One FP64 tiled step vs the plain FP64 path on the same state (used by
    the package smoke test on cuda:0)."""
    import numpy as np
    from .init import thermal_plasma
    from .picsar import PicsarModule
    n = (16, 16, 16)
    st = thermal_plasma(n, 2, 0.05, seed=3, shuffle=True)
    m = PicsarModule(*n, nguards=3, nox=2)
    m.add_species("e", -1.0, 1.0, st.x, st.y, st.z, st.ux, st.uy, st.uz, st.w)
    m.step(1)
    t = TiledSim(n, order=2, precision="fp64", config=TiledConfig(tile=(8, 8, 8)))
    t.load_state(st.to(device="cuda"))
    t.step(1, keep_j=True)
    torch.cuda.synchronize()
    for name in ("jx", "ey", "bz"):
        a = t.export_field(name, 3).cpu().numpy()
        b = getattr(m, name).cpu().numpy()
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
        assert err <= 1e-12, (name, err)
