"""Seeded synthetic initial states for the benchmark and test workloads.

The reference mini-app's own loader (src/parallelization/tiling/tiling.F90:876-1003)
places particles on a per-cell diagonal (pdistr=1) or uniformly over the whole
domain (pdistr=2) and draws a spherical-angle velocity; it cannot produce the
workloads used here.  These generators build the states directly: positions
uniform inside each cell, momentum u = gamma*beta Gaussian per component, one
seed for everything.  They run on any torch device (CPU for the oracle and
the host-side end-to-end path, CUDA for device-resident runs).
"""
from __future__ import annotations

from dataclasses import dataclass

import math
import torch


@dataclass
class PlasmaState:
    """Particles of one species as flat float64/float32 tensors (SoA)."""
    x: torch.Tensor
    y: torch.Tensor
    z: torch.Tensor
    ux: torch.Tensor
    uy: torch.Tensor
    uz: torch.Tensor
    w: torch.Tensor

    @property
    def np(self) -> int:
        return int(self.x.numel())

    def to(self, device=None, dtype=None):
        return PlasmaState(*[getattr(self, c).to(device=device, dtype=dtype)
                             for c in ("x", "y", "z", "ux", "uy", "uz", "w")])

    def numpy(self):
        return {c: getattr(self, c).detach().cpu().double().numpy()
                for c in ("x", "y", "z", "ux", "uy", "uz", "w")}


def cfl_dt(d=(1.0, 1.0, 1.0), dtcoef=0.95, clight=1.0) -> float:
    """dt = dtcoef / (c sqrt(1/dx^2 + 1/dy^2 + 1/dz^2)) (src/submain.F90:581)."""
    return dtcoef / (clight * math.sqrt(1.0 / d[0] ** 2 + 1.0 / d[1] ** 2 + 1.0 / d[2] ** 2))


def thermal_plasma(n, ppc, sigma, seed, n0=1.0, d=(1.0, 1.0, 1.0), xmin=(0.0, 0.0, 0.0),
                   drift=(0.0, 0.0, 0.0), device="cpu", dtype=torch.float64,
                   shuffle=False) -> PlasmaState:
    """Homogeneous thermal plasma: ``ppc`` particles uniform in every cell,
    u ~ drift + N(0, sigma^2) per component, weight n0*dV/ppc."""
    nx, ny, nz = n
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    ncell = nx * ny * nz
    N = ncell * ppc
    cell = torch.arange(ncell, device=device, dtype=torch.int64).repeat_interleave(ppc)
    cx = cell % nx
    cy = (cell // nx) % ny
    cz = cell // (nx * ny)
    r = torch.rand((3, N), generator=g, device=device, dtype=torch.float64)
    x = xmin[0] + (cx.double() + r[0]) * d[0]
    y = xmin[1] + (cy.double() + r[1]) * d[1]
    z = xmin[2] + (cz.double() + r[2]) * d[2]
    u = torch.randn((3, N), generator=g, device=device, dtype=torch.float64) * sigma
    ux, uy, uz = u[0] + drift[0], u[1] + drift[1], u[2] + drift[2]
    w = torch.full((N,), n0 * d[0] * d[1] * d[2] / ppc, device=device, dtype=torch.float64)
    if shuffle:
        perm = torch.randperm(N, generator=g, device=device)
        x, y, z, ux, uy, uz = (a[perm] for a in (x, y, z, ux, uy, uz))
    st = PlasmaState(x, y, z, ux, uy, uz, w)
    return st.to(dtype=dtype) if dtype != torch.float64 else st


def two_stream_ramp(n, ppc, u_drift, sigma, seed, ramp_cells=256, d=(1.0, 1.0, 1.0),
                    device="cpu", dtype=torch.float64) -> PlasmaState:
    """Uneven-density workload: density ramps linearly from 0 to n0=1 over
    the first ``ramp_cells`` cells along x, flat afterwards; ``ppc`` particles
    per cell at n0 (fewer on the ramp, rounded per cell), two counter-drifting
    electron beams u_x = +-u_drift with thermal spread sigma.  Weights are
    n0*dV/ppc so the density follows the particle count."""
    nx, ny, nz = n
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    ix = torch.arange(nx, device=device, dtype=torch.float64)
    dens = torch.clamp((ix + 0.5) / ramp_cells, max=1.0)
    cnt_x = torch.round(dens * ppc).to(torch.int64)          # per cell column along x
    cnt = cnt_x.repeat(ny * nz)                                # cell order x fastest
    ncell = nx * ny * nz
    cell = torch.arange(ncell, device=device, dtype=torch.int64).repeat_interleave(cnt)
    N = int(cell.numel())
    cx = cell % nx
    cy = (cell // nx) % ny
    cz = cell // (nx * ny)
    r = torch.rand((3, N), generator=g, device=device, dtype=torch.float64)
    x = (cx.double() + r[0]) * d[0]
    y = (cy.double() + r[1]) * d[1]
    z = (cz.double() + r[2]) * d[2]
    u = torch.randn((3, N), generator=g, device=device, dtype=torch.float64) * sigma
    sign = torch.where(torch.rand(N, generator=g, device=device) < 0.5, -1.0, 1.0).to(
        device=device, dtype=torch.float64)
    ux = u[0] + sign * u_drift
    w = torch.full((N,), d[0] * d[1] * d[2] / ppc, device=device, dtype=torch.float64)
    st = PlasmaState(x, y, z, ux, u[1], u[2], w)
    return st.to(dtype=dtype) if dtype != torch.float64 else st
