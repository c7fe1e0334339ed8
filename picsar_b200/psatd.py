"""Spectral (PSATD) field solver of one periodic domain on the GPU.

The reference's pseudo-spectral analytical time-domain push with a local
FFT (src/field_solvers/Maxwell/maxwell_solver_manager.F90:574-642,
GPSTD_solver/): the fields of the FFT region (nodes -g .. n+g-1 of each
guarded array, n + 2g points per axis, copy_field_forward,
init_kspace_3D.F90:1559-1649) are transformed with real-to-complex FFTs
(cuFFT), advanced by one analytical step per Fourier mode
(``pxrb_psatd_push``, one CUDA kernel) and transformed back (unnormalised,
the 1/N scaling sits in the coefficients as in the reference).

The k-vectors follow compute_k_1d (init_kspace_3D.F90:751-812): finite-order
stencils with the weights of FD_weights_hvincenti (:1515-1537), staggered by
default; order 0 takes fftfreq (:830-865), which scales the integer
frequencies by pi / (2 n d).  The operators follow init_kspace (:341-541),
including the special values of the mode k = 0.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib

_lib.register({"pxrb_psatd_push": "i i i " + "p " * 23 + "d d d d d s"})


def _logfactorial(n):
    if n == 0:
        return 0.0
    s = math.log(1.0 * n)
    for k in range(2, n):
        s += math.log(1.0 * k)
    return s


def fd_weights_hvincenti(p, staggered=True):
    """The p/2 weights of the order-p (staggered or centred) stencil."""
    w = np.zeros(p // 2)
    for l in range(1, p // 2 + 1):
        if staggered:
            num = math.log(16.0) * (1.0 - p / 2.0) + _logfactorial(p - 1) * 2.0
            den = (math.log(2.0 * l - 1.0) * 2.0 + _logfactorial(p // 2 + l - 1) +
                   _logfactorial(p // 2 - l) + 2.0 * _logfactorial(p // 2 - 1))
        else:
            num = _logfactorial(p // 2) * 2.0
            den = _logfactorial(p // 2 + l) + _logfactorial(p // 2 - l) + math.log(1.0 * l)
        w[l - 1] = (-1.0) ** (l + 1) * math.exp(num - den)
    return w


def k_vectors(nfft, norder, d, staggered=True):
    """(centred, forward, backward) complex k-vectors of one axis."""
    j = np.arange(nfft, dtype=np.float64)
    hi = np.arange(1, nfft + 1) > nfft // 2 + 1
    ones = np.where(hi, -j, j)
    onesp = np.where(hi, nfft + j, j)
    k = np.zeros(nfft)
    if norder != 0:
        w = fd_weights_hvincenti(norder, staggered)
        for i in range(1, norder // 2 + 1):
            if staggered:
                k = k + 2.0 / d * w[i - 1] * np.sin((i * 2.0 - 1.0) * math.pi * ones / nfft)
            else:
                k = k + 2.0 / d * w[i - 1] * np.sin(i * 2.0 * math.pi * onesp / nfft)
    else:
        f = np.concatenate([np.arange(0, (nfft + 1) // 2), np.arange(-(nfft // 2), 0)])
        k = f / (d * nfft) / 2.0 * math.pi
    k = k.astype(np.complex128)
    if staggered:
        return k, k * np.exp(-1j * math.pi * onesp / nfft), k * np.exp(1j * math.pi * onesp / nfft)
    return k, k.copy(), k.copy()


class PsatdSolver:
    """PSATD push of a periodic domain of n cells per axis with g guard
    cells per axis, cell sizes d, time step dt."""

    def __init__(self, n, g, d, dt, norder=(2, 2, 2), staggered=True, clight=1.0, eps0=1.0,
                 mu0=1.0, device="cuda"):
        self.n, self.g = tuple(int(v) for v in n), tuple(int(v) for v in g)
        self.N = tuple(self.n[a] + 2 * self.g[a] for a in range(3))
        self.dt, self.c, self.eps0, self.mu0 = float(dt), float(clight), float(eps0), float(mu0)
        self.device = torch.device(device)
        N, c = self.N, self.c
        kx = k_vectors(N[0], norder[0], d[0], staggered)
        ky = k_vectors(N[1], norder[1], d[1], staggered)
        kz = k_vectors(N[2], norder[2], d[2], staggered)
        h = N[0] // 2 + 1
        kx = tuple(v[:h] for v in kx)
        dev = self.device
        cplx = lambda v: torch.view_as_real(torch.from_numpy(np.ascontiguousarray(v))).to(
            dev).contiguous()
        self.kxf, self.kxb = cplx(kx[1]), cplx(kx[2])
        self.kyf, self.kyb = cplx(ky[1]), cplx(ky[2])
        self.kzf, self.kzb = cplx(kz[1]), cplx(kz[2])
        a2 = lambda v: torch.from_numpy(np.abs(v) ** 2).to(dev)
        self.kxc2, self.kyc2, self.kzc2 = a2(kx[0]), a2(ky[0]), a2(kz[0])
        # per-mode operators, modes (z, y, x) with x fastest
        k10 = torch.sqrt(self.kzc2[:, None, None] + self.kyc2[None, :, None] +
                         self.kxc2[None, None, :])
        t = dt * c * k10
        sinc = torch.where(t != 0.0, torch.sin(t) / torch.where(t != 0.0, t, 1.0),
                           torch.ones_like(t))
        self.at1 = (c * dt * sinc).contiguous()
        self.at2 = torch.cos(t).contiguous()
        switch = bool(k10[0, 0, 0] == 0.0)
        k10s = k10.clone()
        if switch:
            k10s[0, 0, 0] = 1.0
        at3 = (1.0 - self.at2) / (k10s * k10s)
        if switch:
            at3[0, 0, 0] = (c * dt) ** 2 / 2.0
        self.at3 = at3.contiguous()
        self.norm = 1.0 / (N[0] * N[1] * N[2])
        self.nk = (h, N[1], N[2])
        self.launches = 0

    def _region(self, a):
        N = self.N
        return a[:N[0], :N[1], :N[2]].permute(2, 1, 0)

    def push(self, ex, ey, ez, bx, by, bz, jx, jy, jz, rho, rhoold, stream=None):
        """One PSATD step of the guarded FP64 Fortran-layout arrays (E, B
        updated in place over nodes -g .. n+g-1)."""
        s = torch.cuda.current_stream(self.device).cuda_stream if stream is None else stream
        fwd = lambda a: torch.fft.rfftn(self._region(a), dim=(0, 1, 2)).contiguous()
        F = [fwd(a) for a in (ex, ey, ez, bx, by, bz, jx, jy, jz, rho, rhoold)]
        _lib.call("pxrb_psatd_push", self.nk[0], self.nk[1], self.nk[2],
                  *[f.data_ptr() for f in F],
                  self.kxf.data_ptr(), self.kxb.data_ptr(), self.kyf.data_ptr(),
                  self.kyb.data_ptr(), self.kzf.data_ptr(), self.kzb.data_ptr(),
                  self.kxc2.data_ptr(), self.kyc2.data_ptr(), self.kzc2.data_ptr(),
                  self.at1.data_ptr(), self.at2.data_ptr(), self.at3.data_ptr(),
                  self.c, self.eps0, self.mu0, self.dt, self.norm, s)
        self.launches += 1
        N = self.N
        for a, f in zip((ex, ey, ez, bx, by, bz), F[:6]):
            self._region(a).copy_(torch.fft.irfftn(f, s=(N[2], N[1], N[0]), dim=(0, 1, 2),
                                                   norm="forward"))
