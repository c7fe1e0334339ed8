"""CPU restatement of the reference's PSATD field push (test infrastructure:
only tests may import it; the product path is picsar_b200.psatd).

The single-domain form of the reference's spectral solver with a local FFT
(fftw_with_mpi = .FALSE., the non-LIBRARY build), in NumPy (complex128):

  * k-vectors: compute_k_1d and fftfreq
    (src/field_solvers/Maxwell/GPSTD_solver/init_kspace_3D.F90:751-865), with
    the finite-order weights FD_weights_hvincenti (:1515-1537);
  * the operators |k|, at_op(1..4) (init_kspace, :341-541);
  * the coefficient blocks of compute_cc_mat_merged_fields (:1316-1495),
    scaled by 1 / (nfftx nffty nfftz) (init_gpstd, :1025-1040);
  * push_psaotd_ebfielfs_3d (fourier_psaotd.F90:1538-1643);
  * the FFT region: nodes -g .. n+g-1 of each guarded array, FFT extent
    n + 2g per axis (copy_field_forward / backward, init_kspace_3D.F90:
    1559-1721; select_case_dims_local, :185-244), r2c forward and an
    unnormalised c2r backward (FFTW's conventions).

Quirks kept: fftfreq scales the integer frequencies by pi / (2 n d) (the
expression divides by 2 and then multiplies by pi), and the mode k = 0 takes
the special values of init_kspace and compute_cc_mat_merged_fields.
"""
import math

import numpy as np


def logfactorial(n):
    """init_kspace_3D.F90:66-82 (sum of logs, 0 for n = 0)."""
    if n == 0:
        return 0.0
    s = math.log(1.0 * n)
    for k in range(2, n):
        s = s + math.log(1.0 * k)
    return s


def fd_weights_hvincenti(p, staggered):
    """init_kspace_3D.F90:1515-1537: p/2 weights of the order-p stencil."""
    w = np.zeros(p // 2)
    for i in range(1, p // 2 + 1):
        l = i
        if staggered:
            lognumer = math.log(16.0) * (1.0 - p / 2.0) + logfactorial(p - 1) * 2.0
            logdenom = (math.log(2.0 * l - 1.0) * 2.0 + logfactorial(p // 2 + l - 1) +
                        logfactorial(p // 2 - l) + 2.0 * logfactorial(p // 2 - 1))
        else:
            lognumer = logfactorial(p // 2) * 2.0
            logdenom = logfactorial(p // 2 + l) + logfactorial(p // 2 - l) + math.log(1.0 * l)
        w[i - 1] = (-1.0) ** (l + 1) * math.exp(lognumer - logdenom)
    return w


def fftfreq(n, d):
    """init_kspace_3D.F90:830-865 (integer frequencies * pi / (2 n d))."""
    k = np.zeros(n, dtype=np.complex128)
    if n % 2 == 0:
        for i in range(1, n // 2):
            k[i] = k[i - 1] + 1.0
        k[n // 2] = -(n // 2)
        for i in range(n // 2 + 1, n):
            k[i] = k[i - 1] + 1.0
    else:
        for i in range(1, (n - 1) // 2 + 1):
            k[i] = k[i - 1] + 1.0
        k[(n - 1) // 2 + 1] = -((n - 1) // 2)
        for i in range((n - 1) // 2 + 2, n):
            k[i] = k[i - 1] + 1.0
    return k / (d * n) / 2.0 * math.pi


def compute_k_1d(nfft, norder, d, stg):
    """init_kspace_3D.F90:751-812: (k, k_forward, k_backward)."""
    j = np.arange(1, nfft + 1)
    ones = (j - 1.0).astype(np.complex128)
    onesp = (j - 1.0).astype(np.complex128)
    hi = j > nfft // 2 + 1
    ones[hi] = -ones[hi]
    onesp[hi] = nfft + onesp[hi]
    kvec = np.zeros(nfft, dtype=np.complex128)
    if norder != 0:
        fd = fd_weights_hvincenti(norder, stg)
        for i in range(1, norder // 2 + 1):
            if stg:
                kvec = kvec + 2.0 / d * fd[i - 1] * np.sin((i * 2.0 - 1.0) * math.pi * ones / nfft)
            else:
                kvec = kvec + 2.0 / d * fd[i - 1] * np.sin(i * 2.0 * math.pi * onesp / nfft)
    else:
        kvec = fftfreq(nfft, d)
    if stg:
        kf = kvec * np.exp(-1j * math.pi * onesp / nfft)
        kb = kvec * np.exp(1j * math.pi * onesp / nfft)
    else:
        kf = kvec.copy()
        kb = kvec.copy()
    return kvec, kf, kb


def sinc(x):
    out = np.ones_like(x)
    nz = x != 0.0
    out[nz] = np.sin(x[nz]) / x[nz]
    return out


class Psatd:
    """The reference's PSATD push on a guarded periodic domain of n cells
    per axis with g guards per axis (FFT extent n + 2g)."""

    def __init__(self, n, g, d, dt, norder=(2, 2, 2), stg=True, clight=1.0, eps0=1.0,
                 mu0=1.0):
        self.n, self.g = tuple(n), tuple(g)
        N = tuple(n[a] + 2 * g[a] for a in range(3))
        self.N = N
        c = clight
        kxc, kxf, kxb = compute_k_1d(N[0], norder[0], d[0], stg)
        kyc, kyf, kyb = compute_k_1d(N[1], norder[1], d[1], stg)
        kzc, kzf, kzb = compute_k_1d(N[2], norder[2], d[2], stg)
        h = N[0] // 2 + 1
        kxc, kxf, kxb = kxc[:h], kxf[:h], kxb[:h]
        # arrays indexed (ix, iy, iz) like the Fortran blocks
        X = lambda v: v[:, None, None] * np.ones((1, N[1], N[2]))
        Y = lambda v: v[None, :, None] * np.ones((h, 1, N[2]))
        Z = lambda v: v[None, None, :] * np.ones((h, N[1], 1))
        kv = [None, X(kxf), X(kxb), X(kxc), Y(kyf), Y(kyb), Y(kyc), Z(kzf), Z(kzb), Z(kzc)]
        k10 = np.sqrt(np.abs(kv[9]) ** 2 + np.abs(kv[6]) ** 2 + np.abs(kv[3]) ** 2).astype(
            np.complex128)
        temp = dt * c * k10.real
        at1 = (c * dt * sinc(temp)).astype(np.complex128)
        at2 = np.cos(temp).astype(np.complex128)
        switch = abs(k10[0, 0, 0]) == 0.0
        if switch:
            k10[0, 0, 0] = 1.0
        at3 = (1.0 - at2) / k10 ** 2
        if switch:
            at3[0, 0, 0] = (c * dt) ** 2 / 2.0
            k10[0, 0, 0] = 0.0
        ii = 1j
        cc = {}
        cc[(1, 5)] = -ii * kv[7] * c * at1
        cc[(1, 6)] = ii * kv[4] * c * at1
        cc[(2, 4)] = ii * kv[7] * c * at1
        cc[(2, 6)] = -ii * kv[1] * c * at1
        cc[(3, 4)] = -ii * kv[4] * c * at1
        cc[(3, 5)] = ii * kv[1] * c * at1
        cc[(4, 2)] = ii * kv[8] / c * at1
        cc[(4, 3)] = -ii * kv[5] / c * at1
        cc[(5, 1)] = -ii * kv[8] / c * at1
        cc[(5, 3)] = ii * kv[2] / c * at1
        cc[(6, 1)] = ii * kv[5] / c * at1
        cc[(6, 2)] = -ii * kv[2] / c * at1
        for i in range(1, 7):
            cc[(i, i)] = at2.copy()
        for i in range(1, 4):
            cc[(i, i + 6)] = (-1.0) * c * mu0 * at1
        cc[(4, 8)] = -mu0 * ii * kv[8] * at3
        cc[(4, 9)] = -mu0 * (-ii) * kv[5] * at3
        cc[(5, 7)] = -mu0 * (-ii) * kv[8] * at3
        cc[(5, 9)] = -mu0 * ii * kv[2] * at3
        cc[(6, 7)] = -mu0 * ii * kv[5] * at3
        cc[(6, 8)] = -mu0 * (-ii) * kv[2] * at3
        if switch:
            k10[0, 0, 0] = 1.0
        for i in range(1, 4):
            v = 1j * (at2 - 1.0 / (c * dt) * at1) / k10 ** 2
            v = v * kv[3 * i - 1]
            if switch:
                v[0, 0, 0] = -1.0 / 3.0 * 1j * (c * dt) ** 2
            cc[(i, 10)] = 1.0 / eps0 * v
        for i in range(1, 4):
            v = 1j * (1.0 / (c * dt) * at1 - 1.0) / k10 ** 2
            v = v * kv[3 * i - 1]
            if switch:
                v[0, 0, 0] = -1.0 / 6.0 * 1j * (c * dt) ** 2
            cc[(i, 11)] = 1.0 / eps0 * v
        if switch:
            k10[0, 0, 0] = 0.0
        norm = 1.0 / (N[0] * N[1] * N[2])
        self.cc = {k: norm * v for k, v in cc.items()}
        self.kv, self.k10, self.at = kv, k10, (at1, at2, at3)

    def push_spectra(self, F):
        """push_psaotd_ebfielfs_3d on spectra F (dict ex..bz, jx..jz, rho,
        rhoold of complex (nkx, nky, nkz) arrays): new ex..bz."""
        c = self.cc
        ex, ey, ez, bx, by, bz = (F[k] for k in ("ex", "ey", "ez", "bx", "by", "bz"))
        jx, jy, jz, rho, rhoo = (F[k] for k in ("jx", "jy", "jz", "rho", "rhoold"))
        out = {}
        out["bx"] = c[(4, 4)] * bx + c[(4, 2)] * ey + c[(4, 3)] * ez + c[(4, 8)] * jy + c[(4, 9)] * jz
        out["by"] = c[(5, 5)] * by + c[(5, 1)] * ex + c[(5, 3)] * ez + c[(5, 7)] * jx + c[(5, 9)] * jz
        out["bz"] = c[(6, 6)] * bz + c[(6, 1)] * ex + c[(6, 2)] * ey + c[(6, 7)] * jx + c[(6, 8)] * jy
        out["ex"] = (c[(1, 1)] * ex + c[(1, 5)] * by + c[(1, 6)] * bz + c[(1, 7)] * jx +
                     c[(1, 11)] * rho + c[(1, 10)] * rhoo)
        out["ey"] = (c[(2, 2)] * ey + c[(2, 4)] * bx + c[(2, 6)] * bz + c[(2, 8)] * jy +
                     c[(2, 11)] * rho + c[(2, 10)] * rhoo)
        out["ez"] = (c[(3, 3)] * ez + c[(3, 4)] * bx + c[(3, 5)] * by + c[(3, 9)] * jz +
                     c[(3, 11)] * rho + c[(3, 10)] * rhoo)
        return out

    def push(self, grids):
        """push_psatd_ebfield (local FFT) on guarded Fortran-layout arrays
        (dict of ex..bz, jx..jz, rho, rhoold with extent n+1+2g per axis):
        ex..bz updated in place over nodes -g .. n+g-1."""
        N = self.N
        reg = (slice(0, N[0]), slice(0, N[1]), slice(0, N[2]))
        F = {k: np.fft.rfftn(np.asarray(a)[reg].transpose(2, 1, 0)).transpose(2, 1, 0)
             for k, a in grids.items()}
        new = self.push_spectra(F)
        for k, v in new.items():
            r = np.fft.irfftn(v.transpose(2, 1, 0), s=(N[2], N[1], N[0]), axes=(0, 1, 2),
                              norm="forward")
            grids[k][reg] = r.transpose(2, 1, 0)
