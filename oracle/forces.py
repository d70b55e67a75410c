"""FP64 NumPy restatement of KohnSham::CalculateForce (real-space path).

Test infrastructure (see ``oracle/__init__.py``).  Follows
src/SCF/hamiltonian.cpp:2670-3056:
  * local part, pseudocharge formulation (:2716-2800):
      dV_H/dx_d = IFFT( rho_tot(G) * 2 pi / gkk * i G_d ),  gkk = 0 -> 0,
      F_a,d += sum_{i in ball_a} rho_ps,a(r_i) * dV_H/dx_d(r_i) * vol / N_fine
  * nonlocal part, "Method 4" (:2907-3006): per band, psi_F and d_d psi_F on
    the fine grid (C2C coarse FFT, idxFineGrid placement, C2C fine IFFT, real
    part, factor sqrt(N_c/N_fine)), then per projector
      res(VAL) = sum beta psi_F sqrt(w), res(D) = sum beta d psi_F sqrt(w),
      F_a,d -= 2 f gamma res(VAL) res(D) numSpin.
"""
from __future__ import annotations

import math

import numpy as np

from . import pw


def _placement(dm: pw.Domain):
    """idxFineGrid: coarse full-spectrum index -> fine index (fourier.cpp:291-311)."""
    n0, n1, n2 = dm.numGrid
    N0, N1, N2 = dm.numGridFine
    k, j, i = np.meshgrid(np.arange(n2), np.arange(n1), np.arange(n0), indexing="ij")
    iF = np.where(i <= n0 // 2, i, N0 - n0 + i)
    jF = np.where(j <= n1 // 2, j, N1 - n1 + j)
    kF = np.where(k <= n2 // 2, k, N2 - n2 + k)
    return (iF + N0 * (jF + N1 * kF)).ravel()


def local_force(dm: pw.Domain, rho: np.ndarray, rho_ps: np.ndarray, ps_sets):
    """ps_sets: list of (idx, val) pseudocharge sparse vectors per atom."""
    N0, N1, N2 = dm.numGridFine
    X = np.fft.fftn((rho - rho_ps).reshape(N2, N1, N0)) * (dm.vol / dm.ntotFine)
    g = pw.gvec_full(dm, fine=True)
    gkk = 0.5 * np.sum(g * g, axis=-1)
    fac = np.where(gkk == 0, 0.0, 2 * math.pi / np.where(gkk == 0, 1.0, gkk))
    dv = []
    for d in range(3):
        Y = X * fac * (1j * g[..., d])
        dv.append((np.fft.ifftn(Y) * (dm.ntotFine / dm.vol)).real.ravel())
    w = dm.vol / dm.ntotFine
    F = np.zeros((len(ps_sets), 3))
    for a, (idx, val) in enumerate(ps_sets):
        for d in range(3):
            F[a, d] = np.sum(val * dv[d][idx]) * w
    return F


def nonlocal_force(T: pw.HamTables, psi: np.ndarray, occ: np.ndarray, numSpin: int = 2):
    dm = T.dm
    n0, n1, n2 = dm.numGrid
    N0, N1, N2 = dm.numGridFine
    place = _placement(dm)
    g = pw.gvec_full(dm, fine=True).reshape(-1, 3)
    fac = math.sqrt(dm.ntot / dm.ntotFine)
    w = dm.vol / dm.ntotFine
    sw = math.sqrt(w)
    F = np.zeros((len(T.pseudo), 3))
    for b in range(psi.shape[0]):
        X = np.fft.fftn(psi[b].reshape(n2, n1, n0)).ravel() * (dm.vol / dm.ntot)
        Y = np.zeros(dm.ntotFine, complex)
        Y[place] = X
        pf = (np.fft.ifftn(Y.reshape(N2, N1, N0)).ravel() * (dm.ntotFine / dm.vol)).real * fac
        dps = [(np.fft.ifftn((Y * 1j * g[:, d]).reshape(N2, N1, N0)).ravel() * (dm.ntotFine / dm.vol)).real * fac
               for d in range(3)]
        for a, app in enumerate(T.pseudo):
            for pp in app:
                v = pp.val[:, 0]
                rv = np.sum(v * pf[pp.idx]) * sw
                for d in range(3):
                    rd = np.sum(v * dps[d][pp.idx]) * sw
                    F[a, d] += -2.0 * occ[b] * pp.wgt * rv * rd * numSpin
    return F
