"""FP64 NumPy restatement of the reference's Gamma-point hybrid exchange.

Test infrastructure (see ``oracle/__init__.py``).  Follows:
  * KohnSham::InitializeEXX       src/SCF/hamiltonian.cpp:3454-3551 (R2C half
    spectrum, divergence types 0 and 1, optional screening mu)
  * KohnSham::SetPhiEXX           src/SCF/hamiltonian.cpp:3554-3641 (real space:
    phi = sqrt(N_c / vol) psi)
  * Spinor::AddMultSpinorEXX      src/SCF/spinor.cpp:682-781 (R2C with vol/N,
    multiply by the kernel, C2R with 1/vol, times phi, times -alpha f_j)
  * KohnSham::CalculateVexxACE    src/SCF/hamiltonian.cpp:3686-3818
  * ACE apply in MultSpinor       src/SCF/hamiltonian.cpp:3135-3218
  * KohnSham::CalculateEXXEnergy  src/SCF/hamiltonian.cpp:3936-4192
"""
from __future__ import annotations

import math

import numpy as np

from . import pw


def exx_kernel_r2c(dm: pw.Domain, ecut: float, mu: float = 0.0, div_type: int = 1):
    """(exxgkkR2C on the R2C half grid, exxDiv); hamiltonian.cpp:3454-3551."""
    eps_div = 1e-8
    alpha = 10.0 / (ecut * 2.0)
    div = 0.0
    if div_type == 1:
        gf = pw.gvec_full(dm)
        q = np.sum(gf * gf, axis=-1).ravel()            # gkk * 2 over the whole grid
        sel = q > eps_div
        if mu > 0.0:
            div = np.sum(np.exp(-alpha * q[sel]) / q[sel] * (1.0 - np.exp(-q[sel] / (4 * mu * mu))))
            div += 1.0 / (4 * mu * mu)
        else:
            div = np.sum(np.exp(-alpha * q[sel]) / q[sel])
            div -= alpha
        div *= 4.0 * math.pi
        if mu > 0.0:
            aa = 1.0 / math.sqrt(alpha * math.pi) - 1.0 / math.sqrt(math.pi * (alpha + 1.0 / (4 * mu * mu)))
        else:
            aa = 1.0 / math.sqrt(alpha * math.pi)
        div -= dm.vol * aa
    elif div_type != 0:
        raise ValueError("divergence types 0 and 1")
    g = pw.gvec_r2c(dm)
    q = np.sum(g * g, axis=-1)
    k = np.empty_like(q)
    big = q > eps_div
    qs = np.where(big, q, 1.0)
    if mu > 0.0:
        k = np.where(big, 4 * math.pi / qs * (1.0 - np.exp(-qs / (4 * mu * mu))), -div + math.pi / (mu * mu))
    else:
        k = np.where(big, 4 * math.pi / qs, -div)
    return k, div


def set_phi(dm: pw.Domain, psi: np.ndarray):
    """phi = sqrt(N_c / vol) psi (real-space branch of SetPhiEXX)."""
    return psi * math.sqrt(dm.ntot / dm.vol)


def add_mult_spinor_exx(dm: pw.Domain, psi: np.ndarray, phi: np.ndarray, kern_r2c: np.ndarray, frac: float,
                        occ: np.ndarray, a3: np.ndarray | None = None):
    """a3 += V_x psi; psi (nb, N_c), phi (nphi, N_c), occ per phi state."""
    n0, n1, n2 = dm.numGrid
    nb = psi.shape[0]
    if a3 is None:
        a3 = np.zeros_like(psi)
    for j in range(phi.shape[0]):
        if occ[j] == 0.0:
            # the reference still runs the transforms; the product is zero
            continue
        rho = psi * phi[j][None, :]
        X = pw.r2c(rho.reshape(nb, n2, n1, n0), dm) * kern_r2c[None]
        v = pw.c2r(X, dm).reshape(nb, -1)
        a3 += -frac * occ[j] * v * phi[j][None, :]
    return a3


def ace_build(dm, psi, phi, kern_r2c, frac, occ):
    """xi with V_x ~ -xi xi^T on span(psi) (CalculateVexxACE)."""
    W = add_mult_spinor_exx(dm, psi, phi, kern_r2c, frac, occ)
    M = -(psi @ W.T)
    M = 0.5 * (M + M.T)
    L = np.linalg.cholesky(M)
    xi = np.linalg.solve(L, W)          # rows: (W^T L^-T)^T = L^-1 W
    return xi


def ace_apply(xi, psi, a3=None):
    if a3 is None:
        a3 = np.zeros_like(psi)
    a3 -= (psi @ xi.T) @ xi
    return a3


def exx_energy(vxpsi: np.ndarray, psi: np.ndarray, occ: np.ndarray, numSpin: int = 2):
    return float(np.sum(occ * np.einsum("bi,bi->b", vxpsi, psi))) * numSpin / 2.0


def pair_convolution_direct(dm: pw.Domain, rho: np.ndarray, kern_r2c: np.ndarray):
    """(1/N_c) sum_G v(G) rho(G) e^{iGr} by explicit DFT sums (no FFT), for
    the small-grid known-answer test; rho real on the coarse grid."""
    n0, n1, n2 = dm.numGrid
    N = dm.ntot
    # full-spectrum kernel from the R2C half (v is even in G)
    k0 = pw.kgrid(n0)
    kz, ky, kx = np.meshgrid(np.arange(n2), np.arange(n1), np.arange(n0), indexing="ij")
    xh = np.where(kx <= n0 // 2, kx, (n0 - kx) % n0)
    yh = np.where(kx <= n0 // 2, ky, (n1 - ky) % n1)
    zh = np.where(kx <= n0 // 2, kz, (n2 - kz) % n2)
    vfull = kern_r2c[zh, yh, xh].ravel()
    del k0
    z, y, x = np.meshgrid(np.arange(n2), np.arange(n1), np.arange(n0), indexing="ij")
    ph = (np.outer(kx.ravel(), x.ravel()) / n0 + np.outer(ky.ravel(), y.ravel()) / n1 +
          np.outer(kz.ravel(), z.ravel()) / n2)
    F = np.exp(-2j * math.pi * ph)             # F[G, r]
    rhoG = F @ rho
    out = (F.conj().T @ (vfull * rhoG)) / N
    return out.real
