"""FP64 NumPy restatement of the reference's Gamma-point SCF around H*psi.

Test infrastructure (see ``oracle/__init__.py``).  Follows:
  * KohnSham::CalculateDensity    src/SCF/hamiltonian.cpp:2455-2627
  * KohnSham::CalculateHartree    src/SCF/hamiltonian.cpp:1990-2026
  * KohnSham::CalculateXC         src/SCF/hamiltonian.cpp:1242-1308 (LDA Teter93; the
    reference calls libxc XC_LDA_XC_TETER93, restated here from Goedecker, Teter,
    Hutter, PRB 54, 1703 (1996); parity at the libxc boundary is unpinned)
  * KohnSham::CalculateVtot       src/SCF/hamiltonian.cpp:2029-2069 (Use_VLocal 0)
  * SCF::CalculateOccupationRate  src/SCF/scf.cpp:1748-1830, wgauss/getEntropy
    src/utility.cpp:4404-4444
  * SCF::CalculateEnergy / CalculateHarrisEnergy  src/SCF/scf.cpp:1834-2140
  * SCF::andersonMix              src/SCF/scf.cpp:2299-2365
  * SCF::Iterate / InnerSolve     src/SCF/scf.cpp:372-591, 1261-1589
  * initial density from the pseudocharge  src/SCF/scf.cpp:232-255
The eigensolver is ARPACK (scipy eigsh) on the FP64 operator: the converged SCF
fixed point does not depend on the eigensolver.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import hgh as _hgh
from . import pw

AU2K = 315774.67          # include/environment.hpp:175

# Goedecker-Teter-Hutter Pade coefficients (unpolarised)
_A = (0.4581652932831429, 2.217058676663745, 0.7405551735357053, 0.01968227878617998)
_B = (1.0, 4.504130959426697, 1.110667363742916, 0.02359291751427506)


def xc_teter93(rho: np.ndarray):
    """LDA Teter93: eps_xc(rs) = -(a0+a1 rs+a2 rs^2+a3 rs^3)/(b1 rs+b2 rs^2+b3 rs^3+b4 rs^4),
    v_xc = eps - rs/3 d eps/d rs; points with rho < 1e-10 are zeroed
    (hamiltonian.cpp:1298-1307)."""
    rho = np.asarray(rho, dtype=np.float64)
    bad = rho < 1e-10
    r = np.where(bad, 1.0, rho)
    rs = (3.0 / (4.0 * math.pi * r)) ** (1.0 / 3.0)
    a0, a1, a2, a3 = _A
    b1, b2, b3, b4 = _B
    N = a0 + rs * (a1 + rs * (a2 + rs * a3))
    D = rs * (b1 + rs * (b2 + rs * (b3 + rs * b4)))
    dN = a1 + rs * (2 * a2 + rs * 3 * a3)
    dD = b1 + rs * (2 * b2 + rs * (3 * b3 + rs * 4 * b4))
    eps = -N / D
    deps = -(dN * D - N * dD) / (D * D)
    v = eps - rs / 3.0 * deps
    eps = np.where(bad, 0.0, eps)
    v = np.where(bad, 0.0, v)
    return eps, v


def density(T: pw.HamTables, psi: np.ndarray, occ: np.ndarray, nocc: int, numSpin: int = 2, chunk: int = 16):
    """rho = sum_k numSpin f_k |psi_k,fine|^2, renormalised to numSpin*nocc
    electrons (hamiltonian.cpp:2511-2600).  The fine-grid wavefunction is the
    interpolation used by H*psi (the reference's idxFineGrid placement plus
    real part is the same map up to a constant that the renormalisation
    removes)."""
    dm = T.dm
    n0, n1, n2 = dm.numGrid
    N0, N1, N2 = dm.numGridFine
    rho = np.zeros(dm.ntotFine)
    for b0 in range(0, psi.shape[0], chunk):
        p = psi[b0:b0 + chunk]
        Xc = pw.r2c(p.reshape(-1, n2, n1, n0), dm)
        Xf = T.ip.c2f(Xc.reshape(p.shape[0], -1)).reshape(p.shape[0], N2, N1, N0 // 2 + 1)
        pf = pw.c2r(Xf, dm, fine=True).reshape(p.shape[0], -1)
        rho += (numSpin * occ[b0:b0 + chunk])[:, None].T @ (pf * pf) if False else \
            np.einsum("b,bi->i", numSpin * occ[b0:b0 + chunk], pf * pf)
    val = rho.sum()
    rho *= (numSpin * nocc * dm.ntotFine) / (dm.vol * val)
    return rho


def gkk_fine(dm: pw.Domain):
    g = pw.gvec_full(dm, fine=True)
    return 0.5 * np.sum(g * g, axis=-1)


def hartree(dm: pw.Domain, rho: np.ndarray, rho_ps: np.ndarray, ecut: float, gkk=None):
    """V_H = IFFT( 2 pi / gkk * FFT(rho - rho_ps) ), gkk = |G|^2/2, zero for
    gkk <= 1e-16 or gkk > 4 Ecut (hamiltonian.cpp:2003-2023)."""
    N0, N1, N2 = dm.numGridFine
    if gkk is None:
        gkk = gkk_fine(dm)
    X = np.fft.fftn((rho - rho_ps).reshape(N2, N1, N0)) * (dm.vol / dm.ntotFine)
    mask = (gkk <= 1e-16) | (gkk > 4.0 * ecut)
    fac = np.where(mask, 0.0, 2.0 * math.pi / np.where(mask, 1.0, gkk))
    v = np.fft.ifftn(X * fac) * (dm.ntotFine / dm.vol)
    return v.real.reshape(-1)


def wgauss(ev, ef, tbeta):
    return 1.0 / (1.0 + np.exp(-tbeta * (ef - ev)))


def entropy(ev, ef, tbeta):
    x = tbeta * (ef - ev)
    out = np.zeros_like(np.asarray(ev, dtype=np.float64))
    m = np.abs(x) <= 36.0
    occ = 1.0 / (1.0 + np.exp(-x[m]))
    with np.errstate(divide="ignore", invalid="ignore"):
        e = (occ * np.log(occ) + (1.0 - occ) * np.log(1.0 - occ)) / tbeta
    out[m] = np.nan_to_num(e)
    return out


def occupations(eig: np.ndarray, nocc: int, tbeta: float):
    """Fermi-Dirac bisection, scf.cpp:1780-1822."""
    ev = np.sort(eig)
    npsi = ev.size
    if npsi == nocc:
        return np.ones(npsi), ev[-1]
    lb, ub = ev[0], ev[-1]
    ef = 0.5 * (lb + ub)
    occsum = wgauss(ev, ef, tbeta).sum()
    it = 1
    while abs(occsum - nocc) > 1e-16 and it < 200:
        if occsum < nocc:
            lb = ef
        else:
            ub = ef
        ef = 0.5 * (lb + ub)
        occsum = wgauss(ev, ef, tbeta).sum()
        it += 1
    return wgauss(eig, ef, tbeta), ef


@dataclass
class SCFResult:
    eig: np.ndarray
    occ: np.ndarray
    etot: float
    efree: float
    eharris: float
    exc: float
    ehart: float
    eself: float
    history: list = field(default_factory=list)
    rho: np.ndarray = None
    vtot: np.ndarray = None
    psi: np.ndarray = None
    iterations: int = 0


def _eigsh(T: pw.HamTables, nband: int, v0=None, tol=1e-11):
    from scipy.sparse.linalg import LinearOperator, eigsh
    n = T.dm.ntot

    def mv(x):
        x = np.asarray(x).reshape(-1, n) if x.ndim > 1 else x.reshape(1, n)
        return pw.mult_spinor(T, np.ascontiguousarray(x.reshape(-1, n))).reshape(x.shape).T.squeeze() \
            if False else pw.mult_spinor(T, x.reshape(1, n)).reshape(-1)

    def mm(X):
        return pw.mult_spinor(T, np.ascontiguousarray(X.T)).T

    A = LinearOperator((n, n), matvec=mv, matmat=mm, dtype=np.float64)
    w, V = eigsh(A, k=nband, which="SA", tol=tol, v0=v0, ncv=min(n, max(2 * nband + 1, nband + 32)))
    o = np.argsort(w)
    return w[o], np.ascontiguousarray(V[:, o].T)


def scf(L, znuc, pos, numGrid, numGridFine, nocc: int, nextra: int, ecut: float,
        temperature: float = 300.0, tol_efree: float = 1e-7, max_iter: int = 60, mix_dim: int = 8,
        mix_step: float = 0.7, eig_tol: float = 1e-11, verbose: bool = False) -> SCFResult:
    """Restated SCF::Iterate with potential Anderson mixing; converges when
    |E_free - E_Harris| / N_atom < tol_efree (the reference's efreeDifPerAtom,
    scf.cpp:467)."""
    L = np.asarray(L, dtype=np.float64)
    zs = np.broadcast_to(np.asarray(znuc), (len(pos),))
    dm = pw.Domain(tuple(L), tuple(numGrid), tuple(numGridFine))
    ekin, teter = pw.ekin_teter(dm)
    species = {int(z): _hgh.hgh_table(int(z)) for z in set(int(z) for z in zs)}
    pseudo = [pw.nonlocal_pp(pw.Atom(int(z), p), dm, species[int(z)]) for z, p in zip(zs, pos)]
    rho_ps = np.zeros(dm.ntotFine)
    for z, p in zip(zs, pos):
        idx, dv = pw.pseudo_charge(pw.Atom(int(z), p), dm, species[int(z)])
        np.add.at(rho_ps, idx, dv[:, 0])
    eself = float(sum(species[int(z)].eself for z in zs))
    natom = len(pos)
    nband = nocc + nextra
    tbeta = AU2K / temperature
    gkk = gkk_fine(dm)
    w = dm.vol / dm.ntotFine
    # initial density from the pseudocharge (scf.cpp:232-255)
    rho = np.where(rho_ps > 1e-6, rho_ps, 1e-6)
    rho *= rho_ps.sum() / rho.sum()
    eps, vxc = xc_teter93(rho)
    exc = float(np.sum(eps * rho) * w)
    vh = hartree(dm, rho, rho_ps, ecut, gkk)
    vtot = vh + vxc
    T = pw.HamTables(dm, ekin, teter, vtot, pseudo)
    dv_hist, df_hist = [], []
    psi = None
    hist = []
    res = None
    for it in range(1, max_iter + 1):
        T.vtot = vtot
        v0 = psi[0] if psi is not None else None
        eig, psi = _eigsh(T, nband, v0=v0, tol=eig_tol)
        occ, ef = occupations(eig, nocc, tbeta)
        # Harris energy with the input density / potentials (scf.cpp:1987-2140)
        ekin_b = float(np.sum(2 * eig * occ))
        ehart_h = float(np.sum(0.5 * vh * (rho + rho_ps)) * w)
        evxc = float(np.sum(vxc * rho) * w)
        ecor_h = (exc - evxc) - ehart_h - eself
        efree_h = ekin_b + ecor_h + float(np.sum(2 * entropy(eig, ef, tbeta)))
        # new density and potentials
        rho_out = density(T, psi, occ, nocc)
        eps, vxc = xc_teter93(rho_out)
        exc = float(np.sum(eps * rho_out) * w)
        vh = hartree(dm, rho_out, rho_ps, ecut, gkk)
        vtot_new = vh + vxc
        # KS energy (scf.cpp:1834-1984), vtotOld = the input potential
        ecor = float(np.sum(-vtot * rho_out) * w)
        ehart = float(np.sum(0.5 * vh * (rho_out - rho_ps)) * w)
        ecor = ecor + exc + ehart - eself
        etot = ekin_b + ecor
        efree = etot + float(np.sum(2 * entropy(eig, ef, tbeta)))
        dif = abs(efree - efree_h) / natom
        hist.append(dict(iter=it, etot=etot, efree=efree, eharris=efree_h, dif=dif))
        if verbose:
            print(f"iter {it:3d} Etot {etot:.10f} Efree {efree:.10f} Eharris {efree_h:.10f} dif {dif:.3e}")
        res = SCFResult(eig=eig, occ=occ, etot=etot, efree=efree, eharris=efree_h, exc=exc, ehart=ehart,
                        eself=eself, history=hist, rho=rho_out, vtot=vtot, psi=psi, iterations=it)
        rho = rho_out
        if dif < tol_efree:
            break
        # Anderson mixing of the potential (scf.cpp:2299-2365)
        vtot = anderson(it, mix_step, mix_dim, vtot, vtot_new, dv_hist, df_hist)
    return res


def anderson(it, step, mix_dim, vin, vout, dv_hist, df_hist):
    F = vout - vin
    if it > 1:
        dim = min(it - 1, mix_dim)
        difv = np.stack([h - vin for h in dv_hist[-dim:]], axis=1)
        diff = np.stack([h - F for h in df_hist[-dim:]], axis=1)
        work = diff.T @ F
        ov = diff.T @ diff
        theta = np.linalg.solve(ov, work)
        xbar = vin - difv @ theta
        fbar = F - diff @ theta
    else:
        xbar, fbar = vin, F
    dv_hist.append(vin.copy())
    df_hist.append(F.copy())
    if len(dv_hist) > mix_dim:
        dv_hist.pop(0)
        df_hist.pop(0)
    return xbar + step * fbar
