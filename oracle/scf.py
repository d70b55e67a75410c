"""FP64 NumPy restatement of the reference's Gamma-point SCF around H*psi.

Test infrastructure (see ``oracle/__init__.py``).  Follows:
  * KohnSham::CalculateDensity    src/SCF/hamiltonian.cpp:2455-2627
  * KohnSham::CalculateHartree    src/SCF/hamiltonian.cpp:1990-2026
  * KohnSham::CalculateXC         src/SCF/hamiltonian.cpp:1242-1308 (LDA Teter93; the
    reference calls libxc XC_LDA_XC_TETER93, restated here from Goedecker, Teter,
    Hutter, PRB 54, 1703 (1996); parity at the libxc boundary is unpinned)
  * KohnSham::CalculateGradDensity src/SCF/hamiltonian.cpp:1153-1239 and the PBE
    branch of CalculateXC without libxc (Use_Libxc 0), hamiltonian.cpp:1381-1419,
    1560-1612, 1680-1760: Slater + PW92 LDA, PBE gradient corrections
    (VExchange_sla, VCorrelation_pw, VGCExchange_pbx, VGCCorrelation_pbc,
    src/utility.cpp:3913-4244; pinned by tests/golden/ref_xc_pbe.npz from those
    functions), V_xc = v1 - div(v2 grad rho) with spectral derivatives
  * KohnSham::CalculateVtot       src/SCF/hamiltonian.cpp:2029-2069 (Use_VLocal 0)
  * SCF::CalculateOccupationRate  src/SCF/scf.cpp:1748-1830, wgauss/getEntropy
    src/utility.cpp:4404-4444
  * SCF::CalculateEnergy / CalculateHarrisEnergy  src/SCF/scf.cpp:1834-2140
  * SCF::andersonMix              src/SCF/scf.cpp:2299-2365
  * SCF::BroydenMix / RhoDdot      src/SCF/scf.cpp:2144-2296 (potential mixing)
  * SCF::Iterate / InnerSolve     src/SCF/scf.cpp:372-591, 1261-1589
  * the nested hybrid scheme of SCF::Iterate (scf.cpp:409-425, 628-925): PBE SCF,
    then the semilocal HSE06 (oracle/hse.py) with phi iterations over an ACE
    operator (oracle/exx.py), Fock energies and dExx
  * initial density from the pseudocharge  src/SCF/scf.cpp:232-255
The eigensolver is ARPACK (scipy eigsh) on the FP64 operator, or, for large
cells, scipy's block LOBPCG over a caller-supplied block H*psi
(``set_block_hx``, e.g. a process pool): the converged SCF fixed point does not
depend on the eigensolver.  With ``wfn_ecut`` the SCF runs on the filtered
operator of the reference's CheFSI path (KohnSham::MultSpinor's wavefunction
cut-off filter, hamiltonian.cpp:316-321, 3090-3116, 3240-3265): P H P on the
span of P, the complement shifted out of the wanted spectrum.
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


# ---------------------------------------------------------------------------
# PBE (unpolarised), Perdew-Burke-Ernzerhof PRL 77, 3865 (1996) with the
# Perdew-Wang 1992 LDA correlation, in the constants of the reference's
# internal functions (src/utility.cpp:3913-4244)
# ---------------------------------------------------------------------------
_SLATER = -0.458165293283143               # -(3/4pi) (9pi/4)^(1/3)
_PW92 = (0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294)     # A, alpha1, beta1..beta4
_KAPPA, _MU = 0.804, 0.2195149727645171
_GAMMA, _BETA = 0.03109069086965, 0.06672455060314922
_C2 = 3.093667726280136                    # (3 pi^2)^(1/3)
_PI34, _XKF, _XKS = 0.6203504908994, 1.919158292677513, 1.128379167095513


def slater(rs):
    """(eps_x, v_x) of the uniform gas at rs (VExchange_sla)."""
    ux = _SLATER / rs
    return ux, 4.0 / 3.0 * ux


def pw92(rs):
    """(eps_c, v_c = eps_c - rs/3 d eps_c/d rs) (VCorrelation_pw)."""
    a, a1, b1, b2, b3, b4 = _PW92
    q = np.sqrt(rs)
    om = 2 * a * (b1 * q + b2 * rs + b3 * rs * q + b4 * rs * rs)
    rdom = 2 * a * (0.5 * b1 * q + b2 * rs + 1.5 * b3 * rs * q + 2 * b4 * rs * rs)   # rs d om / d rs
    lg = np.log(1 + 1 / om)
    ec = -2 * a * (1 + a1 * rs) * lg
    vc = -2 * a * (1 + 2.0 / 3.0 * a1 * rs) * lg - 2.0 / 3.0 * a * (1 + a1 * rs) * rdom / (om * (om + 1))
    return ec, vc


def pbe_x(rho, sigma):
    """Gradient part of PBE exchange: (e per particle, d(rho e)/d rho, 2 d(rho e)/d sigma)
    with F_x - 1 = kappa - kappa / (1 + mu s^2 / kappa), s = |grad rho| / (2 k_F rho)
    (VGCExchange_pbx)."""
    g = np.sqrt(sigma)
    kf = _C2 * np.power(rho, 1.0 / 3.0)
    dsg = 0.5 / kf
    sr = g * dsg / rho
    den = 1 + sr * sr * _MU / _KAPPA
    fx = _KAPPA - _KAPPA / den
    exu = -0.75 / math.pi * kf
    dfx = 2 * _MU * sr / (den * den)
    e = exu * fx
    return e, e + exu / 3 * fx - exu * dfx * (4.0 / 3.0) * sr, exu * dfx * dsg / g


def pbe_c(rho, sigma):
    """Gradient part of PBE correlation H(t, A) (VGCCorrelation_pbc):
    (H, d(rho H)/d rho, 2 d(rho H)/d sigma)."""
    rs = _PI34 / np.power(rho, 1.0 / 3.0)
    ec, vc = pw92(rs)
    ks = _XKS * np.sqrt(_XKF / rs)
    t2 = sigma / (2 * ks * rho) ** 2
    ex = np.exp(-ec / _GAMMA)
    A = _BETA / _GAMMA * (1.0 / (ex - 1.0))
    y = A * t2
    d = 1 + y + y * y
    xy = (1 + y) / d
    qy = y * y * (2 + y) / (d * d)
    s1 = 1 + _BETA / _GAMMA * t2 * xy
    H = _GAMMA * np.log(s1)
    # rho dH/drho: t^2 ~ rho^(-7/3) and A through eps_c (rho d eps_c / d rho = v_c - eps_c)
    rdh = _BETA * t2 / s1 * (-7.0 / 3.0 * xy - qy * (A * ex * (vc - ec) / _BETA - 7.0 / 3.0))
    return H, H + rdh, _BETA / (2 * ks * ks * rho) * (xy - qy) / s1


def xc_pbe_point(rho, sigma):
    """Per point (hamiltonian.cpp:1581-1612): LDA part where |rho| > 1e-10,
    gradient part where |rho| > 1e-6 and sigma > 1e-10.  Returns (eps per
    particle, v1 = d e/d rho, v2 = 2 d e/d sigma) with e = rho eps."""
    rho = np.asarray(rho, np.float64)
    sigma = np.asarray(sigma, np.float64)
    ar = np.abs(rho)
    eps = np.zeros_like(rho)
    v1 = np.zeros_like(rho)
    v2 = np.zeros_like(rho)
    m = ar > 1e-10
    if m.any():
        rs = np.power(3.0 / 4.0 / math.pi / ar[m], 1.0 / 3.0)
        ux, vx = slater(rs)
        uc, vc = pw92(rs)
        eps[m] += ux + uc
        v1[m] += vx + vc
    g = (ar > 1e-6) & (sigma > 1e-10)
    if g.any():
        ex, v1x, v2x = pbe_x(ar[g], sigma[g])
        ec, v1c, v2c = pbe_c(ar[g], sigma[g])
        eps[g] += ex + ec
        v1[g] += v1x + v1c
        v2[g] += v2x + v2c
    return eps, v1, v2


def _spectral_ik(dm: pw.Domain, ecut: float):
    """i G_d on the fine grid, zero where gkk = 0 or gkk > 4 Ecut (ikFine with the
    cut of hamiltonian.cpp:1196-1201)."""
    g = pw.gvec_full(dm, fine=True)
    gkk = 0.5 * np.sum(g * g, axis=-1)
    keep = ~((gkk == 0) | (gkk > 4.0 * ecut))
    return [1j * g[..., d] * keep for d in range(3)]


def grad_density(dm: pw.Domain, rho: np.ndarray, ecut: float):
    """CalculateGradDensity: d_d rho = Re IFFT(i G_d FFT(rho)) with the cut."""
    N0, N1, N2 = dm.numGridFine
    X = np.fft.fftn(rho.reshape(N2, N1, N0))
    return np.stack([np.fft.ifftn(X * ik).real.reshape(-1) for ik in _spectral_ik(dm, ecut)])


def xc_pbe(dm: pw.Domain, rho: np.ndarray, ecut: float, point=None):
    """(eps per particle, V_xc) of PBE: V_xc = v1 - sum_d d_d(v2 d_d rho), the
    divergence spectral with the same cut (hamiltonian.cpp:1750-1775).
    ``point`` replaces the point functional (default xc_pbe_point; the
    semilocal HSE06 passes oracle.hse.hse06_point)."""
    N0, N1, N2 = dm.numGridFine
    gr = grad_density(dm, rho, ecut)
    sigma = np.sum(gr * gr, axis=0)
    eps, v1, v2 = (point or xc_pbe_point)(rho, sigma)
    div = np.zeros((N2, N1, N0), complex)
    for d, ik in enumerate(_spectral_ik(dm, ecut)):
        div += np.fft.fftn((v2 * gr[d]).reshape(N2, N1, N0)) * ik
    return eps, v1 - np.fft.ifftn(div).real.reshape(-1)


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


def wgauss(ev, ef, tbeta, smearing: str = "FD"):
    """Occupation rate of a state (wgauss, src/utility.cpp:4404-4420):
    Fermi-Dirac 1 / (1 + exp(-x)) or Gaussian erfc(-x) / 2, x = beta (E_F - e)."""
    x = tbeta * (ef - np.asarray(ev, dtype=np.float64))
    if smearing == "GB":
        return 0.5 * _erfc(-x)
    return 1.0 / (1.0 + np.exp(-x))


def _erfc(x):
    from scipy.special import erfc
    return erfc(x)


def entropy(ev, ef, tbeta, smearing: str = "FD"):
    """-T S term of a state (getEntropy, src/utility.cpp:4422-4444)."""
    x = tbeta * (ef - np.asarray(ev, dtype=np.float64))
    if smearing == "GB":
        return -0.5 / tbeta * np.exp(-np.minimum(200.0, x * x)) / math.sqrt(math.pi)
    out = np.zeros_like(x)
    m = np.abs(x) <= 36.0
    occ = 1.0 / (1.0 + np.exp(-x[m]))
    with np.errstate(divide="ignore", invalid="ignore"):
        e = (occ * np.log(occ) + (1.0 - occ) * np.log(1.0 - occ)) / tbeta
    out[m] = np.nan_to_num(e)
    return out


def occupations(eig: np.ndarray, nocc: int, tbeta: float, smearing: str = "FD"):
    """Bisection on the electron count, scf.cpp:1780-1822 (either smearing)."""
    ev = np.sort(eig)
    npsi = ev.size
    if npsi == nocc:
        return np.ones(npsi), ev[-1]
    lb, ub = ev[0], ev[-1]
    ef = 0.5 * (lb + ub)
    occsum = wgauss(ev, ef, tbeta, smearing).sum()
    it = 1
    while abs(occsum - nocc) > 1e-16 and it < 200:
        if occsum < nocc:
            lb = ef
        else:
            ub = ef
        ef = 0.5 * (lb + ub)
        occsum = wgauss(ev, ef, tbeta, smearing).sum()
        it += 1
    return wgauss(eig, ef, tbeta, smearing), ef


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
    efock: float = 0.0
    dexx: float = 0.0
    phi_iterations: int = 0


_BLOCK = {"hx": None, "tol": 1e-8, "maxiter": 400}
NULL_SHIFT = 100.0      # Ha: where the filtered operator puts the span of I - P


def set_block_hx(hx_block=None, tol: float = 1e-8, maxiter: int = 400):
    """Use block LOBPCG (scipy) with ``hx_block(T, rows) -> H rows`` (rows:
    nb x ntot) instead of ARPACK; None restores ARPACK.  ``tol`` is the
    residual tolerance of the last SCF steps (earlier steps use a looser one)."""
    _BLOCK["hx"], _BLOCK["tol"], _BLOCK["maxiter"] = hx_block, tol, maxiter


def _operator(T: pw.HamTables, xi=None, wfn_ecut=None, hx_block=None):
    """rows -> rows of H (+ ACE), or of P H P + NULL_SHIFT (I - P) with the filter."""
    def hx(rows):
        rows = np.ascontiguousarray(rows)
        f = pw.wfn_ecut_filter(T, rows, wfn_ecut) if wfn_ecut is not None else rows
        out = hx_block(T, f) if hx_block is not None else pw.mult_spinor(T, f)
        if xi is not None:
            out = out - (f @ xi.T) @ xi
        if wfn_ecut is not None:
            out = pw.wfn_ecut_filter(T, out, wfn_ecut) + NULL_SHIFT * (rows - f)
        return out
    return hx


def _lobpcg(T: pw.HamTables, nband: int, X0: np.ndarray, tol: float, xi=None, wfn_ecut=None):
    """Lowest eigenpairs by scipy's block LOBPCG (Teter preconditioner, the
    block H*psi of set_block_hx), started from X0 (nband x ntot)."""
    from scipy.sparse.linalg import lobpcg
    hx = _operator(T, xi, wfn_ecut, _BLOCK["hx"])
    A = lambda X: hx(np.asarray(X).T).T                         # noqa: E731
    M = lambda R: pw.add_teter_precond(T, np.ascontiguousarray(np.asarray(R).T)).T   # noqa: E731
    w, V = lobpcg(A, np.ascontiguousarray(X0.T), M=M, tol=tol, maxiter=_BLOCK["maxiter"], largest=False)
    o = np.argsort(w)
    return w[o], np.ascontiguousarray(V[:, o].T)


def _eigsh(T: pw.HamTables, nband: int, v0=None, tol=1e-11, xi=None, wfn_ecut=None):
    """Lowest eigenpairs of H (plus the ACE term -xi^T xi when xi is given;
    the filtered operator with wfn_ecut)."""
    from scipy.sparse.linalg import LinearOperator, eigsh
    n = T.dm.ntot
    hx = _operator(T, xi, wfn_ecut)

    def mv(x):
        return hx(np.asarray(x).reshape(1, n)).reshape(-1)

    def mm(X):
        return hx(X.T).T

    A = LinearOperator((n, n), matvec=mv, matmat=mm, dtype=np.float64)
    w, V = eigsh(A, k=nband, which="SA", tol=tol, v0=v0, ncv=min(n, max(2 * nband + 1, nband + 32)))
    o = np.argsort(w)
    return w[o], np.ascontiguousarray(V[:, o].T)


def scf(L, znuc, pos, numGrid, numGridFine, nocc: int, nextra: int, ecut: float,
        temperature: float = 300.0, tol_efree: float = 1e-7, max_iter: int = 60, mix_dim: int = 8,
        mix_step: float = 0.7, eig_tol: float = 1e-11, verbose: bool = False, xc: str = "teter93",
        mix: str = "anderson", tol_rho: float | None = None, phi_max_iter: int = 10,
        phi_tol: float = 1e-6, wfn_ecut: float | None = None, seed: int = 20261203,
        smearing: str = "FD") -> SCFResult:
    """Restated SCF::Iterate with potential Anderson mixing; converges when
    |E_free - E_Harris| / N_atom < tol_efree (the reference's efreeDifPerAtom,
    scf.cpp:467).  xc = "hse06": the nested hybrid scheme (PBE SCF, then phi
    iterations with ACE until dExx < phi_tol; inner loops restart the mixing
    history and, with tol_rho, test the scfNorm of the potential change)."""
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
    hybrid = xc == "hse06"
    xcf = xc_teter93 if xc == "teter93" else (lambda r: xc_pbe(dm, r, ecut))
    eps, vxc = xcf(rho)
    exc = float(np.sum(eps * rho) * w)
    vh = hartree(dm, rho, rho_ps, ecut, gkk)
    vtot = vh + vxc
    T = pw.HamTables(dm, ekin, teter, vtot, pseudo)
    psi = None
    hist = []
    res = None
    xi = None
    inner = False

    def loop():
        nonlocal vtot, rho, exc, vxc, vh, psi, res
        dv_hist, df_hist = [], []
        bst = BroydenState(mix_dim)
        for it in range(1, max_iter + 1):
            if step(it, dv_hist, df_hist, bst):
                return

    def step(it, dv_hist, df_hist, bst):
        nonlocal vtot, rho, exc, vxc, vh, psi, res
        T.vtot = vtot
        if _BLOCK["hx"] is not None:
            X0 = psi if psi is not None else pw.random_orthonormal_psi(dm.ntot, nband, seed)
            if wfn_ecut is not None:
                X0 = pw.wfn_ecut_filter(T, X0, wfn_ecut)
            # loose residual tolerance while the potential still moves
            prev = hist[-1]["dif"] if hist else 1.0
            tol = float(np.clip(1e-4 * math.sqrt(prev), _BLOCK["tol"], 1e-5))
            eig, psi = _lobpcg(T, nband, X0, tol, xi=xi, wfn_ecut=wfn_ecut)
        else:
            v0 = psi[0] if psi is not None else None
            eig, psi = _eigsh(T, nband, v0=v0, tol=eig_tol, xi=xi, wfn_ecut=wfn_ecut)
        occ, ef = occupations(eig, nocc, tbeta, smearing)
        # Harris energy with the input density / potentials (scf.cpp:1987-2140)
        ekin_b = float(np.sum(2 * eig * occ))
        ehart_h = float(np.sum(0.5 * vh * (rho + rho_ps)) * w)
        evxc = float(np.sum(vxc * rho) * w)
        ecor_h = (exc - evxc) - ehart_h - eself
        efree_h = ekin_b + ecor_h + float(np.sum(2 * entropy(eig, ef, tbeta, smearing)))
        # new density and potentials
        rho_out = density(T, psi, occ, nocc)
        eps, vxc = xcf(rho_out)
        exc = float(np.sum(eps * rho_out) * w)
        vh = hartree(dm, rho_out, rho_ps, ecut, gkk)
        vtot_new = vh + vxc
        # KS energy (scf.cpp:1834-1984), vtotOld = the input potential
        ecor = float(np.sum(-vtot * rho_out) * w)
        ehart = float(np.sum(0.5 * vh * (rho_out - rho_ps)) * w)
        ecor = ecor + exc + ehart - eself
        etot = ekin_b + ecor
        efree = etot + float(np.sum(2 * entropy(eig, ef, tbeta, smearing)))
        dif = abs(efree - efree_h) / natom
        snorm = scf_norm(dm, (vtot_new - vtot) if inner else (rho_out - rho), ecut)
        hist.append(dict(iter=it, etot=etot, efree=efree, eharris=efree_h, dif=dif, scf_norm=snorm))
        if verbose:
            print(f"iter {it:3d} Etot {etot:.10f} Efree {efree:.10f} Eharris {efree_h:.10f} dif {dif:.3e} "
                  f"scfnorm {snorm:.3e}")
        res = SCFResult(eig=eig, occ=occ, etot=etot, efree=efree, eharris=efree_h, exc=exc, ehart=ehart,
                        eself=eself, history=hist, rho=rho_out, vtot=vtot, psi=psi, iterations=len(hist))
        rho = rho_out
        if (tol_rho is None and dif < tol_efree) or (tol_rho is not None and snorm < tol_rho):
            return True
        # Anderson mixing of the potential (scf.cpp:2299-2365)
        if mix == "broyden":
            vtot = broyden(dm, it, mix_step, vtot, vtot_new, bst, ecut)
        else:
            vtot = anderson(it, mix_step, mix_dim, vtot, vtot_new, dv_hist, df_hist)
        return False

    loop()
    if not hybrid:
        return res
    # hybrid part (scf.cpp:628-925): semilocal HSE06 from the last density,
    # phi <- psi, ACE, Fock energies
    from . import exx as _exx
    from . import hse as _hse
    xcf = lambda r: _hse.xc_hse06(dm, r, ecut)  # noqa: E731
    eps, vxc = xcf(rho)
    exc = float(np.sum(eps * rho) * w)
    vh = hartree(dm, rho, rho_ps, ecut, gkk)
    vtot = vh + vxc
    kern = _exx.exx_kernel_r2c(dm, ecut, mu=_hse.OMEGA_HSE06, div_type=1)[0]

    def fock(p_, o_, xi_):
        return _exx.exx_energy(-(p_ @ xi_.T) @ xi_, p_, o_, numSpin=2)

    def ace(p_, o_):
        return _exx.ace_build(dm, p_, _exx.set_phi(dm, p_), kern, _hse.FRAC_HSE06, o_)

    xi = ace(psi, res.occ)
    fock0 = fock(psi, res.occ, xi)
    inner = True
    conv = False
    efock = dexx = 0.0
    for phi_it in range(1, phi_max_iter + 1):
        loop()
        fock1 = fock(psi, res.occ, xi)
        xi = ace(psi, res.occ)
        fock2 = fock(psi, res.occ, xi)
        dexx = 4.0 * abs(fock1 - 0.5 * (fock0 + fock2))
        fock0 = fock2
        efock = fock2
        res.etot = res.etot - 2.0 * fock1 + efock
        res.efree = res.efree - 2.0 * fock1 + efock
        if verbose:
            print(f"phi {phi_it} Efock {efock:.10f} Etot {res.etot:.10f} dExx {dexx:.3e}")
        if dexx < phi_tol:
            conv = True
            break
    res.efock, res.dexx, res.phi_iterations = efock, dexx, phi_it
    res.converged = conv
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


class BroydenState:
    """History of SCF::BroydenMix: df, dv (mix_dim slots) and the previous
    (residual, input) pair (the reference's GdfMat_, GdvMat_, GcdfMat_)."""

    def __init__(self, mix_dim: int):
        self.mix_dim = mix_dim
        self.df = [None] * mix_dim
        self.dv = [None] * mix_dim
        self.cdf = None


def broyden(dm: pw.Domain, it: int, step: float, vin: np.ndarray, vout: np.ndarray, st: BroydenState,
            ecut: float):
    """SCF::BroydenMix (src/SCF/scf.cpp:2144-2261) for the potential: Fourier
    components inside the density sphere 1/2|G|^2 < 4 Ecut (idxFineCutDensity),
    inner product RhoDdot = pi vol sum Re(conj(a) b) / gkk over gkk != 0
    (scf.cpp:2263-2296), the mixed potential back from those components only."""
    N0, N1, N2 = dm.numGridFine
    gkk = gkk_fine(dm).reshape(-1)
    sph = gkk < 4.0 * ecut
    wgt = np.where(sph & (gkk != 0), math.pi * dm.vol / np.where(gkk != 0, gkk, 1.0), 0.0)
    fwd = lambda v: (np.fft.fftn(v.reshape(N2, N1, N0)) * (dm.vol / dm.ntotFine)).reshape(-1)[sph]

    def ddot(a, b):
        return float(np.sum(wgt[sph] * np.real(np.conj(a) * b)))

    gold = fwd(vin)
    gnew = fwd(vout) - gold
    m = st.mix_dim
    used = min(it - 1, m)
    ipos = it - 1 - ((it - 2) // m) * m
    if it > 1:
        st.df[ipos - 1] = st.cdf[0] - gnew
        st.dv[ipos - 1] = st.cdf[1] - gold
    st.cdf = (gnew.copy(), gold.copy())
    if used > 0:
        beta = np.empty((used, used))
        for i in range(used):
            for j in range(i, used):
                beta[i, j] = beta[j, i] = ddot(st.df[j], st.df[i])
        beta = np.linalg.inv(beta)
        work = np.array([ddot(st.df[i], gnew) for i in range(used)])
        for i in range(used):
            g0 = float(beta[:, i] @ work)
            gold = gold - g0 * st.dv[i]
            gnew = gnew - g0 * st.df[i]
    gmix = gold + step * gnew
    full = np.zeros(dm.ntotFine, complex)
    full[sph] = gmix
    return (np.fft.ifftn(full.reshape(N2, N1, N0)) * (dm.ntotFine / dm.vol)).real.reshape(-1)


def scf_norm(dm: pw.Domain, drho: np.ndarray, ecut: float) -> float:
    """SCF::CalculateError (src/SCF/scf.cpp:2368-2396): RhoDdot of the change of
    the output density, pi vol sum_{G != 0, 1/2|G|^2 < 4 Ecut} |drho(G)|^2 / gkk
    with drho(G) the forward transform (x vol/N) divided by vol."""
    N0, N1, N2 = dm.numGridFine
    gkk = gkk_fine(dm).reshape(-1)
    X = np.fft.fftn(drho.reshape(N2, N1, N0)).reshape(-1) / dm.ntotFine
    m = (gkk < 4.0 * ecut) & (gkk != 0)
    return float(math.pi * dm.vol * np.sum(np.abs(X[m]) ** 2 / gkk[m]))
