"""FP64 NumPy restatement of the reference's sphere-cut (G-space) Gamma path.

Test infrastructure (see ``oracle/__init__.py``).  In this mode
(``Use_Real_Space: 0``) the wavefunction of a band is its Fourier coefficients
on the half sphere 1/2 |G|^2 < Ecut, stored with the sqrt(2) convention, and
the density grid equals the wavefunction grid (``Density_Grid_Factor`` 1,
``src/esdf.cpp:2786-2795,2840-2856``).  Follows:

  * sphere maps            Fourier::Initialize, ``src/SCF/fourier.cpp:542-640``
                           (idxCoarseCut in ascending R2C order; idxCoarsePadding
                           for the G_x = 0 plane)
  * ekin / Teter           KohnSham::CalculateEkin sphere branch,
                           ``src/SCF/hamiltonian.cpp:2630-2667``
  * local + kinetic        Spinor::AddMultSpinorFineR2C (complex overload),
                           ``src/SCF/spinor.cpp:528-680``
  * nonlocal               EigenSolver::NonlocalMultX,
                           ``src/EigenSolver/eigensolver.cpp:471-515`` with the
                           real Gram Re(A^H B) of ``src/MathLibs/blas.cpp:997-1029``
  * projector table        PeriodTable::CalculateNonlocalPP (Fourier space),
                           ``src/SCF/periodtable.cpp:1599-1849``; Simpson
                           ``src/utility.cpp:3329-3338``; spherical Bessel
                           ``src/utility.cpp:4314-4380``; vnlc assembly with the
                           structure factor and sqrt(2),
                           ``src/SCF/hamiltonian.cpp:700-797``
  * Teter                  Spinor::AddTeterPrecond (complex),
                           ``src/SCF/spinor.cpp:349-374``
  * density                KohnSham::CalculateDensity sphere branch,
                           ``src/SCF/hamiltonian.cpp:2508-2600``

The reference's Fourier-space projector builder integrates UPF samples r*beta(r)
on a uniform radial mesh of step 0.01 bohr; here those samples are the HGH
projector radial functions of ``oracle/hgh.py`` (the library's own HGH tables)
evaluated by the same spline the real-space path uses.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import hgh as _hgh
from . import pw

SQRT2 = math.sqrt(2.0)
MIN_RADIAL = 1e-10


@dataclass
class Sphere:
    """Sphere-cut maps of one Gamma-point G-space domain."""
    L: np.ndarray
    N: tuple                    # (n0, n1, n2): wavefunction = density grid
    ecut: float
    idx: np.ndarray             # idxCoarseCut: flat R2C indices, ascending
    pad_src: np.ndarray         # idxCoarsePadding.first
    pad_dst: np.ndarray         # idxCoarsePadding.second
    m: np.ndarray               # (ns, 3) signed Miller indices of the sphere points
    g: np.ndarray               # (ns, 3) Cartesian G
    ekin: np.ndarray            # (ns,)  |G|^2 / 2
    teter: np.ndarray           # (ns,)

    @property
    def ns(self):
        return int(self.idx.size)

    @property
    def vol(self):
        return float(np.prod(self.L))

    @property
    def ntot(self):
        return int(np.prod(self.N))

    @property
    def nr2c(self):
        return (self.N[0] // 2 + 1) * self.N[1] * self.N[2]


def r2c_miller(N):
    """Signed Miller indices (m0, m1, m2) of the R2C half grid in flat order
    i = x + (n0/2+1)(y + n1 z) (KGrid with Nyquist at +n/2, fourier.cpp:124-133)."""
    n0, n1, n2 = N
    k0 = pw.kgrid(n0)[: n0 // 2 + 1]
    M2, M1, M0 = np.meshgrid(pw.kgrid(n2), pw.kgrid(n1), k0, indexing="ij")
    return np.stack([M0.ravel(), M1.ravel(), M2.ravel()], axis=-1).astype(np.int64)


def sphere(L, N, ecut: float) -> Sphere:
    """``Fourier::Initialize`` sphere maps (fourier.cpp:542-640) and the sphere
    ekin / Teter tables (hamiltonian.cpp:2630-2667).  G_d = (2 pi / L_d) m_d."""
    L = np.asarray(L, np.float64)
    n0, n1, n2 = N
    h0 = n0 // 2 + 1
    m = r2c_miller(N)
    g = m * (2.0 * math.pi / L)[None, :]
    gkk = (g[:, 0] * g[:, 0] + g[:, 1] * g[:, 1] + g[:, 2] * g[:, 2]) / 2.0
    m0, m1, m2 = m[:, 0], m[:, 1], m[:, 2]
    in_grid = (m0 > 0) | ((m0 == 0) & ((m1 > 0) | ((m1 == 0) & (m2 >= 0))))
    do_pad = (m0 == 0) & ((m1 < 0) | ((m1 == 0) & (m2 < 0)))
    in_sphere = gkk < ecut
    idx = np.nonzero(in_grid & in_sphere)[0]
    dst = np.nonzero(do_pad & in_sphere)[0]
    src = h0 * np.mod(-m1[dst], n1) + h0 * n1 * np.mod(-m2[dst], n2)
    keep = src < h0 * n1 * n2
    a = 2.0 * gkk[idx]
    b = 27.0 + a * (18.0 + a * (12.0 + a * 8.0))
    teter = b / (b + 16.0 * a ** 4)
    return Sphere(L, tuple(N), float(ecut), idx, src[keep], dst[keep], m[idx], g[idx], gkk[idx], teter)


def to_r2c(sp: Sphere, c: np.ndarray) -> np.ndarray:
    """Sphere coefficients (nb, ns) -> R2C half spectrum (nb, n2, n1, n0/2+1):
    c_0 at G = 0, c_i / sqrt(2) elsewhere, then the G_x = 0 padding
    (spinor.cpp:568-590)."""
    nb = c.shape[0]
    n0, n1, n2 = sp.N
    X = np.zeros((nb, sp.nr2c), np.complex128)
    X[:, sp.idx[0]] = c[:, 0]
    X[:, sp.idx[1:]] = c[:, 1:] / SQRT2
    X[:, sp.pad_dst] = np.conj(X[:, sp.pad_src])
    return X.reshape(nb, n2, n1, n0 // 2 + 1)


def c2r_unnormalised(sp: Sphere, X: np.ndarray) -> np.ndarray:
    """FFTW's unnormalised C2R on the G-space grid, (nb, N)."""
    n0, n1, n2 = sp.N
    nb = X.shape[0]
    return (np.fft.irfftn(X, s=(n2, n1, n0), axes=(1, 2, 3)) * sp.ntot).reshape(nb, -1)


def from_r2c(sp: Sphere, Y: np.ndarray) -> np.ndarray:
    """R2C half spectrum -> sphere coefficients with sqrt(2) on G != 0
    (spinor.cpp:665-676)."""
    nb = Y.shape[0]
    Yf = Y.reshape(nb, -1)
    out = np.empty((nb, sp.ns), np.complex128)
    out[:, 0] = Yf[:, sp.idx[0]]
    out[:, 1:] = Yf[:, sp.idx[1:]] * SQRT2
    return out


def add_mult_spinor_gspace(sp: Sphere, vtot: np.ndarray, c: np.ndarray) -> np.ndarray:
    """Local + kinetic part of H on sphere coefficients c (nb, ns):
    C2R, x 1/N, x V_tot, R2C, pick with sqrt(2), plus ekin * c
    (spinor.cpp:562-676; the kinetic term is assigned, spinor.cpp:638-640)."""
    n0, n1, n2 = sp.N
    nb = c.shape[0]
    psi = c2r_unnormalised(sp, to_r2c(sp, c)) / sp.ntot
    upd = psi * vtot[None, :]
    Y = np.fft.rfftn(upd.reshape(nb, n2, n1, n0), axes=(1, 2, 3))
    return c * sp.ekin[None, :] + from_r2c(sp, Y)


def nonlocal_mult(vnlc: np.ndarray, wgt: np.ndarray, c: np.ndarray) -> np.ndarray:
    """V_nl c = vnlc (wgt o Re(vnlc^H c)) (NonlocalMultX), c (nb, ns)."""
    W = np.real(vnlc.conj().T @ c.T) * wgt[:, None]
    return (vnlc @ W).T


def hpsi(sp: Sphere, vtot, c, vnlc=None, wgt=None):
    """Full G-space H c: MultSpinor (a3 := 0 + AddMultSpinorFineR2C) plus
    NonlocalMultX, summed as in lobpcg.cpp:201-211."""
    out = add_mult_spinor_gspace(sp, vtot, c)
    if vnlc is not None and vnlc.shape[1] > 0:
        out = out + nonlocal_mult(vnlc, wgt, c)
    return out


def add_teter_precond(sp: Sphere, r: np.ndarray, a3: np.ndarray | None = None):
    """a3 += teter o r on the sphere (spinor.cpp:349-374)."""
    out = r * sp.teter[None, :]
    if a3 is None:
        return out
    a3 += out
    return a3


def density(sp: Sphere, c: np.ndarray, occ: np.ndarray, num_spin: int = 2, nocc: int | None = None):
    """Sphere-branch CalculateDensity (hamiltonian.cpp:2508-2600): psi(r) =
    C2R(...) / sqrt(N), rho = sum numSpin f |psi|^2, renormalised to
    numSpin * nocc electrons."""
    psi = c2r_unnormalised(sp, to_r2c(sp, c)) / math.sqrt(sp.ntot)
    rho = np.einsum("b,bi->i", num_spin * occ, psi * psi)
    if nocc is None:
        nocc = c.shape[0]
    val = rho.sum()
    return rho * (num_spin * nocc * sp.ntot) / (sp.vol * val)


# ---------------------------------------------------------------------------
# Fourier-space projectors (periodtable.cpp:1599-1849, hamiltonian.cpp:700-797)
# ---------------------------------------------------------------------------
def _double_factorial(n: int) -> float:
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def bessel(l: int, x: np.ndarray) -> np.ndarray:
    """Spherical Bessel j_l (utility.cpp:4314-4380): j_0(0) = 1, j_l(0) = 0,
    four-term series for |x| <= 0.05, closed forms above."""
    x = np.asarray(x, np.float64)
    out = np.empty_like(x)
    ax = np.abs(x)
    zero = ax < 1e-16
    small = (~zero) & (ax <= 0.05)
    big = ~(zero | small)
    out[zero] = 1.0 if l == 0 else 0.0
    xs = x[small]
    x2 = xs * xs
    out[small] = xs ** l / _double_factorial(2 * l + 1) * (
        1 - x2 / 1.0 / 2.0 / (2.0 * l + 3.0) * (
            1 - x2 / 2.0 / 2.0 / (2.0 * l + 5.0) * (
                1 - x2 / 3.0 / 2.0 / (2.0 * l + 7.0) * (
                    1 - x2 / 4.0 / 2.0 / (2.0 * l + 9.0)))))
    xb = x[big]
    if l == 0:
        out[big] = np.sin(xb) / xb
    elif l == 1:
        out[big] = (np.sin(xb) / xb - np.cos(xb)) / xb
    else:
        raise NotImplementedError("HGH Si / Al use l = 0, 1")
    return out


def simpson(f: np.ndarray, rab: float) -> float:
    """utility.cpp:3329-3338: sum over i = 0, 2, ..., n-3 of (f_i + 4 f_{i+1} + f_{i+2}) rab / 3."""
    n = f.size
    s = 0.0
    for i in range(0, n - 2, 2):
        s += (f[i] + 4 * f[i + 1] + f[i + 2]) / 3.0 * rab
    return s


RAB = 0.01          # uniform radial mesh step of the UPF-style samples
DQ = 0.01           # q-table step (periodtable.cpp:1611)


def radial_mesh(rcut: float):
    nr = int(math.floor(rcut / RAB + 1e-9)) + 1
    return RAB * np.arange(nr, dtype=np.float64)


def vq_tables(sp_hgh: _hgh.HGHSpecies, ecut: float):
    """Per projector channel k: (l, h, tab[q_j]) with tab(j) = Simpson of
    (r beta(r)) j_l(q_j r) r over r <= Rcut (periodtable.cpp:1655-1688)."""
    nqxq = int(pw.cround(math.sqrt(2 * ecut) / DQ + 4.0))
    r = radial_mesh(sp_hgh.wavcut)
    out = []
    for k, (l, h, _, _) in enumerate(sp_hgh.proj):
        rbeta = r * _hgh.spl_eval(sp_hgh, ("val", k), r)
        tab = np.empty(nqxq)
        for j in range(nqxq):
            tab[j] = simpson(rbeta * bessel(l, r * (DQ * j)) * r, RAB)
        out.append((l, h, tab))
    return out


def _interp(tab, gk):
    """Four-point Lagrange interpolation of the q table (periodtable.cpp:1703-1714)."""
    t = gk / DQ
    it0 = t.astype(np.int64)
    px = t - it0
    ux, vx, wx = 1.0 - px, 2.0 - px, 3.0 - px
    return (tab[it0] * ux * vx * wx / 6.0 + tab[it0 + 1] * px * vx * wx / 2.0
            - tab[it0 + 2] * px * ux * wx / 2.0 + tab[it0 + 3] * px * ux * vx / 6.0)


def vkb_species(sp: Sphere, tables):
    """vkb (ns, numpp) and the per-projector weight h (4 pi)^2 / vol
    (periodtable.cpp:1646-1653,1717-1745)."""
    g = sp.g
    gk = np.sqrt(g[:, 0] * g[:, 0] + g[:, 1] * g[:, 1] + g[:, 2] * g[:, 2])
    cols, wgt = [], []
    big = gk > MIN_RADIAL
    safe = np.where(big, gk, 1.0)
    for l, h, tab in tables:
        vq = _interp(tab, gk)
        if l == 0:
            cols.append(math.sqrt(1.0 / (4 * math.pi)) * vq.astype(np.complex128))
            wgt.append(h * (4 * math.pi) ** 2 / sp.vol)
        elif l == 1:
            coef = -1j * math.sqrt(3.0 / (4 * math.pi))
            for comp in (2, 0, 1):          # p_z, p_x, p_y
                cols.append(np.where(big, coef * g[:, comp] / safe * vq, 0.0))
                wgt.append(h * (4 * math.pi) ** 2 / sp.vol)
        else:
            raise NotImplementedError("HGH Si / Al use l = 0, 1")
    return np.stack(cols, axis=1), np.asarray(wgt)


def vnlc(sp: Sphere, znuc, pos):
    """vnlc (ns, n_proj) and weights for atoms at Cartesian pos (natom, 3), one
    species: vkb times the structure factor e^{-i G.R}, sqrt(2) on G != 0
    (hamiltonian.cpp:740-797)."""
    spec = _hgh.hgh_table(znuc)
    vkb, w = vkb_species(sp, vq_tables(spec, sp.ecut))
    cols, wgt = [], []
    for R in np.asarray(pos, np.float64):
        cc = np.exp(-1j * (sp.g @ R))
        for k in range(vkb.shape[1]):
            col = vkb[:, k] * cc
            col[1:] *= SQRT2
            cols.append(col)
            wgt.append(w[k])
    return np.stack(cols, axis=1), np.asarray(wgt)


# ---------------------------------------------------------------------------
# seeded states
# ---------------------------------------------------------------------------
def random_orthonormal_c(sp: Sphere, nb: int, seed: int) -> np.ndarray:
    """Gaussian sphere coefficients with Im c_0 = 0, orthonormal in the real
    inner product Re(c^H d) (the sqrt(2)-convention Gram), rows are bands."""
    rng = np.random.Generator(np.random.Philox(seed))
    Z = rng.standard_normal((nb, sp.ns)) + 1j * rng.standard_normal((nb, sp.ns))
    Z[:, 0] = Z[:, 0].real
    S = np.real(Z.conj() @ Z.T)
    U = np.linalg.cholesky(S).T
    return np.linalg.solve(U.T, Z)


def real_view(c: np.ndarray) -> np.ndarray:
    """(nb, ns) complex -> (nb, 2 ns) real, interleaved (re, im) per point."""
    return np.ascontiguousarray(c).view(np.float64).reshape(c.shape[0], -1)


def complex_view(x: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(x).view(np.complex128).reshape(x.shape[0], -1)


def _full_g2(sp: Sphere) -> np.ndarray:
    """|G|^2 on the full N^3 grid, (N2, N1, N0) x fastest."""
    n0, n1, n2 = sp.N
    m0 = np.fft.fftfreq(n0, 1.0 / n0)
    m1 = np.fft.fftfreq(n1, 1.0 / n1)
    m2 = np.fft.fftfreq(n2, 1.0 / n2)
    L = np.asarray(sp.L, float)
    g0 = 2 * np.pi / L[0] * m0
    g1 = 2 * np.pi / L[1] * m1
    g2 = 2 * np.pi / L[2] * m2
    return g2[:, None, None] ** 2 + g1[None, :, None] ** 2 + g0[None, None, :] ** 2


def exx_kernel(sp: Sphere, ecut: float, mu: float = 0.0, div_type: int = 1):
    """(exxgkkR2C on the R2C half grid, zero outside the Fock set, exxDiv) of
    KohnSham::InitializeEXX with a sphere cut (src/SCF/hamiltonian.cpp:
    3454-3551): exxDiv sums over eps < |G|^2 < 4 Ecut of the full grid, the
    kernel lives on the R2C points with 1/2 |G|^2 < 4 Ecut (Fock set,
    src/SCF/fourier.cpp:642-666)."""
    eps = 1e-8
    alpha = 10.0 / (ecut * 2.0)
    q = _full_g2(sp).reshape(-1)
    div = 0.0
    if div_type == 1:
        sel = (q > eps) & (q < ecut * 4.0)
        if mu > 0.0:
            div = float(np.sum(np.exp(-alpha * q[sel]) / q[sel] * (1.0 - np.exp(-q[sel] / (4 * mu * mu)))))
            div += 1.0 / (4 * mu * mu)
        else:
            div = float(np.sum(np.exp(-alpha * q[sel]) / q[sel])) - alpha
        div *= 4.0 * np.pi
        aa = 1.0 / math.sqrt(alpha * np.pi)
        if mu > 0.0:
            aa -= 1.0 / math.sqrt(np.pi * (alpha + 1.0 / (4 * mu * mu)))
        div -= sp.vol * aa
    n0, n1, n2 = sp.N
    qh = _full_g2(sp)[:, :, : n0 // 2 + 1]
    k = np.zeros_like(qh)
    fock = 0.5 * qh < 4.0 * ecut
    big = fock & (qh > eps)
    if mu > 0.0:
        k[big] = 4 * np.pi / qh[big] * (1.0 - np.exp(-qh[big] / (4 * mu * mu)))
    else:
        k[big] = 4 * np.pi / qh[big]
    zero = fock & (qh <= eps)
    k[zero] = -div + (np.pi / (mu * mu) if mu > 0.0 else 0.0)
    return k, div


def set_phi(sp: Sphere, c: np.ndarray) -> np.ndarray:
    """phi = sqrt(1 / (vol N)) c (SetPhiEXX sphere-cut branch, hamiltonian.cpp:3568-3580)."""
    return c * math.sqrt(1.0 / (sp.vol * sp.ntot))


def add_mult_spinor_exx(sp: Sphere, c: np.ndarray, phi: np.ndarray, kern: np.ndarray, frac: float,
                        occ: np.ndarray) -> np.ndarray:
    """V_x c of Spinor::AddMultSpinorEXX, complex overload
    (src/SCF/spinor.cpp:783-945): psi(r), phi(r) by the unnormalised C2R of
    their sphere coefficients, pair products transformed with the reference's
    forward (x vol/N) and backward (x 1/vol) conventions around the kernel,
    times -alpha f_j phi_j, unnormalised R2C and sqrt(2) on G != 0."""
    n0, n1, n2 = sp.N
    shp = (n2, n1, n0)
    pr = c2r_unnormalised(sp, to_r2c(sp, c))
    fr = c2r_unnormalised(sp, to_r2c(sp, phi))
    acc = np.zeros_like(pr)
    for j in range(fr.shape[0]):
        prod = (pr * fr[j][None, :]).reshape((-1,) + shp)
        X = np.fft.rfftn(prod, axes=(1, 2, 3)) * (sp.vol / sp.ntot) * kern[None]
        v = np.fft.irfftn(X, s=shp, axes=(1, 2, 3)) * sp.ntot / sp.vol
        acc += -frac * occ[j] * v.reshape(pr.shape) * fr[j][None, :]
    Y = np.fft.rfftn(acc.reshape((-1,) + shp), axes=(1, 2, 3))
    return from_r2c(sp, Y)
