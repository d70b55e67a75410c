"""FP64 NumPy restatement of the reference's real (Gamma-point) H*psi path.

Test infrastructure (see ``oracle/__init__.py``).  Grid index convention as
in the reference: ``idx = i + n0*j + n0*n1*k`` (x fastest), so a real-space
array is stored as ``a[k, j, i]`` and a real-to-complex half spectrum as
``A[k, j, i]`` with ``i`` in ``[0, n0/2]`` (FFTW dims passed as (n2,n1,n0),
``src/SCF/fourier.cpp:112-122,178-188``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import hgh as _hgh

MIN_RADIAL = 1e-10          # include/periodtable.hpp:158


def cround(x):
    """C/C++ ``round``: half away from zero."""
    x = np.asarray(x, dtype=np.float64)
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


# ---------------------------------------------------------------------------
# Domain and Fourier tables
# ---------------------------------------------------------------------------
@dataclass
class Domain:
    """Orthorhombic ``Domain`` (include/domain.hpp:55-139)."""
    length: tuple                       # (Lx, Ly, Lz) bohr
    numGrid: tuple                      # coarse (n0, n1, n2)
    numGridFine: tuple                  # fine  (N0, N1, N2)

    @property
    def supercell(self):
        return np.diag(np.asarray(self.length, dtype=np.float64))

    @property
    def recipcell(self):
        # recipcell = 2*pi*inv(supercell)^T  (src/esdf.cpp:2314-2336)
        return 2 * math.pi * np.linalg.inv(self.supercell).T

    @property
    def vol(self):
        return float(abs(np.linalg.det(self.supercell)))

    @property
    def ntot(self):
        return int(np.prod(self.numGrid))

    @property
    def ntotFine(self):
        return int(np.prod(self.numGridFine))


def kgrid(n: int) -> np.ndarray:
    """Signed FFT frequencies with Nyquist at +n/2 (fourier.cpp:124-133)."""
    k = np.arange(n, dtype=np.float64)
    k[n // 2 + 1:] -= n
    return k


def gvec_r2c(dm: Domain, fine: bool = False):
    """Cartesian G on the R2C half grid, shape (n2, n1, n0/2+1, 3)
    (fourier.cpp:200-238 / 365-380)."""
    n0, n1, n2 = dm.numGridFine if fine else dm.numGrid
    k0 = kgrid(n0)[: n0 // 2 + 1]
    k1 = kgrid(n1)
    k2 = kgrid(n2)
    m = np.stack(np.meshgrid(k2, k1, k0, indexing="ij")[::-1], axis=-1)  # (m0,m1,m2)
    rec = dm.recipcell
    # gmesh_car[ip] = sum_jp recipcell(jp, ip) * gmesh[jp]
    return m @ rec


def gvec_full(dm: Domain, fine: bool = False):
    n0, n1, n2 = dm.numGridFine if fine else dm.numGrid
    m = np.stack(np.meshgrid(kgrid(n2), kgrid(n1), kgrid(n0), indexing="ij")[::-1], axis=-1)
    return m @ dm.recipcell


def ekin_teter(dm: Domain):
    """``KohnSham::CalculateEkin`` (src/SCF/hamiltonian.cpp:2630-2667):
    ekin = |G|^2/2, teter = b/(b+16 a^4), a = |G|^2,
    b = 27 + a(18 + a(12 + 8a))."""
    g = gvec_r2c(dm)
    ekin = 0.5 * np.sum(g * g, axis=-1)
    a = ekin * 2.0
    b = 27.0 + a * (18.0 + a * (12.0 + a * 8.0))
    teter = b / (b + 16.0 * a ** 4)
    return ekin, teter


# ---------------------------------------------------------------------------
# FFTWExecute normalisations (src/SCF/fourier.cpp:695-764)
# ---------------------------------------------------------------------------
_FFT = {"backend": "numpy", "workers": 1}


def set_fft_backend(backend: str = "numpy", workers: int = 1):
    """FFT engine of r2c / c2r: "numpy" (pocketfft, one thread) or "scipy"
    (scipy.fft's pocketfft with `workers` threads over the batch and axes).
    Both compute the same transforms; the choice only changes the CPU time."""
    if backend not in ("numpy", "scipy"):
        raise ValueError(backend)
    _FFT["backend"], _FFT["workers"] = backend, int(workers)


def _rfftn(x):
    if _FFT["backend"] == "scipy":
        import scipy.fft as sf
        return sf.rfftn(x, axes=(-3, -2, -1), workers=_FFT["workers"])
    return np.fft.rfftn(x, axes=(-3, -2, -1))


def _irfftn(X, s):
    if _FFT["backend"] == "scipy":
        import scipy.fft as sf
        return sf.irfftn(X, s=s, axes=(-3, -2, -1), workers=_FFT["workers"])
    return np.fft.irfftn(X, s=s, axes=(-3, -2, -1))


def r2c(x, dm: Domain, fine: bool = False):
    """forward R2C with factor vol/N; x has shape (..., n2, n1, n0)."""
    N = dm.ntotFine if fine else dm.ntot
    return _rfftn(x) * (dm.vol / N)


def c2r(X, dm: Domain, fine: bool = False):
    """backward C2R (unnormalised FFTW) with factor 1/vol."""
    n = dm.numGridFine if fine else dm.numGrid
    N = n[0] * n[1] * n[2]
    return _irfftn(X, (n[2], n[1], n[0])) * (N / dm.vol)


# ---------------------------------------------------------------------------
# IP_c2f / IP_f2c  (src/utility.cpp:3150-3211 / 3215-3275)
# ---------------------------------------------------------------------------
def ip_c2f_loop(Nc, Nf, tilde):
    """Literal restatement of IP_c2f on flat half spectra (small grids only)."""
    tildef = np.zeros((Nf[0] // 2 + 1) * Nf[1] * Nf[2], dtype=np.complex128)
    cjF = Nf[1] - Nc[1] // 2
    ckF = Nf[2] - Nc[2] // 2
    fac = 2.0
    hc0, hf0 = Nc[0] // 2 + 1, Nf[0] // 2 + 1
    for k in range(Nc[2]):
        for j in range(Nc[1]):
            for i in range(hc0):
                ptrc = i + j * hc0 + k * hc0 * Nc[1]
                iF = i
                jF = j if j <= Nc[1] // 2 else Nf[1] - Nc[1] + j
                kF = k if k <= Nc[2] // 2 else Nf[2] - Nc[2] + k
                ptrF = iF + jF * hf0 + kF * hf0 * Nf[1]
                tildef[ptrF] = tilde[ptrc]
                xi, yj, zk = iF == Nc[0] // 2, jF == Nc[1] // 2, kF == Nc[2] // 2
                if xi and yj and zk:
                    tildef[ptrF] /= fac
                elif xi and yj:
                    tildef[ptrF] /= fac
                elif xi and zk:
                    tildef[ptrF] /= fac
                elif yj and zk:
                    tildef[ptrF] /= fac
                    tildef[iF + cjF * hf0 + ckF * hf0 * Nf[1]] = tilde[ptrc] / fac
                elif xi:
                    tildef[ptrF] /= fac
                elif yj:
                    tildef[ptrF] /= fac
                    tildef[iF + cjF * hf0 + kF * hf0 * Nf[1]] = tilde[ptrc] / fac
                elif zk:
                    tildef[ptrF] /= fac
                    tildef[iF + jF * hf0 + ckF * hf0 * Nf[1]] = tilde[ptrc] / fac
    return tildef


def ip_f2c_loop(Nc, Nf, tilde, tildef):
    """Literal restatement of IP_f2c (accumulates into ``tilde`` in place)."""
    cjF = Nf[1] - Nc[1] // 2
    ckF = Nf[2] - Nc[2] // 2
    hc0, hf0 = Nc[0] // 2 + 1, Nf[0] // 2 + 1
    for k in range(Nc[2]):
        for j in range(Nc[1]):
            for i in range(hc0):
                ptrc = i + j * hc0 + k * hc0 * Nc[1]
                iF = i
                jF = j if j <= Nc[1] // 2 else Nf[1] - Nc[1] + j
                kF = k if k <= Nc[2] // 2 else Nf[2] - Nc[2] + k
                f1 = iF + jF * hf0 + kF * hf0 * Nf[1]
                xi, yj, zk = i == Nc[0] // 2, j == Nc[1] // 2, k == Nc[2] // 2
                if xi and yj and zk:
                    tilde[ptrc] += complex(tildef[f1].real, 0.0)
                elif xi and yj:
                    kF2 = (Nf[2] - kF) % Nf[2]
                    f2 = iF + jF * hf0 + kF2 * hf0 * Nf[1]
                    tilde[ptrc] += 0.5 * (tildef[f1] + np.conj(tildef[f2]))
                elif xi and zk:
                    jF2 = (Nf[1] - jF) % Nf[1]
                    f2 = iF + jF2 * hf0 + kF * hf0 * Nf[1]
                    tilde[ptrc] += 0.5 * (tildef[f1] + np.conj(tildef[f2]))
                elif yj and zk:
                    f2 = iF + cjF * hf0 + ckF * hf0 * Nf[1]
                    tilde[ptrc] += 0.5 * (tildef[f1] + tildef[f2])
                elif xi:
                    jF2 = (Nf[1] - jF) % Nf[1]
                    kF2 = (Nf[2] - kF) % Nf[2]
                    f2 = iF + jF2 * hf0 + kF2 * hf0 * Nf[1]
                    tilde[ptrc] += 0.5 * (tildef[f1] + np.conj(tildef[f2]))
                elif yj:
                    f2 = iF + cjF * hf0 + kF * hf0 * Nf[1]
                    tilde[ptrc] += 0.5 * (tildef[f1] + tildef[f2])
                elif zk:
                    f2 = iF + jF * hf0 + ckF * hf0 * Nf[1]
                    tilde[ptrc] += 0.5 * (tildef[f1] + tildef[f2])
                else:
                    tilde[ptrc] += tildef[f1]
    return tilde


class IPMaps:
    """Vectorised IP_c2f / IP_f2c for batched half spectra (same arithmetic as
    the loop forms above; cross-checked in tests)."""

    def __init__(self, Nc, Nf):
        self.Nc, self.Nf = tuple(Nc), tuple(Nf)
        hc0, hf0 = Nc[0] // 2 + 1, Nf[0] // 2 + 1
        k, j, i = np.meshgrid(np.arange(Nc[2]), np.arange(Nc[1]), np.arange(hc0), indexing="ij")
        k, j, i = k.ravel(), j.ravel(), i.ravel()
        jF = np.where(j <= Nc[1] // 2, j, Nf[1] - Nc[1] + j)
        kF = np.where(k <= Nc[2] // 2, k, Nf[2] - Nc[2] + k)
        iF = i
        cjF, ckF = Nf[1] - Nc[1] // 2, Nf[2] - Nc[2] // 2
        xi, yj, zk = i == Nc[0] // 2, j == Nc[1] // 2, k == Nc[2] // 2
        flat = lambda a, b, c: a + b * hf0 + c * hf0 * Nf[1]
        f1 = flat(iF, jF, kF)
        nyq = xi | yj | zk
        # --- c2f: primary target with factor, optional duplicate ---
        self.c2f_t1 = f1
        self.c2f_w1 = np.where(nyq, 0.5, 1.0)
        dup_yz = yj & zk & ~xi
        dup_y = yj & ~zk & ~xi
        dup_z = zk & ~yj & ~xi
        t2 = np.full(f1.shape, -1)
        t2[dup_yz] = flat(iF, np.full_like(jF, cjF), np.full_like(kF, ckF))[dup_yz]
        t2[dup_y] = flat(iF, np.full_like(jF, cjF), kF)[dup_y]
        t2[dup_z] = flat(iF, jF, np.full_like(kF, ckF))[dup_z]
        self.c2f_dup = np.nonzero(t2 >= 0)[0]
        self.c2f_t2 = t2[self.c2f_dup]
        # --- f2c ---
        case = np.zeros(f1.shape, dtype=np.int8)   # 0 plain, 1 real, 2 avg+conj, 3 avg
        f2 = np.full(f1.shape, 0)
        allc = xi & yj & zk
        case[allc] = 1
        m = xi & yj & ~zk
        case[m] = 2; f2[m] = flat(iF, jF, (Nf[2] - kF) % Nf[2])[m]
        m = xi & zk & ~yj
        case[m] = 2; f2[m] = flat(iF, (Nf[1] - jF) % Nf[1], kF)[m]
        m = yj & zk & ~xi
        case[m] = 3; f2[m] = flat(iF, np.full_like(jF, cjF), np.full_like(kF, ckF))[m]
        m = xi & ~yj & ~zk
        case[m] = 2; f2[m] = flat(iF, (Nf[1] - jF) % Nf[1], (Nf[2] - kF) % Nf[2])[m]
        m = yj & ~xi & ~zk
        case[m] = 3; f2[m] = flat(iF, np.full_like(jF, cjF), kF)[m]
        m = zk & ~xi & ~yj
        case[m] = 3; f2[m] = flat(iF, jF, np.full_like(kF, ckF))[m]
        self.f1, self.f2, self.case = f1, f2, case
        self.nhc = hc0 * Nc[1] * Nc[2]
        self.nhf = hf0 * Nf[1] * Nf[2]

    def c2f(self, Xc):
        """Xc: (..., nhc) -> (..., nhf)"""
        sh = Xc.shape[:-1]
        Y = np.zeros(sh + (self.nhf,), dtype=np.complex128)
        Y[..., self.c2f_t1] = Xc * self.c2f_w1
        Y[..., self.c2f_t2] = Xc[..., self.c2f_dup] * 0.5
        return Y

    def f2c(self, Yf):
        """Yf: (..., nhf) -> contribution (..., nhc) to accumulate."""
        a = Yf[..., self.f1]
        b = Yf[..., self.f2]
        out = a.copy()
        c = self.case
        out[..., c == 1] = a[..., c == 1].real
        out[..., c == 2] = 0.5 * (a[..., c == 2] + np.conj(b[..., c == 2]))
        out[..., c == 3] = 0.5 * (a[..., c == 3] + b[..., c == 3])
        return out


# ---------------------------------------------------------------------------
# Atoms, projectors, pseudocharge
# ---------------------------------------------------------------------------
@dataclass
class Atom:
    znuc: int
    pos: np.ndarray            # Cartesian, bohr


@dataclass
class NonlocalPP:
    """One ``vnlList`` entry: SparseVec (idx, VAL/DX/DY/DZ) and weight
    (include/periodtable.hpp:62-63, include/utility.hpp:127-151)."""
    idx: np.ndarray
    val: np.ndarray            # (npts, 4): VAL, DX, DY, DZ
    wgt: float
    disp: np.ndarray = None    # (npts, 3): grid point - atom, Cartesian (vnlPos, periodtable.cpp:1096)


def nonlocal_pp(atom: Atom, dm: Domain, sp: _hgh.HGHSpecies):
    """``PeriodTable::CalculateNonlocalPP`` (src/SCF/periodtable.cpp:994-1240),
    L0 and L1 channels."""
    nG = dm.numGridFine
    rec = dm.recipcell
    sc = dm.supercell
    pos = np.linalg.solve(sc.T, atom.pos)     # fractional (pos_frac)
    R = sp.wavcut
    nmin, nmax = [], []
    for d in range(3):
        w = R / (2 * math.pi) * math.sqrt(float(np.sum(rec[d] ** 2)))
        nmin.append(int(cround((pos[d] - w) * nG[d])))
        nmax.append(int(cround((pos[d] + w) * nG[d])))
    ks = np.arange(nmin[2], nmax[2] + 1)
    js = np.arange(nmin[1], nmax[1] + 1)
    is_ = np.arange(nmin[0], nmax[0] + 1)
    K, J, I = np.meshgrid(ks, js, is_, indexing="ij")
    K, J, I = K.ravel(), J.ravel(), I.ravel()
    frac = np.stack([I / nG[0], J / nG[1], K / nG[2]], axis=-1) - pos
    car = frac @ sc                          # gridpos_car[ip] = sum_jp supercell(jp,ip) g[jp]
    dist = np.sqrt(np.sum(car * car, axis=-1))
    sel = dist < R
    ii, jj, kk = I[sel] % nG[0], J[sel] % nG[1], K[sel] % nG[2]
    idx = (ii + jj * nG[0] + kk * nG[0] * nG[1]).astype(np.int64)
    rad = dist[sel]
    xx, yy, zz = car[sel, 0], car[sel, 1], car[sel, 2]
    disp = car[sel].copy()
    out = []
    big = rad > MIN_RADIAL
    safe = np.where(big, rad, 1.0)
    for k, (l, h, _, _) in enumerate(sp.proj):
        val = _hgh.spl_eval(sp, ("val", k), rad)
        der = _hgh.spl_eval(sp, ("der", k), rad)
        if l == _hgh.TYPE_L0:
            coef = math.sqrt(1.0 / (4 * math.pi))
            dv = np.zeros((rad.size, 4))
            dv[:, 0] = coef * val
            dv[:, 1] = np.where(big, coef * der * xx / safe, 0.0)
            dv[:, 2] = np.where(big, coef * der * yy / safe, 0.0)
            dv[:, 3] = np.where(big, coef * der * zz / safe, 0.0)
            out.append(NonlocalPP(idx, dv, h, disp))
        elif l == _hgh.TYPE_L1:
            coef = math.sqrt(3.0 / (4 * math.pi))
            dvr = der - val / safe
            for comp, (cc, dirn) in enumerate(((zz, 2), (xx, 0), (yy, 1))):
                dv = np.zeros((rad.size, 4))
                u = cc / safe
                comps = (xx / safe, yy / safe, zz / safe)
                dv[:, 0] = np.where(big, coef * u * val, 0.0)
                for a in range(3):
                    t = coef * dvr * u * comps[a]
                    if a == dirn:
                        t = t + coef * val / safe
                    dv[:, 1 + a] = np.where(big, t, coef * der if a == dirn else 0.0)
                out.append(NonlocalPP(idx, dv, h, disp))
        else:
            raise NotImplementedError("only L0/L1 channels (Si, Al HGH)")
    return out


def pseudo_charge(atom: Atom, dm: Domain, sp: _hgh.HGHSpecies):
    """``PeriodTable::CalculatePseudoCharge`` (src/SCF/periodtable.cpp:282-377)
    with the Cartesian minimum-image distances that ``CalculateVLocal`` uses
    (periodtable.cpp:669-703); the reference subtracts a Cartesian position
    from fractional grid coordinates here, which is restated as fixed."""
    N = dm.numGridFine
    L = dm.length
    R = sp.rhocut
    dist = []
    for d in range(3):
        x = np.arange(N[d]) / N[d] * L[d] - atom.pos[d]
        x = x - cround(x / L[d]) * L[d]
        dist.append(x)
    Z, Y, X = np.meshgrid(dist[2], dist[1], dist[0], indexing="ij")
    r = np.sqrt(X * X + Y * Y + Z * Z).ravel()
    sel = np.nonzero(r <= R)[0]
    rad = r[sel]
    val = _hgh.spl_eval(sp, "rho", rad)
    der = _hgh.spl_eval(sp, "drho", rad)
    big = rad > MIN_RADIAL
    safe = np.where(big, rad, 1.0)
    dv = np.zeros((sel.size, 4))
    dv[:, 0] = val
    for a, comp in enumerate((X.ravel()[sel], Y.ravel()[sel], Z.ravel()[sel])):
        dv[:, 1 + a] = np.where(big, der * comp / safe, 0.0)
    return sel.astype(np.int64), dv


# ---------------------------------------------------------------------------
# H*psi  (Spinor::AddMultSpinorFineR2C, src/SCF/spinor.cpp:377-525)
# ---------------------------------------------------------------------------
@dataclass
class HamTables:
    dm: Domain
    ekin: np.ndarray                  # (n2, n1, n0/2+1)
    teter: np.ndarray
    vtot: np.ndarray                  # (N_fine,)
    pseudo: list                      # list[list[NonlocalPP]] per atom
    ip: IPMaps = field(default=None)

    def __post_init__(self):
        if self.ip is None:
            self.ip = IPMaps(self.dm.numGrid, self.dm.numGridFine)


def add_mult_spinor_fine_r2c(T: HamTables, psi: np.ndarray, a3: np.ndarray | None = None):
    """a3 += (kinetic + V_loc + V_nl) psi for a block of bands.

    psi: (nb, ntot) real, each row one band in reference grid order.
    Follows spinor.cpp:405-522 step by step, batched over bands.
    """
    dm = T.dm
    n0, n1, n2 = dm.numGrid
    N0, N1, N2 = dm.numGridFine
    nb = psi.shape[0]
    Xc = r2c(psi.reshape(nb, n2, n1, n0), dm)                     # :421
    Xf = T.ip.c2f(Xc.reshape(nb, -1)).reshape(nb, N2, N1, N0 // 2 + 1)   # :426-431
    psiF = c2r(Xf, dm, fine=True).reshape(nb, -1)                  # :444
    upd = psiF * T.vtot[None, :]                                   # :449-456
    fac = dm.vol / dm.ntotFine
    for atom_pp in T.pseudo:                                       # :459-482
        idx = atom_pp[0].idx
        # one index set per atom: gather once; a set without repeated points
        # takes a plain indexed add (the same single addition per point)
        uniq = len(np.unique(idx)) == len(idx)
        sub = psiF[:, idx]
        for pp in atom_pp:
            w = sub @ pp.val[:, 0]
            w = w * fac * pp.wgt
            if uniq and pp.idx is idx:
                upd[:, idx] += w[:, None] * pp.val[None, :, 0]
            else:
                np.add.at(upd, (slice(None), pp.idx), w[:, None] * pp.val[None, :, 0])
    Xc = Xc * T.ekin[None]                                         # :485-488
    Yf = r2c(upd.reshape(nb, N2, N1, N0), dm, fine=True)           # :493-498
    Xc = Xc.reshape(nb, -1) + T.ip.f2c(Yf.reshape(nb, -1))         # :501-506
    out = c2r(Xc.reshape(nb, n2, n1, n0 // 2 + 1), dm).reshape(nb, -1)   # :517
    if a3 is None:
        return out
    a3 += out                                                      # :519
    return a3


def add_teter_precond(T: HamTables, r: np.ndarray, a3: np.ndarray | None = None):
    """``Spinor::AddTeterPrecond`` (src/SCF/spinor.cpp:310-346)."""
    dm = T.dm
    n0, n1, n2 = dm.numGrid
    nb = r.shape[0]
    X = r2c(r.reshape(nb, n2, n1, n0), dm) * T.teter[None]
    out = c2r(X, dm).reshape(nb, -1)
    if a3 is None:
        return out
    a3 += out
    return a3


def wfn_ecut_filter(T: HamTables, psi: np.ndarray, ecut: float):
    """The wavefunction cut-off filter of ``KohnSham::MultSpinor``
    (src/SCF/hamiltonian.cpp:3090-3116 on psi, :3240-3265 on a3): forward R2C,
    coefficients with gkkR2C = |G|^2/2 > ecut set to zero, backward C2R (the
    two normalisations cancel).  Switched on for CheFSI with
    wfn_cutoff_ = Ecut_Wavefunction (hamiltonian.cpp:316-321)."""
    dm = T.dm
    n0, n1, n2 = dm.numGrid
    nb = psi.shape[0]
    X = r2c(psi.reshape(nb, n2, n1, n0), dm)
    X[:, T.ekin > ecut] = 0.0
    return c2r(X, dm).reshape(nb, -1)


def mult_spinor(T: HamTables, psi: np.ndarray, wfn_ecut: float | None = None):
    """``KohnSham::MultSpinor`` (src/SCF/hamiltonian.cpp:3059-3268) without
    hybrid exchange: a3 = 0, then a2.  With ``wfn_ecut`` the exit filter is
    applied to a3 (:3240-3265), i.e. a3 = P H psi; the reference's first call
    also replaces psi by P psi in place (:3090-3116), which a caller does with
    ``wfn_ecut_filter`` before the first application."""
    out = add_mult_spinor_fine_r2c(T, psi, np.zeros_like(psi))
    if wfn_ecut is not None:
        out = wfn_ecut_filter(T, out, wfn_ecut)
    return out


# ---------------------------------------------------------------------------
# Synthetic systems (seeded)
# ---------------------------------------------------------------------------
DIAMOND_FRAC = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                         [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
FCC_FRAC = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]])


def make_crystal(kind: str, reps, a: float, disp: float, seed: int):
    """Si diamond or fcc Al supercell with seeded uniform displacements in
    [-disp, disp]^3 (Philox stream)."""
    rng = np.random.Generator(np.random.Philox(seed))
    base = DIAMOND_FRAC if kind == "Si" else FCC_FRAC
    znuc = 14 if kind == "Si" else 13
    reps = tuple(reps)
    L = np.array([a * reps[0], a * reps[1], a * reps[2]], dtype=np.float64)
    pos = []
    for cz in range(reps[2]):
        for cy in range(reps[1]):
            for cx in range(reps[0]):
                for f in base:
                    pos.append((np.array([cx, cy, cz]) + f) * a)
    pos = np.array(pos)
    pos = pos + rng.uniform(-disp, disp, size=pos.shape)
    return L, znuc, pos


def random_orthonormal_psi(ntot: int, nb: int, seed: int):
    """Gaussian psi (Philox) orthonormalised by Cholesky-QR: rows are bands."""
    rng = np.random.Generator(np.random.Philox(seed))
    X = rng.standard_normal((ntot, nb))
    S = X.T @ X
    U = np.linalg.cholesky(S).T                 # S = U^T U
    X = np.linalg.solve(U.T, X.T).T             # X U^{-1}
    return np.ascontiguousarray(X.T)


def build_tables(L, znuc, pos, numGrid, numGridFine, vtot=None, seed_v=None):
    """Domain + Fourier tables + projectors for a homogeneous crystal."""
    dm = Domain(tuple(L), tuple(numGrid), tuple(numGridFine))
    sp = _hgh.hgh_table(znuc)
    ekin, teter = ekin_teter(dm)
    pseudo = [nonlocal_pp(Atom(znuc, p), dm, sp) for p in pos]
    if vtot is None:
        rng = np.random.Generator(np.random.Philox(seed_v if seed_v is not None else 1))
        vtot = rng.uniform(-1.0, 0.5, size=dm.ntotFine)
    return HamTables(dm, ekin, teter, np.asarray(vtot, dtype=np.float64), pseudo), sp
