"""FP64 NumPy restatement of the reference's complex (k-point) H*psi.

Test infrastructure (see ``oracle/__init__.py``).  Follows:
  * Spinor::AddMultSpinorFine, complex version, real-space branch
    (src/SCF/spinor_complex.cpp:292-542): unnormalised forward C2C FFT on the
    coarse grid, placement into the fine spectrum by idxFineGrid
    (src/SCF/fourier.cpp:291-311), backward fine FFT x 1/N_fine, V_loc,
    nonlocal projectors with the Bloch phase (weights vol / N_fine), kinetic
    1/2 |k+G|^2 on the coarse spectrum, forward fine FFT, pick by idxFineGrid,
    backward coarse FFT x 1/N_coarse.
  * KohnSham::CalculateEkin, complex version (src/SCF/hamiltonian_complex.cpp:
    234-277): ekin = 1/2 |k+G|^2 and Teter b / (b + 16 a^4), a = |k+G|^2.
  * Bloch phase e^{i k.(r - R_a)} with r - R_a the unwrapped grid displacement
    (PeriodTable::CalculateNonlocalPP, src/SCF/periodtable.cpp:1104-1121).
"""
from __future__ import annotations

import numpy as np

from . import forces, pw


def ekin_teter_k(dm: pw.Domain, k):
    g = pw.gvec_full(dm) + np.asarray(k, np.float64)
    ekin = 0.5 * np.sum(g * g, axis=-1)
    a = 2.0 * ekin
    b = 27.0 + a * (18.0 + a * (12.0 + a * 8.0))
    return ekin.ravel(), (b / (b + 16.0 * a ** 4)).ravel()


def mult_spinor_k(T: pw.HamTables, k, psi: np.ndarray) -> np.ndarray:
    """H(k) psi for complex bands psi (nb, N_coarse)."""
    dm = T.dm
    n0, n1, n2 = dm.numGrid
    N0, N1, N2 = dm.numGridFine
    nb = psi.shape[0]
    place = forces._placement(dm)
    ek, _ = ekin_teter_k(dm, k)
    kv = np.asarray(k, np.float64)
    X = np.fft.fftn(psi.reshape(nb, n2, n1, n0), axes=(1, 2, 3)).reshape(nb, -1)
    Y = np.zeros((nb, dm.ntotFine), complex)
    Y[:, place] = X
    pf = np.fft.ifftn(Y.reshape(nb, N2, N1, N0), axes=(1, 2, 3)).reshape(nb, -1)
    upd = pf * T.vtot[None, :]
    w = dm.vol / dm.ntotFine
    for app in T.pseudo:
        if not app:
            continue
        idx = app[0].idx
        ph = np.exp(1j * (app[0].disp @ kv))
        pt = pf[:, idx] * ph[None, :]
        acc = np.zeros((nb, idx.size), complex)
        for pp in app:
            beta = pp.val[:, 0]
            weight = (pt @ beta) * w * pp.wgt
            acc += weight[:, None] * beta[None, :]
        upd[:, idx] += np.conj(ph)[None, :] * acc
    Xk = X * ek[None, :]
    F = np.fft.fftn(upd.reshape(nb, N2, N1, N0), axes=(1, 2, 3)).reshape(nb, -1)
    Xk += F[:, place]
    return np.fft.ifftn(Xk.reshape(nb, n2, n1, n0), axes=(1, 2, 3)).reshape(nb, -1)


def random_complex_psi(ntot: int, nb: int, seed: int):
    rng = np.random.Generator(np.random.Philox(seed))
    Z = rng.standard_normal((ntot, nb)) + 1j * rng.standard_normal((ntot, nb))
    Q, _ = np.linalg.qr(Z)
    return np.ascontiguousarray(Q.T)
