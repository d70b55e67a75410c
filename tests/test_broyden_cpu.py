"""Broyden potential mixing and the density-change norm of the oracle
(oracle/scf.py: SCF::BroydenMix, RhoDdot, CalculateError,
src/SCF/scf.cpp:2144-2296, 2368-2396), on the CPU."""
import math

import numpy as np

from oracle import pw, scf


def _dm():
    return pw.Domain((10.26, 10.26, 10.26), (12, 12, 12), (24, 24, 24))


def test_first_step_is_the_filtered_linear_mix():
    dm = _dm()
    ecut = 5.0
    rng = np.random.Generator(np.random.Philox(3))
    vin, vout = rng.standard_normal(dm.ntotFine), rng.standard_normal(dm.ntotFine)
    st = scf.BroydenState(8)
    vm = scf.broyden(dm, 1, 0.7, vin, vout, st, ecut)
    gkk = scf.gkk_fine(dm).reshape(-1)
    X = np.fft.fftn((vin + 0.7 * (vout - vin)).reshape(24, 24, 24)).reshape(-1)
    X[gkk >= 4 * ecut] = 0
    np.testing.assert_allclose(vm, np.fft.ifftn(X.reshape(24, 24, 24)).real.reshape(-1), atol=1e-13)


def test_broyden_history_slots_and_linear_problem():
    """On a linear fixed-point map v -> K v + c (K symmetric, contractive, acting
    inside the density sphere) the mixed iterates converge, and the history
    wraps around its mix_dim slots."""
    dm = _dm()
    ecut = 5.0
    N = dm.ntotFine
    gkk = scf.gkk_fine(dm).reshape(-1)
    sph = gkk < 4 * ecut
    rng = np.random.Generator(np.random.Philox(9))
    lam = np.where(sph, 0.9 * np.tanh(1.0 / (1.0 + gkk)), 0.0)        # spectral contraction

    def F(v):
        X = np.fft.fftn(v.reshape(24, 24, 24)).reshape(-1) * lam
        return np.fft.ifftn(X.reshape(24, 24, 24)).real.reshape(-1) + c

    Xc = np.fft.fftn(rng.standard_normal(N).reshape(24, 24, 24)).reshape(-1)
    Xc[~sph] = 0
    c = np.fft.ifftn(Xc.reshape(24, 24, 24)).real.reshape(-1)
    st = scf.BroydenState(3)
    v = np.zeros(N)
    for it in range(1, 31):
        v = scf.broyden(dm, it, 0.7, v, F(v), st, ecut)
    assert np.abs(F(v) - v).max() < 1e-8 * np.abs(c).max()
    assert all(x is not None for x in st.df)


def test_scf_norm_definition():
    dm = _dm()
    rng = np.random.Generator(np.random.Philox(4))
    d = rng.standard_normal(dm.ntotFine)
    gkk = scf.gkk_fine(dm).reshape(-1)
    X = np.fft.fftn(d.reshape(24, 24, 24)).reshape(-1) * (dm.vol / dm.ntotFine) / dm.vol
    m = (gkk < 20.0) & (gkk != 0)
    ref = math.pi * dm.vol * np.sum(np.abs(X[m]) ** 2 / gkk[m])
    assert abs(scf.scf_norm(dm, d, 5.0) - ref) <= 1e-13 * ref
