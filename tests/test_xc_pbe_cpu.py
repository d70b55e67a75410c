"""PBE exchange-correlation of the oracle (oracle/scf.py) pinned to the
reference's own internal functions and checked as a functional derivative.

* Golden vectors (tests/golden/ref_xc_pbe.npz) come from VExchange_sla,
  VCorrelation_pw, VGCExchange_pbx and VGCCorrelation_pbc compiled from
  src/utility.cpp:3913-4244 (tests/golden/make_golden.py).  Tolerance 1e-12
  relative, 1e-9 for the correlation v2 term, whose (xy - qy) difference
  cancels for y = A t^2 >> 1 at the low-density edge.
* V_xc is the derivative of E_xc = sum eps rho dV: central differences along
  a smooth direction agree to 1e-6 relative (on a 32^3 grid whose Nyquist
  planes fall outside the 4 Ecut sphere, so the spectral gradient is exactly
  anti-adjoint)."""
import math

import numpy as np

from oracle import pw, scf

from pathlib import Path

GOLD = Path(__file__).resolve().parent / "golden" / "ref_xc_pbe.npz"


def test_point_functions_match_the_reference():
    d = np.load(GOLD)
    rs, rho, g2, out = d["rs"], d["rho"], d["grho2"], d["out"]
    ux, vx = scf.slater(rs)
    uc, vc = scf.pw92(rs)
    ex, v1x, v2x = scf.pbe_x(rho, g2)
    ec, v1c, v2c = scf.pbe_c(rho, g2)
    mine = np.stack([ux, vx, uc, vc, ex, v1x, v2x, ec, v1c, v2c], 1)
    rel = np.abs(mine - out) / np.abs(out)
    tol = np.full(10, 1e-12)
    tol[9] = 1e-9
    assert np.all(rel.max(axis=0) <= tol), rel.max(axis=0)


def test_thresholds_of_the_point_routine():
    rho = np.array([1e-11, 5e-7, 0.02, 0.02, -0.02])
    sigma = np.array([1.0, 1.0, 1e-11, 1e-4, 1e-4])
    eps, v1, v2 = scf.xc_pbe_point(rho, sigma)
    assert eps[0] == 0 and v1[0] == 0 and v2[0] == 0          # |rho| <= 1e-10: nothing
    assert v2[1] == 0 and v2[2] == 0                          # LDA part only
    rs = (3 / (4 * math.pi * 0.02)) ** (1 / 3)
    ux, vx = scf.slater(rs)
    uc, vc = scf.pw92(rs)
    assert abs(eps[2] - (ux + uc)) < 1e-15 and abs(v1[2] - (vx + vc)) < 1e-15
    assert v2[3] != 0 and eps[3] == eps[4]                    # |rho| enters the gradient part


def _smooth(dm, rng, amp, ecut):
    g = pw.gvec_full(dm, fine=True)
    gkk = 0.5 * np.sum(g * g, axis=-1)
    X = (rng.standard_normal(gkk.shape) + 1j * rng.standard_normal(gkk.shape)) * np.exp(-gkk / 2.0)
    X[gkk > 4 * ecut] = 0
    x = np.fft.ifftn(X).real.reshape(-1)
    return amp * x / np.abs(x).max()


def test_potential_is_the_functional_derivative():
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)
    dm = pw.Domain(tuple(L), (16, 16, 16), (32, 32, 32))
    ecut = 10.0
    rng = np.random.Generator(np.random.Philox(5))
    rho = 0.03 + _smooth(dm, rng, 0.02, ecut)
    dlt = _smooth(dm, rng, 1.0, ecut)
    w = dm.vol / dm.ntotFine

    def exc(r):
        e, _ = scf.xc_pbe(dm, r, ecut)
        return float(np.sum(e * r) * w)

    _, v = scf.xc_pbe(dm, rho, ecut)
    h = 1e-5
    fd = (exc(rho + h * dlt) - exc(rho - h * dlt)) / (2 * h)
    an = float(np.sum(v * dlt) * w)
    assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)


def test_uniform_density_reduces_to_lda():
    dm = pw.Domain((10.0, 10.0, 10.0), (12, 12, 12), (24, 24, 24))
    rho = np.full(dm.ntotFine, 0.011)
    eps, v = scf.xc_pbe(dm, rho, 5.0)
    rs = (3 / (4 * math.pi * 0.011)) ** (1 / 3)
    ux, vx = scf.slater(rs)
    uc, vc = scf.pw92(rs)
    np.testing.assert_allclose(eps, ux + uc, rtol=1e-14)
    np.testing.assert_allclose(v, vx + vc, rtol=1e-12)
