"""Short-range PBE exchange of HSE06 (test infrastructure: the oracle).

Restates ``pbexsr`` and ``wpbe_analy_erfc_approx_grad`` (src/utility.cpp:
3340-3846), called by KohnSham::CalculateXC for XC_HYB_GGA_XC_HSE06 with
omega = 0.106 and fraction 0.25 (src/SCF/hamiltonian.cpp:1614-1627): the
semilocal HSE06 functional is PBE minus 0.25 times the erfc-screened PBE
exchange.

The screened enhancement factor follows Heyd, Scuseria and Ernzerhof (J.
Chem. Phys. 118, 8207 (2003); 124, 219906 (2006)): the Ernzerhof-Perdew
exchange hole (J. Chem. Phys. 109, 3313 (1998)) in y = k_F u,

    J(s, y) = [-A / (y^2 (1 + 4/9 A y^2)) + (A / y^2 + B + C (1 + s^2 F) y^2
               + (E + s^2 EG) y^4) e^{-D y^2}] e^{-s^2 H y^2},

    F_x(s, w) = -8/9 int_0^inf y J(s, y) erfc(w y) dy,   w = omega / k_F,

with the published parameters (A ... E, the rational H(s), F = Fc1 H + Fc2,
and EG = E G(s) fixed by the hole normalisation, a quadratic series below
s = 0.08).  As in the reference, erfc is exact in the regular part and
replaced by the fit (1 + sum_k ea_k x^k) e^{-eb1 x^2} in the singular
A / y^2 part.  The integrals are evaluated here in closed forms derived for
this restatement (not the reference's term-by-term expressions):

  regular part  int y^{2n+1} e^{-a y^2} erfc(w y) dy
                  = n! / (2 a^{n+1}) [1 - (w / r) sum_{k<=n} binom(2k,k) / 4^k (a / r^2)^k],
                r = sqrt(a + w^2);
  singular part A sum_k ea_k w^k T_k with
                T_0 = 1/2 ln(q / p) + 1/2 e^x E1(x),
                T_k = M_{k-1}(p) - L_{k-1}(q)   (k >= 1),
                p = a + eb1 w^2, q = s^2 H + eb1 w^2, lambda = 4 A / 9, x = q / lambda,
                M_j(q) = Gamma((j+1)/2) / (2 q^{(j+1)/2}),
                L_j(q) = int y^j e^{-q y^2} / (1 + lambda y^2) dy:
                L_0 = pi / (2 sqrt(lambda)) erfcx(sqrt x), L_1 = e^x E1(x) / (2 lambda),
                L_{j+2} = (M_j(q) - L_j) / lambda.

The derivatives d F / d s and d F / d w come from forward-mode dual numbers;
d F / d rho = d F / d w * (-w / (3 rho)).  Pinned against the reference's
own functions compiled from its sources (oracle/build_ref.py ->
tests/golden/ref_xc_hse.npz) and against direct quadrature of the defining
integrals (tests/test_xc_hse_cpu.py).
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erfcx, exp1

# Ernzerhof-Perdew hole and HSE erfc-fit parameters (the published values,
# which the reference uses too)
A, B, C, D, E = 1.0161144, -3.7170836e-1, -7.7215461e-2, 5.7786348e-1, -5.1955731e-2
HA = (9.79681e-3, 4.10834e-2, 1.87440e-1, 1.20824e-3, 3.47188e-2)
FC1, FC2 = 6.4753871, 4.7965830e-1
EGA = (-2.628417880e-2, -7.117647788e-2, 8.534541323e-2)
EG_SCUT = 8.0e-2
EA = (-1.128223946706117, 1.452736265762971, -1.243162299390327, 0.971824836115601,
      -0.568861079687373, 0.246880514820192, -0.065032363850763, 0.008401793031216)
EB1, EB1_FAR, W_CUT = 1.455915450052607, 2.0, 14.0
X = -8.0 / 9.0
OMEGA_HSE06, FRAC_HSE06 = 0.106, 0.25


class Dual:
    """Value and partial derivatives with respect to (s, w); numpy arrays."""
    __slots__ = ("v", "s", "w")
    __array_ufunc__ = None   # numpy operands defer to the Dual operators

    def __init__(self, v, s=0.0, w=0.0):
        self.v, self.s, self.w = v, s, w

    @staticmethod
    def lift(x):
        return x if isinstance(x, Dual) else Dual(x)

    def __add__(self, o):
        o = Dual.lift(o)
        return Dual(self.v + o.v, self.s + o.s, self.w + o.w)

    __radd__ = __add__

    def __sub__(self, o):
        o = Dual.lift(o)
        return Dual(self.v - o.v, self.s - o.s, self.w - o.w)

    def __rsub__(self, o):
        return Dual.lift(o) - self

    def __neg__(self):
        return Dual(-self.v, -self.s, -self.w)

    def __mul__(self, o):
        o = Dual.lift(o)
        return Dual(self.v * o.v, self.s * o.v + self.v * o.s, self.w * o.v + self.v * o.w)

    __rmul__ = __mul__

    def __truediv__(self, o):
        o = Dual.lift(o)
        q = self.v / o.v
        return Dual(q, (self.s - q * o.s) / o.v, (self.w - q * o.w) / o.v)

    def __rtruediv__(self, o):
        return Dual.lift(o) / self

    def chain(self, f, df):
        return Dual(f, df * self.s, df * self.w)


def d_sqrt(x):
    r = np.sqrt(x.v)
    return x.chain(r, 0.5 / r)


def d_log(x):
    return x.chain(np.log(x.v), 1.0 / x.v)


def d_pow(x, e):
    return x.chain(x.v ** e, e * x.v ** (e - 1.0))


def d_erfcx(x):
    f = erfcx(x.v)
    return x.chain(f, 2.0 * x.v * f - 2.0 / math.sqrt(math.pi))


def d_expe1(x):
    """e^x E1(x), derivative e^x E1(x) - 1/x."""
    f = np.exp(x.v) * exp1(x.v)
    return x.chain(f, f - 1.0 / x.v)


def wpbe_fx(s, w):
    """F_x(s, w) with its partials: returns (F, dF/ds, dF/dw); s, w arrays (w > 0)."""
    s = np.asarray(s, float)
    w = np.asarray(w, float)
    z = np.zeros_like(s + w)
    S = Dual(s + z, 1.0 + z, z)
    W = Dual(w + z, z, 1.0 + z)
    s2 = S * S
    hnum = HA[0] * s2 + HA[1] * s2 * s2
    hden = 1.0 + HA[2] * s2 * s2 + HA[3] * s2 * s2 * S + HA[4] * s2 * s2 * s2
    H = hnum / hden
    F = FC1 * H + FC2
    h = s2 * H
    a = D + h
    # EG from the normalisation int y^2 J dy = -3 pi / 4 (series below EG_SCUT)
    big = s > EG_SCUT
    sb = Dual(np.where(big, S.v, 1.0), np.where(big, S.s, 0.0), np.where(big, S.w, 0.0))
    sb2 = sb * sb
    Hb = (HA[0] * sb2 + HA[1] * sb2 * sb2) / (1.0 + HA[2] * sb2 * sb2 + HA[3] * sb2 * sb2 * sb + HA[4] * sb2 * sb2 * sb2)
    Fb = FC1 * Hb + FC2
    ab = D + sb2 * Hb
    a72 = d_pow(ab, 3.5)
    spi = math.sqrt(math.pi)
    ga = spi * (15.0 * E + 6.0 * C * (1.0 + Fb * sb2) * ab + 4.0 * B * ab * ab + 8.0 * A * ab * ab * ab) / (16.0 * a72) \
        - 0.75 * math.pi * math.sqrt(A) * d_erfcx(1.5 * sb * d_sqrt(Hb / A))
    gb = (15.0 / 16.0) * spi * sb2 / a72
    eg_big = -(0.75 * math.pi + ga) / gb
    eg_small = EGA[0] + EGA[1] * s2 + EGA[2] * s2 * s2
    EG = Dual(np.where(big, eg_big.v, eg_small.v), np.where(big, eg_big.s, eg_small.s),
              np.where(big, eg_big.w, eg_small.w))
    # regular part: B K0 + C (1 + s^2 F) K1 + (E + s^2 EG) K2, exact erfc
    r = d_sqrt(a + W * W)
    t = a / (r * r)
    wr = W / r
    k0 = (1.0 - wr) / (2.0 * a)
    k1 = (1.0 - wr * (1.0 + 0.5 * t)) / (2.0 * a * a)
    k2 = (1.0 - wr * (1.0 + 0.5 * t + 0.375 * t * t)) * 2.0 / (2.0 * a * a * a)
    reg = B * k0 + C * (1.0 + s2 * F) * k1 + (E + s2 * EG) * k2
    # singular part with the erfc fit
    far = w > W_CUT
    eb1 = np.where(far, EB1_FAR, EB1)
    beta = eb1 * W * W
    p = a + beta
    q = h + beta
    lam = 4.0 * A / 9.0
    x = q / lam
    ex1 = d_expe1(x)
    sing = 0.5 * (d_log(q) - d_log(p)) + 0.5 * ex1
    L = [0.5 * math.pi / math.sqrt(lam) * d_erfcx(d_sqrt(x)), ex1 / (2.0 * lam)]

    def M(j, y):
        return math.gamma(0.5 * (j + 1)) / (2.0 * d_pow(y, 0.5 * (j + 1)))

    for j in range(2, 8):
        L.append((M(j - 2, q) - L[j - 2]) / lam)
    wk = Dual(1.0 + z)
    poly = Dual(z)
    for k in range(1, 9):
        wk = wk * W
        poly = poly + EA[k - 1] * wk * (M(k - 1, p) - L[k - 1])
    poly = Dual(np.where(far, 0.0, poly.v), np.where(far, 0.0, poly.s), np.where(far, 0.0, poly.w))
    fx = X * (A * (sing + poly) + reg)
    return fx.v, fx.s, fx.w


def pbexsr(rho, grho2, omega=OMEGA_HSE06):
    """Short-range PBE exchange energy density sx (per volume), v1 = d sx /
    d rho and v2 = (1 / |grad rho|) d sx / d |grad rho| (pbexsr,
    src/utility.cpp:3340-3374, including its clamp of s above 8.3)."""
    rho = np.asarray(rho, float)
    grho2 = np.asarray(grho2, float)
    us, ax = 0.161620459673995492, -0.738558766382022406
    rs = rho ** (1.0 / 3.0)
    vx = (4.0 / 3.0) * ax * rs
    rr = 1.0 / (rho * rs)
    ex = ax / rr
    s2 = grho2 * rr * rr * us * us
    s = np.sqrt(s2)
    s = np.where(s > 8.3, 8.572844 - 18.796223 / s2, s)
    kf = (3.0 * math.pi ** 2 * rho) ** (1.0 / 3.0)
    w = omega / kf
    fx, dfs, dfw = wpbe_fx(s, w)
    d1x = dfw * (-w / (3.0 * rho))
    sx = ex * fx
    v1 = vx * fx + (-4.0 / 3.0 * s / rho * dfs + d1x) * ex
    v2 = ex / np.sqrt(grho2) * (us * rr) * dfs
    return sx, v1, v2


def hse06_point(rho, sigma):
    """Semilocal HSE06 at points: PBE (oracle.scf.xc_pbe_point) minus 0.25 times
    the short-range PBE exchange where rho > 1e-6 and sigma > 1e-10
    (hamiltonian.cpp:1614-1627).  Returns (eps per particle, v1, v2) in the
    convention of xc_pbe_point (v2 = 2 d e / d sigma)."""
    from oracle.scf import xc_pbe_point
    rho = np.asarray(rho, float)
    sigma = np.asarray(sigma, float)
    eps, v1, v2 = xc_pbe_point(rho, sigma)
    eps, v1, v2 = np.array(eps, float), np.array(v1, float), np.array(v2, float)
    m = (np.abs(rho) > 1e-6) & (np.abs(sigma) > 1e-10)
    if np.any(m):
        sx, a1, a2 = pbexsr(rho[m], sigma[m])
        eps[m] -= FRAC_HSE06 * sx / rho[m]
        v1[m] -= FRAC_HSE06 * a1
        v2[m] -= FRAC_HSE06 * a2
    return eps, v1, v2


def xc_hse06(dm, rho, ecut):
    """(eps per particle, V_xc) of the semilocal HSE06 functional on the fine
    grid: the PBE assembly of oracle.scf.xc_pbe with hse06_point."""
    from oracle.scf import xc_pbe
    return xc_pbe(dm, rho, ecut, point=hse06_point)
