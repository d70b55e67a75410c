"""HGH pseudopotential tables and the reference's cubic spline, restated in NumPy.

Test infrastructure (see ``oracle/__init__.py``).

* ``hgh_table``   follows ``utilities/HGH.m`` (parameters for Si :262-276 and
  Al :234-248, derived h-coefficients :284-300, functional forms :303-383,
  channel diagonalisation :387-432, radial sampling and table columns
  :467-1128).  Projector derivatives use the analytic derivative instead of
  MATLAB ``csape``/``fnder`` (a ~1e-10 deviation that only touches the force
  columns).
* ``spline`` / ``seval`` follow ``src/utility.cpp:54-232`` (Forsythe-Malcolm-
  Moler cubic spline with divided-difference end conditions).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Published HGH parameters (Hartwigsen-Goedecker-Hutter 1998) as listed in
# utilities/HGH.m.  Keys: Znuc -> dict.
_HGH_PARAMS = {
    14: dict(name="Si", Zion=4.0, mass=28.0855, rloc=0.44, C=(-7.336103, 0.0, 0.0, 0.0),
             r0=0.422738, h0=(5.906928, 3.258196, 0.0), r1=0.484278, h1=(2.727013, 0.0, 0.0),
             rhocut=3.5, wavcut=3.5),
    13: dict(name="Al", Zion=3.0, mass=26.9815386, rloc=0.45, C=(-8.491351, 0.0, 0.0, 0.0),
             r0=0.460104, h0=(5.088340, 2.679700, 0.0), r1=0.536744, h1=(2.193438, 0.0, 0.0),
             rhocut=3.5, wavcut=3.5),
}

# PeriodTable type codes (src/SCF/periodtable.cpp:171-183)
TYPE_L0, TYPE_L1, TYPE_L2, TYPE_L3 = 0, 1, 2, 3


def spline(x: np.ndarray, y: np.ndarray):
    """Cubic spline coefficients b, c, d -- src/utility.cpp:54-154."""
    n = x.size
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    b = np.zeros(n)
    c = np.zeros(n)
    d = np.zeros(n)
    nm1 = n - 1
    if n < 3:
        b[0] = (y[1] - y[0]) / (x[1] - x[0])
        b[1] = b[0]
        return b, c, d
    # tridiagonal set-up (utility.cpp:105-112), vectorised where independent
    d[:nm1] = x[1:] - x[:-1]
    b[1:nm1] = 2.0 * (d[0:nm1 - 1] + d[1:nm1])
    dd = (y[1:] - y[:-1]) / d[:nm1]          # c[i+1] before differencing
    c[1:nm1] = dd[1:] - dd[:-1]
    c[nm1] = dd[-1]
    # end conditions (utility.cpp:118-128)
    b[0] = -d[0]
    b[n - 1] = -d[n - 2]
    c[0] = 0.0
    c[n - 1] = 0.0
    if n > 3:
        c0 = c[2] / (x[3] - x[1]) - c[1] / (x[2] - x[0])
        cn = c[n - 2] / (x[n - 1] - x[n - 3]) - c[n - 3] / (x[n - 2] - x[n - 4])
        c[0] = c0 * d[0] * d[0] / (x[3] - x[0])
        c[n - 1] = -cn * d[n - 2] * d[n - 2] / (x[n - 1] - x[n - 4])
    # forward elimination / back substitution (utility.cpp:132-143): sequential
    bl = b.tolist()
    cl = c.tolist()
    dl = d.tolist()
    for i in range(1, n):
        t = dl[i - 1] / bl[i - 1]
        bl[i] = bl[i] - t * dl[i - 1]
        cl[i] = cl[i] - t * cl[i - 1]
    cl[n - 1] = cl[n - 1] / bl[n - 1]
    for i in range(n - 2, -1, -1):
        cl[i] = (cl[i] - dl[i] * cl[i + 1]) / bl[i]
    c = np.array(cl)
    b = np.array(bl)
    # polynomial coefficients (utility.cpp:146-153)
    b_last = (y[n - 1] - y[nm1 - 1]) / d[nm1 - 1] + d[nm1 - 1] * (c[nm1 - 1] + 2.0 * c[n - 1])
    bo = np.empty(n)
    bo[:nm1] = (y[1:] - y[:-1]) / d[:nm1] - d[:nm1] * (c[1:] + 2.0 * c[:-1])
    bo[n - 1] = b_last
    do = np.empty(n)
    do[:nm1] = (c[1:] - c[:-1]) / d[:nm1]
    do[n - 1] = do[n - 2]
    co = 3.0 * c
    return bo, co, do


def seval(u, x, y, b, c, d):
    """Evaluate the spline -- src/utility.cpp:157-225 (binary search interval,
    constant extrapolation of the end polynomials)."""
    u = np.asarray(u, dtype=np.float64)
    n = x.size
    i = np.searchsorted(x, u, side="right") - 1
    i = np.clip(i, 0, n - 1)
    dx = u - x[i]
    return y[i] + dx * (b[i] + dx * (c[i] + dx * d[i]))


def _proj_radial(l: int, i: int, rl: float):
    """HGH projector radial form p_{l,i}(r) -- utilities/HGH.m:336-383."""
    ex = l + (4 * i - 1) / 2.0
    pw = l + 2 * (i - 1)
    norm = math.sqrt(2.0) / (rl ** ex * math.sqrt(math.gamma(ex)))

    def f(r):
        return norm * r ** pw * np.exp(-r * r / (2.0 * rl * rl))

    def df(r):
        e = np.exp(-r * r / (2.0 * rl * rl))
        if pw == 0:
            return norm * e * (-r / (rl * rl))
        return norm * e * (pw * r ** (pw - 1) - r ** (pw + 1) / (rl * rl))

    return f, df


@dataclass
class HGHSpecies:
    """One species table: the PTEntry of ``include/periodtable.hpp`` restricted
    to the HGH real-space path (samples, weights, types, cutoffs, params)."""
    znuc: int
    zion: float
    mass: float
    eself: float
    rhocut: float
    wavcut: float
    r: np.ndarray                       # radial grid (column RADIAL_GRID)
    rho: np.ndarray                     # column PSEUDO_CHARGE (= -rho0)
    drho: np.ndarray                    # column DRV_PSEUDO_CHARGE
    proj: list = field(default_factory=list)     # [(type l, weight h, val, der)]
    splines: dict = field(default_factory=dict)  # name -> (x, y, b, c, d)

    def spl(self, key):
        return self.splines[key]


def hgh_table(znuc: int, with_splines: bool = True) -> HGHSpecies:
    """Build the HGH table for one element -- utilities/HGH.m:284-1128."""
    p = _HGH_PARAMS[znuc]
    Zion, rloc = p["Zion"], p["rloc"]
    C1, C2, C3, C4 = p["C"]
    stp = 0.0005
    # r = [-10+stp/2 : stp : 10]  (HGH.m:893-894): 40000 symmetric samples
    nr = int(math.floor((10.0 - (-10.0 + stp / 2)) / stp + 1e-9)) + 1
    r = -10.0 + stp / 2 + stp * np.arange(nr)

    def vloc(rr):
        with np.errstate(divide="ignore", invalid="ignore"):
            v = -Zion / rr * np.vectorize(math.erf)(rr / (math.sqrt(2.0) * rloc))
        return v + np.exp(-0.5 * (rr / rloc) ** 2) * (
            C1 + C2 * (rr / rloc) ** 2 + C3 * (rr / rloc) ** 4 + C4 * (rr / rloc) ** 6)

    def rho0(rr):
        e = np.exp(-0.5 * (rr / rloc) ** 2)
        return 1.0 / (4 * math.pi) * (
            -math.sqrt(2 / math.pi) * Zion / rloc ** 3 * e
            + e * ((-6 * C2 + 3 * C1) / rloc ** 2 + (-20 * C3 + 7 * C2 - C1) * rr ** 2 / rloc ** 4
                   + (-42 * C4 + 11 * C3 - C2) * rr ** 4 / rloc ** 6
                   + (15 * C4 - C3) * rr ** 6 / rloc ** 8 - C4 * rr ** 8 / rloc ** 10))

    def drho0(rr):
        e = np.exp(-0.5 * (rr / rloc) ** 2)
        return 1.0 / (4 * math.pi) * (
            math.sqrt(2 / math.pi) * Zion * rr / rloc ** 5 * e
            + e * ((-40 * C3 + 20 * C2 - 5 * C1) * rr / rloc ** 4
                   + (-168 * C4 + 64 * C3 - 11 * C2 + C1) * rr ** 3 / rloc ** 6
                   + (132 * C4 - 17 * C3 + C2) * rr ** 5 / rloc ** 8
                   + (-23 * C4 + C3) * rr ** 7 / rloc ** 10 + C4 * rr ** 9 / rloc ** 12))

    rho = rho0(r)
    drho = drho0(r)
    gd = r > 0
    Vl = vloc(r[gd])
    eself = 0.5 * float(np.sum(4 * math.pi * r[gd] ** 2 * Vl * rho[gd] * stp))   # HGH.m:995

    sp = HGHSpecies(znuc=znuc, zion=Zion, mass=p["mass"], eself=eself,
                    rhocut=p["rhocut"], wavcut=p["wavcut"], r=r, rho=-rho, drho=-drho)

    # channel diagonalisation (HGH.m:387-432): h-matrices with derived
    # off-diagonals (HGH.m:284-293); eigenvalues sorted descending; only
    # |h| > 1e-10 kept (HGH.m:1032-1093)
    for l, rl, hd in ((0, p["r0"], p["h0"]), (1, p["r1"], p["h1"])):
        h11, h22, h33 = hd
        if l == 0:
            h12 = -0.5 * math.sqrt(3.0 / 5.0) * h22
            h13 = 0.5 * math.sqrt(5.0 / 21.0) * h33
            h23 = -0.5 * math.sqrt(100.0 / 63.0) * h33
        else:
            h12 = -0.5 * math.sqrt(5.0 / 7.0) * h22
            h13 = 1.0 / 6.0 * math.sqrt(35.0 / 11.0) * h33
            h23 = -1.0 / 6.0 * 14.0 / math.sqrt(11.0) * h33
        H = np.array([[h11, h12, h13], [h12, h22, h23], [h13, h23, h33]])
        D, V = np.linalg.eigh(H)
        order = np.argsort(-D, kind="stable")
        D, V = D[order], V[:, order]
        # eigenvector sign is arbitrary (MATLAB eig); fix it: largest |component| > 0
        for a in range(3):
            if V[np.argmax(np.abs(V[:, a])), a] < 0:
                V[:, a] = -V[:, a]
        fns = [_proj_radial(l, i, rl) for i in (1, 2, 3)]
        for a in range(3):
            if abs(D[a]) <= 1e-10:
                continue
            val = sum(V[i, a] * fns[i][0](r) for i in range(3))
            der = sum(V[i, a] * fns[i][1](r) for i in range(3))
            sp.proj.append((l, float(D[a]), val, der))

    if with_splines:
        sp.splines["rho"] = (r,) + (sp.rho,) + spline(r, sp.rho)
        sp.splines["drho"] = (r,) + (sp.drho,) + spline(r, sp.drho)
        for k, (l, h, val, der) in enumerate(sp.proj):
            sp.splines[("val", k)] = (r, val) + spline(r, val)
            sp.splines[("der", k)] = (r, der) + spline(r, der)
    return sp


def spl_eval(sp: HGHSpecies, key, u):
    x, y, b, c, d = sp.splines[key]
    return seval(u, x, y, b, c, d)
