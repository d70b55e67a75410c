"""Regenerate the golden fixtures in this folder from reference functions.

The vectors come from the reference's own ``IP_c2f``, ``IP_f2c``, ``spline``
and ``seval`` (src/utility.cpp) -> ``ref_utility.npz``, and its internal PBE
pieces ``VExchange_sla``, ``VCorrelation_pw``, ``VGCExchange_pbx``,
``VGCCorrelation_pbc`` (src/utility.cpp:3913-4244) -> ``ref_xc_pbe.npz``, and
the HSE06 short-range exchange ``pbexsr`` / ``wpbe_analy_erfc_approx_grad``
(src/utility.cpp:3340-3846) -> ``ref_xc_hse.npz``, all compiled from the
reference source tree by ``oracle/build_ref.py``.  Inputs are seeded.  Run
from the repository root:
``python tests/golden/make_golden.py [utility|pbe|hse]`` (all by default).
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import build_ref  # noqa: E402

OUT = Path(__file__).resolve().parent / "ref_utility.npz"
OUT_PBE = Path(__file__).resolve().parent / "ref_xc_pbe.npz"
OUT_HSE = Path(__file__).resolve().parent / "ref_xc_hse.npz"


def main():
    lib = C.CDLL(str(build_ref.build()))
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    rng = np.random.Generator(np.random.Philox(20261203))
    data = {}
    for tag, Nc, Nf in (("a", (4, 4, 4), (8, 8, 8)), ("b", (6, 4, 8), (12, 8, 16)), ("c", (8, 6, 4), (16, 12, 8))):
        nhc = (Nc[0] // 2 + 1) * Nc[1] * Nc[2]
        nhf = (Nf[0] // 2 + 1) * Nf[1] * Nf[2]
        X = rng.standard_normal(nhc) + 1j * rng.standard_normal(nhc)
        Y = np.zeros(nhf, complex)
        nc = (C.c_int * 3)(*Nc)
        nf = (C.c_int * 3)(*Nf)
        lib.ref_ip_c2f(nc, nf, X.ctypes.data_as(dp), Y.ctypes.data_as(dp))
        Yin = rng.standard_normal(nhf) + 1j * rng.standard_normal(nhf)
        Z = np.zeros(nhc, complex)
        lib.ref_ip_f2c(nc, nf, Z.ctypes.data_as(dp), Yin.ctypes.data_as(dp))
        data[f"c2f_{tag}_Nc"] = np.array(Nc)
        data[f"c2f_{tag}_Nf"] = np.array(Nf)
        data[f"c2f_{tag}_in"] = X
        data[f"c2f_{tag}_out"] = Y
        data[f"f2c_{tag}_in"] = Yin
        data[f"f2c_{tag}_out"] = Z
    n = 200
    x = np.sort(rng.uniform(-3, 3, n))
    y = np.exp(-x * x) * np.cos(3 * x)
    b, c, d = np.zeros(n), np.zeros(n), np.zeros(n)
    lib.ref_spline(n, x.ctypes.data_as(dp), y.ctypes.data_as(dp), b.ctypes.data_as(dp), c.ctypes.data_as(dp),
                   d.ctypes.data_as(dp))
    u = rng.uniform(-3.5, 3.5, 100)
    v = np.zeros(100)
    lib.ref_seval(v.ctypes.data_as(dp), 100, u.ctypes.data_as(dp), n, x.ctypes.data_as(dp), y.ctypes.data_as(dp),
                  b.ctypes.data_as(dp), c.ctypes.data_as(dp), d.ctypes.data_as(dp))
    data.update(spl_x=x, spl_y=y, spl_b=b, spl_c=c, spl_d=d, sev_u=u, sev_v=v)
    np.savez_compressed(OUT, **data)
    print(OUT, OUT.stat().st_size)


def pbe():
    """(rs, rho, grho2) samples over densities 1e-6..10 and reduced gradients
    s = |grad rho| / (2 k_F rho) in 0..6, and the ten outputs of the four
    reference functions per sample."""
    lib = C.CDLL(str(build_ref.build()))
    dp = C.POINTER(C.c_double)
    rng = np.random.Generator(np.random.Philox(20261203 + 77))
    n = 400
    rho = 10.0 ** rng.uniform(-6, 1, n)
    s = np.concatenate([rng.uniform(0, 6, n - 20), np.zeros(10), rng.uniform(0, 1e-3, 10)])
    kf = (3 * np.pi ** 2 * rho) ** (1 / 3)
    grho2 = (s * 2 * kf * rho) ** 2 + 1e-9
    rs = (3 / (4 * np.pi * rho)) ** (1 / 3)
    out = np.zeros((n, 10))
    for i in range(n):
        lib.ref_pbe_parts(C.c_double(rs[i]), C.c_double(rho[i]), C.c_double(grho2[i]), out[i].ctypes.data_as(dp))
    np.savez_compressed(OUT_PBE, rs=rs, rho=rho, grho2=grho2, out=out)
    print(OUT_PBE, OUT_PBE.stat().st_size)


def hse():
    """pbexsr at (rho, grho2) samples over densities 1e-6..10 and reduced
    gradients s in 0..10 (s > 8.3 exercises the clamp, s < 0.08 the series
    branch of the normalisation), omega = 0.106: (sx, v1x, v2x); and the
    screened enhancement factor at (rho, s): (F_x, d1rfx, d1sfx)."""
    lib = C.CDLL(str(build_ref.build()))
    dp = C.POINTER(C.c_double)
    rng = np.random.Generator(np.random.Philox(20261203 + 78))
    n = 400
    rho = 10.0 ** rng.uniform(-5.9, 1, n)
    s = np.concatenate([rng.uniform(0, 10, n - 40), rng.uniform(0, 0.08, 20), rng.uniform(8.2, 9, 20)])
    kf = (3 * np.pi ** 2 * rho) ** (1 / 3)
    grho2 = (s * 2 * kf * rho) ** 2 + 1e-9
    out = np.zeros((n, 3))
    fx = np.zeros((n, 3))
    for i in range(n):
        lib.ref_pbexsr(C.c_double(rho[i]), C.c_double(grho2[i]), C.c_double(0.106), out[i].ctypes.data_as(dp))
        lib.ref_wpbe(C.c_double(rho[i]), C.c_double(min(s[i], 8.5)), C.c_double(0.106), fx[i].ctypes.data_as(dp))
    np.savez_compressed(OUT_HSE, rho=rho, grho2=grho2, out=out, s=np.minimum(s, 8.5), fx=fx)
    print(OUT_HSE, OUT_HSE.stat().st_size)


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "all"
    if which in ("all", "utility"):
        main()
    if which in ("all", "pbe"):
        pbe()
    if which in ("all", "hse"):
        hse()
