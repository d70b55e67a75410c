"""Regenerate the golden fixtures in this folder from reference functions.

The vectors come from the reference's own ``IP_c2f``, ``IP_f2c``, ``spline``
and ``seval`` (src/utility.cpp) -> ``ref_utility.npz``, and its internal PBE
pieces ``VExchange_sla``, ``VCorrelation_pw``, ``VGCExchange_pbx``,
``VGCCorrelation_pbc`` (src/utility.cpp:3913-4244) -> ``ref_xc_pbe.npz``, and
the HSE06 short-range exchange ``pbexsr`` / ``wpbe_analy_erfc_approx_grad``
(src/utility.cpp:3340-3846) -> ``ref_xc_hse.npz``, all compiled from the
reference source tree by ``oracle/build_ref.py``.  Inputs are seeded.  Run
from the repository root:
``python tests/golden/make_golden.py [utility|pbe|hse|hpsi|smearing]`` (all by default).

``smearing`` -> ``ref_smearing.npz``: the occupation and entropy functions
``wgauss`` / ``getEntropy`` (src/utility.cpp:4404-4444) for the Fermi-Dirac
and Gaussian schemes at seeded arguments.

``hpsi`` -> ``ref_hpsi.npz``: the reference's own H*psi composition,
Spinor::AddMultSpinorFineR2C and Spinor::AddTeterPrecond (src/SCF/spinor.cpp:
310-346, 377-525) with FFTWExecute (src/SCF/fourier.cpp:695-764) and
IP_c2f / IP_f2c, compiled by ``oracle/build_ref.py`` (``libpwref_hpsi.so``), on
seeded Si8 cells: the projector sets, kinetic and Teter tables come from the
oracle's restatement of PeriodTable::CalculateNonlocalPP / CalculateEkin
(oracle/pw.py), the potential and the bands from the seeds stored with them.
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


OUT_HPSI = Path(__file__).resolve().parent / "ref_hpsi.npz"
HPSI_CASES = {"c12": ((12, 12, 12), 3), "c16": ((16, 16, 16), 2)}


def hpsi():
    from oracle import pw
    lib = C.CDLL(str(build_ref.build_hpsi()))
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    lib.ref_add_mult_spinor.argtypes = [ip, ip, dp, dp, dp, C.c_int, ip, ip, ip, dp, dp, C.c_int, dp, dp]
    lib.ref_add_teter.argtypes = [ip, ip, dp, dp, C.c_int, dp, dp]
    data = {}
    for tag, (nc, nb) in HPSI_CASES.items():
        seed_cell, seed_v, seed_psi = 20261203 + 1, 31, 32
        L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, seed_cell)
        nf = tuple(2 * n for n in nc)
        T, _ = pw.build_tables(L, z, pos, nc, nf, seed_v=seed_v)
        psi = pw.random_orthonormal_psi(T.dm.ntot, nb, seed_psi)
        npts = np.array([len(a[0].idx) for a in T.pseudo], np.int32)
        nproj = np.array([len(a) for a in T.pseudo], np.int32)
        idx = np.concatenate([a[0].idx for a in T.pseudo]).astype(np.int32)
        beta = np.concatenate([pp.val[:, 0] for a in T.pseudo for pp in a]).astype(np.float64)
        wgt = np.array([pp.wgt for a in T.pseudo for pp in a], np.float64)
        h = np.zeros_like(psi)
        w = np.zeros_like(psi)
        ncv, nfv, Lv = np.array(nc, np.int32), np.array(nf, np.int32), np.array(L, np.float64)
        assert lib.ref_add_mult_spinor(ncv, nfv, Lv, np.ascontiguousarray(T.ekin.ravel()), T.vtot, len(T.pseudo),
                                       npts, nproj, idx, beta, wgt, nb, np.ascontiguousarray(psi), h) == 0
        assert lib.ref_add_teter(ncv, nfv, Lv, np.ascontiguousarray(T.teter.ravel()), nb, np.ascontiguousarray(psi),
                                 w) == 0
        data[f"{tag}_grid"] = np.array(nc)
        data[f"{tag}_seeds"] = np.array([seed_cell, seed_v, seed_psi])
        data[f"{tag}_nband"] = np.array(nb)
        data[f"{tag}_hpsi"] = h
        data[f"{tag}_teter"] = w
    np.savez_compressed(OUT_HPSI, **data)
    print(OUT_HPSI, OUT_HPSI.stat().st_size)


OUT_SMEAR = Path(__file__).resolve().parent / "ref_smearing.npz"


def smearing():
    """wgauss and getEntropy (src/utility.cpp:4404-4444) for both smearing
    schemes ("FD", "GB") at seeded (e, E_F, beta) triples spanning the
    |x| <= 36 cut of the Fermi-Dirac entropy and the 200 cap of the Gaussian
    one -> ref_smearing.npz."""
    lib = C.CDLL(str(build_ref.build()))
    lib.ref_wgauss.restype = C.c_double
    lib.ref_entropy.restype = C.c_double
    rng = np.random.Generator(np.random.Philox(20261203 + 7))
    n = 400
    ev = rng.uniform(-0.5, 0.5, n)
    ef = rng.uniform(-0.2, 0.2, n)
    tbeta = 10.0 ** rng.uniform(1.0, 4.0, n)
    out = np.zeros((n, 4))
    for i in range(n):
        a = (C.c_double(ev[i]), C.c_double(ef[i]), C.c_double(tbeta[i]))
        out[i] = [lib.ref_wgauss(*a, 0), lib.ref_wgauss(*a, 1), lib.ref_entropy(*a, 0), lib.ref_entropy(*a, 1)]
    np.savez_compressed(OUT_SMEAR, ev=ev, ef=ef, tbeta=tbeta, out=out)
    print(OUT_SMEAR, OUT_SMEAR.stat().st_size)


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "all"
    if which in ("all", "utility"):
        main()
    if which in ("all", "pbe"):
        pbe()
    if which in ("all", "hse"):
        hse()
    if which in ("all", "hpsi"):
        hpsi()
    if which in ("all", "smearing"):
        smearing()
