"""CPU tests of the FP64 oracle: pinned against reference functions compiled
from the reference tree (golden fixtures) and against known-answer tests."""
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import hgh, pw

GOLD = Path(__file__).resolve().parent / "golden" / "ref_utility.npz"


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_ip_c2f_f2c_match_reference_functions(gold, tag):
    Nc = tuple(int(x) for x in gold[f"c2f_{tag}_Nc"])
    Nf = tuple(int(x) for x in gold[f"c2f_{tag}_Nf"])
    X = gold[f"c2f_{tag}_in"]
    ip = pw.IPMaps(Nc, Nf)
    assert np.array_equal(pw.ip_c2f_loop(Nc, Nf, X), gold[f"c2f_{tag}_out"])
    assert np.array_equal(ip.c2f(X), gold[f"c2f_{tag}_out"])
    Y = gold[f"f2c_{tag}_in"]
    Z = pw.ip_f2c_loop(Nc, Nf, np.zeros(ip.nhc, complex), Y)
    assert np.allclose(Z, gold[f"f2c_{tag}_out"], rtol=0, atol=1e-15)
    assert np.allclose(ip.f2c(Y), gold[f"f2c_{tag}_out"], rtol=0, atol=1e-15)


def test_spline_seval_match_reference_functions(gold):
    x, y = gold["spl_x"], gold["spl_y"]
    b, c, d = hgh.spline(x, y)
    assert np.allclose(b, gold["spl_b"], rtol=1e-12, atol=1e-13)
    assert np.allclose(c, gold["spl_c"], rtol=1e-12, atol=1e-13)
    assert np.allclose(d, gold["spl_d"], rtol=1e-12, atol=1e-12)
    v = hgh.seval(gold["sev_u"], x, y, gold["spl_b"], gold["spl_c"], gold["spl_d"])
    assert np.allclose(v, gold["sev_v"], rtol=1e-14, atol=1e-15)


def test_reference_functions_rebuild_here_when_tree_present():
    """When the reference tree is present, rebuild the reference functions and
    re-check one IP case live (fixtures above cover machines without it)."""
    from oracle import build_ref
    if not (build_ref.DEFAULT_REF / "src" / "utility.cpp").exists():
        pytest.skip("reference tree not present")
    import ctypes as C
    lib = C.CDLL(str(build_ref.build()))
    dp = C.POINTER(C.c_double)
    Nc, Nf = (6, 6, 6), (12, 12, 12)
    rng = np.random.default_rng(3)
    ip = pw.IPMaps(Nc, Nf)
    X = rng.standard_normal(ip.nhc) + 1j * rng.standard_normal(ip.nhc)
    Y = np.zeros(ip.nhf, complex)
    lib.ref_ip_c2f((C.c_int * 3)(*Nc), (C.c_int * 3)(*Nf), X.ctypes.data_as(dp), Y.ctypes.data_as(dp))
    assert np.array_equal(ip.c2f(X), Y)


def test_hgh_table_normalisation():
    """utilities/HGH.m:1136-1158 prints int(-rho) = Zion and the projector
    normalisation; the l=1 projector is normalised to 1, the two s-channel
    combinations sum to 2."""
    sp = hgh.hgh_table(14, with_splines=False)
    r, stp = sp.r, 5e-4
    pk = (r > 0) & (r < sp.rhocut)
    assert abs(np.sum(4 * np.pi * r[pk] ** 2 * sp.rho[pk] * stp) - 4.0) < 1e-8
    pk = (r > 0) & (r < sp.wavcut)
    norms = [np.sum(r[pk] ** 2 * v[pk] ** 2 * stp) for _, _, v, _ in sp.proj]
    assert [l for l, *_ in sp.proj] == [0, 0, 1]
    assert abs(norms[2] - 1.0) < 1e-6
    assert abs(norms[0] + norms[1] - 2.0) < 1e-6
    # weights: eigenvalues of the 2x2 s-channel h-matrix, sorted descending
    h22 = 3.258196
    H = np.array([[5.906928, -0.5 * math.sqrt(0.6) * h22], [-0.5 * math.sqrt(0.6) * h22, h22]])
    ev = np.sort(np.linalg.eigvalsh(H))[::-1]
    assert np.allclose([sp.proj[0][1], sp.proj[1][1]], ev, rtol=1e-14)
    assert sp.proj[2][1] == 2.727013


def test_teter_closed_form():
    dm = pw.Domain((10.26,) * 3, (8, 8, 8), (16, 16, 16))
    ekin, teter = pw.ekin_teter(dm)
    a = 2 * ekin
    b = 27 + 18 * a + 12 * a ** 2 + 8 * a ** 3
    assert np.allclose(teter, b / (b + 16 * a ** 4), rtol=1e-15)
    assert teter.flat[0] == 1.0
    g = 2 * np.pi / 10.26
    assert abs(ekin[0, 0, 1] - g * g / 2) < 1e-15
    assert abs(ekin[0, 0, 4] - (4 * g) ** 2 / 2) < 1e-14     # Nyquist at +n/2


def test_parseval_conventions():
    """forward x vol/N, backward x 1/vol (src/SCF/fourier.cpp:695-764)."""
    dm = pw.Domain((7.0, 8.0, 9.0), (6, 8, 10), (12, 16, 20))
    rng = np.random.default_rng(1)
    x = rng.standard_normal((10, 8, 6))
    X = pw.r2c(x, dm)
    assert np.allclose(pw.c2r(X, dm), x, atol=1e-13)
    full = np.fft.fftn(x) * dm.vol / dm.ntot
    assert abs(np.sum(np.abs(full) ** 2) / dm.vol - np.sum(x * x) * dm.vol / dm.ntot) < 1e-9


def _free_tables(numGrid, L=(9.0, 9.0, 9.0)):
    dm = pw.Domain(L, numGrid, tuple(2 * n for n in numGrid))
    ekin, teter = pw.ekin_teter(dm)
    return pw.HamTables(dm, ekin, teter, np.zeros(dm.ntotFine), [])


def test_single_plane_wave_kinetic_eigenvalue():
    """V = 0, no projectors: cos(G.r) is an eigenvector with eigenvalue |G|^2/2."""
    T = _free_tables((8, 8, 8))
    n = 8
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    for m in [(1, 0, 0), (2, 1, 0), (1, 2, 3), (3, 3, 1)]:
        ph = 2 * np.pi * (m[0] * x + m[1] * y + m[2] * z) / n
        psi = np.cos(ph).reshape(1, -1)
        out = pw.mult_spinor(T, psi)
        g2 = sum((2 * np.pi / 9.0 * mi) ** 2 for mi in m)
        assert np.allclose(out, 0.5 * g2 * psi, atol=1e-12)


def test_free_electron_spectrum():
    """V = 0: the eigenvalues of the full H matrix on a 4^3 grid are |G|^2/2
    over the grid's frequencies (Nyquist components at +n/2)."""
    T = _free_tables((4, 4, 4), L=(6.0, 6.0, 6.0))
    N = 64
    Hm = pw.mult_spinor(T, np.eye(N))
    assert np.allclose(Hm, Hm.T, atol=1e-13)
    ev = np.sort(np.linalg.eigvalsh(Hm))
    g = pw.gvec_full(T.dm)
    ref = np.sort(0.5 * np.sum(g * g, axis=-1).ravel())
    assert np.allclose(ev, ref, atol=1e-12)


@pytest.fixture(scope="module")
def si8_small():
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)
    T, sp = pw.build_tables(L, z, pos, (12, 12, 12), (24, 24, 24), seed_v=11)
    return T, sp, pos


def test_hamiltonian_hermitian(si8_small):
    T, _, _ = si8_small
    psi = pw.random_orthonormal_psi(T.dm.ntot, 6, 2)
    H = pw.mult_spinor(T, psi)
    M = psi @ H.T
    assert np.abs(M - M.T).max() < 1e-13 * np.abs(M).max()


def test_projector_sets(si8_small):
    T, sp, pos = si8_small
    assert len(T.pseudo) == 8 and all(len(a) == 5 for a in T.pseudo)
    pp = T.pseudo[0][0]
    # every point of the index set lies within Rcut of the atom (minimum image)
    N = np.array(T.dm.numGridFine)
    g = pp.idx
    ijk = np.stack([g % N[0], (g // N[0]) % N[1], g // (N[0] * N[1])], -1)
    d = ijk / N * np.array(T.dm.length) - pos[0]
    d -= np.round(d / np.array(T.dm.length)) * np.array(T.dm.length)
    assert np.all(np.sqrt((d ** 2).sum(-1)) < sp.wavcut + 1e-12)
    assert len(np.unique(g)) == g.size


def test_pseudocharge_integrates_to_zion(si8_small):
    T, sp, pos = si8_small
    dm = T.dm
    idx, dv = pw.pseudo_charge(pw.Atom(14, pos[3]), dm, sp)
    q = dv[:, 0].sum() * dm.vol / dm.ntotFine
    assert abs(q - 4.0) < 2e-2     # grid quadrature of a 0.44-bohr Gaussian on a 0.21-bohr grid


def test_teter_precond_matches_direct(si8_small):
    T, _, _ = si8_small
    rng = np.random.default_rng(4)
    r = rng.standard_normal((3, T.dm.ntot))
    w = pw.add_teter_precond(T, r)
    X = np.fft.rfftn(r.reshape(3, 12, 12, 12), axes=(1, 2, 3)) * T.teter
    assert np.allclose(w, np.fft.irfftn(X, s=(12, 12, 12), axes=(1, 2, 3)).reshape(3, -1), atol=1e-13)


def test_pipeline_model_equals_oracle():
    """The band-pair / Nyquist-slot decomposition used by the CUDA kernels
    reproduces the reference restatement to rounding (cubic and non-cubic)."""
    from tests.pipeline_model import model_hpsi
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 7)
    for nc in [(8, 8, 8), (12, 8, 10)]:
        nf = tuple(2 * n for n in nc)
        T, _ = pw.build_tables(L, z, pos, nc, nf)
        psi = pw.random_orthonormal_psi(int(np.prod(nc)), 5, 3)
        ref = pw.mult_spinor(T, psi)
        got = model_hpsi(T, psi)
        assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-14


def test_nonlocal_force_coarse_identity():
    """The device's nonlocal force form -- coarse projectors q_l = T beta_l and
    derivative projectors T(d beta_l), T the fine->coarse transpose of the
    interpolation, F = 2 numSpin f gamma (vol/N_c)(q.psi)(Tdbeta.psi) -- equals
    the reference's per-band fine-grid "Method 4" (hamiltonian.cpp:2907-3006)."""
    from oracle import forces
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.05, 7)
    nc, nf = (8, 8, 8), (16, 16, 16)
    T, _ = pw.build_tables(L, z, pos, nc, nf)
    dm = T.dm
    N0, N1, N2 = nf
    n0, n1, n2 = nc
    gf = pw.gvec_full(dm, fine=True)

    def t_of(B, d=None):
        Y = np.fft.fftn(B.reshape(N2, N1, N0))
        if d is not None:
            Y = Y * (1j * gf[..., d])
        X = T.ip.f2c(Y[..., :N0 // 2 + 1].reshape(-1)) / dm.ntotFine
        return np.fft.irfftn(X.reshape(n2, n1, n0 // 2 + 1), s=(n2, n1, n0)).ravel() * dm.ntot

    psi = pw.random_orthonormal_psi(dm.ntot, 5, 3)
    occ = np.array([1, 1, .9, .5, .1])
    ref = forces.nonlocal_force(T, psi, occ)
    F = np.zeros_like(ref)
    for a, app in enumerate(T.pseudo):
        for pp in app:
            B = np.zeros(dm.ntotFine)
            B[pp.idx] = pp.val[:, 0]
            q = psi @ t_of(B)
            for d in range(3):
                F[a, d] += np.sum(2 * 2 * occ * pp.wgt * (dm.vol / dm.ntot) * q * (psi @ t_of(B, d)))
    assert np.abs(F - ref).max() <= 1e-12 * np.abs(ref).max()


def test_exx_pair_fft_matches_direct_convolution():
    """Known answer: the pair-FFT Poisson solve of AddMultSpinorEXX
    (spinor.cpp:743-756, R2C x vol/N, kernel, C2R x 1/vol) equals the explicit
    G-space convolution sum on an 8^3 grid."""
    from oracle import exx
    dm = pw.Domain((7.0, 7.5, 8.0), (8, 8, 8), (16, 16, 16))
    k, div = exx.exx_kernel_r2c(dm, ecut=5.0)
    rng = np.random.default_rng(2)
    rho = rng.standard_normal(dm.ntot)
    fft = pw.c2r(pw.r2c(rho.reshape(8, 8, 8), dm) * k, dm).ravel()
    direct = exx.pair_convolution_direct(dm, rho, k)
    assert np.abs(fft - direct).max() <= 1e-12 * np.abs(direct).max()
    assert k[0, 0, 0] == -div and div != 0.0


def test_exx_kernel_divergence_and_screening():
    from oracle import exx
    dm = pw.Domain((10.26, 10.26, 10.26), (16, 16, 16), (32, 32, 32))
    k0, d0 = exx.exx_kernel_r2c(dm, ecut=10.0, div_type=0)
    assert d0 == 0.0 and k0[0, 0, 0] == 0.0
    k1, d1 = exx.exx_kernel_r2c(dm, ecut=10.0, div_type=1)
    assert np.array_equal(k0.ravel()[1:], k1.ravel()[1:])
    # the short-range (screened) kernel 4 pi / G^2 (1 - exp(-G^2 / 4 mu^2)) tends
    # to the bare one as mu -> 0 away from G = 0
    ks, _ = exx.exx_kernel_r2c(dm, ecut=10.0, mu=1e-3, div_type=0)
    assert np.allclose(ks.ravel()[1:], k0.ravel()[1:], rtol=1e-12)


def test_exx_operator_symmetric_and_ace_exact_on_span():
    from oracle import exx
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 3)
    dm = pw.Domain(tuple(L), (8, 8, 8), (16, 16, 16))
    k, _ = exx.exx_kernel_r2c(dm, ecut=5.0)
    psi = pw.random_orthonormal_psi(dm.ntot, 6, 1)
    occ = np.array([1.0, 1.0, 1.0, 0.7, 0.2, 0.0])
    phi = exx.set_phi(dm, psi)
    Vx = exx.add_mult_spinor_exx(dm, psi, phi, k, 0.25, occ)
    M = psi @ Vx.T
    assert np.abs(M - M.T).max() <= 1e-12 * np.abs(M).max()
    assert np.linalg.eigvalsh(-0.5 * (M + M.T)).min() > 0      # V_x negative definite on span
    xi = exx.ace_build(dm, psi, phi, k, 0.25, occ)
    assert np.abs(exx.ace_apply(xi, psi) - Vx).max() <= 1e-11 * np.abs(Vx).max()


def test_kpoint_hamiltonian_hermitian():
    """H(k) of the complex restatement is Hermitian (<x, H y> = <H x, y>) and its
    kinetic / Teter tables are positive."""
    from oracle import kpoints
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 5)
    T, _ = pw.build_tables(L, z, pos, (8, 8, 8), (16, 16, 16), seed_v=2)
    k = np.array([0.11, -0.05, 0.23])
    x = kpoints.random_complex_psi(T.dm.ntot, 3, 1)
    y = kpoints.random_complex_psi(T.dm.ntot, 3, 2)
    hx = kpoints.mult_spinor_k(T, k, x)
    hy = kpoints.mult_spinor_k(T, k, y)
    lhs = np.conj(x) @ hy.T
    rhs = np.conj(hx) @ y.T
    assert np.abs(lhs - rhs).max() <= 1e-12 * np.abs(lhs).max()
    ek, te = kpoints.ekin_teter_k(T.dm, k)
    assert ek.min() > 0 and np.all((te > 0) & (te <= 1))


def test_kpoint_gamma_matches_real_hamiltonian_without_nyquist():
    """At k = 0, on real bands with no Nyquist content (where the R2C and the
    complex placements agree), the complex H equals the Gamma-point real H."""
    from oracle import kpoints
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 5)
    T, _ = pw.build_tables(L, z, pos, (8, 8, 8), (16, 16, 16), seed_v=2)
    dm = T.dm
    psi = pw.random_orthonormal_psi(dm.ntot, 3, 4)
    X = np.fft.fftn(psi.reshape(3, 8, 8, 8), axes=(1, 2, 3))
    X[:, 4, :, :] = 0
    X[:, :, 4, :] = 0
    X[:, :, :, 4] = 0
    psi = np.fft.ifftn(X, axes=(1, 2, 3)).real.reshape(3, -1)
    hr = pw.mult_spinor(T, psi)
    hc = kpoints.mult_spinor_k(T, np.zeros(3), psi.astype(complex))
    # outputs agree away from the Nyquist components, which the two paths treat differently
    Fr = np.fft.fftn(hr.reshape(3, 8, 8, 8), axes=(1, 2, 3))
    Fc = np.fft.fftn(hc.reshape(3, 8, 8, 8), axes=(1, 2, 3))
    for F in (Fr, Fc):
        F[:, 4, :, :] = 0
        F[:, :, 4, :] = 0
        F[:, :, :, 4] = 0
    assert np.abs(Fr - Fc).max() <= 1e-10 * np.abs(Fr).max()


def test_wfn_ecut_filter_is_an_orthogonal_projector():
    """MultSpinor's wavefunction filter (hamiltonian.cpp:3090-3116): P is
    idempotent and symmetric, keeps exactly the coefficients with
    |G|^2/2 <= Ecut, and the filtered MultSpinor is P applied to H psi."""
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)
    T, _ = pw.build_tables(L, z, pos, (16, 16, 16), (32, 32, 32), seed_v=4)
    rng = np.random.default_rng(2)
    x, y = rng.standard_normal((2, 3, T.dm.ntot))
    ecut = 5.0
    px = pw.wfn_ecut_filter(T, x, ecut)
    assert np.abs(pw.wfn_ecut_filter(T, px, ecut) - px).max() < 1e-13
    assert abs(np.sum(px * y) - np.sum(x * pw.wfn_ecut_filter(T, y, ecut))) < 1e-10
    X = pw.r2c(px.reshape(3, 16, 16, 16), T.dm)
    assert np.abs(X[:, T.ekin > ecut]).max() < 1e-12
    assert np.abs(X[:, T.ekin <= ecut] - pw.r2c(x.reshape(3, 16, 16, 16), T.dm)[:, T.ekin <= ecut]).max() < 1e-12
    h = pw.mult_spinor(T, x, wfn_ecut=ecut)
    assert np.abs(h - pw.wfn_ecut_filter(T, pw.mult_spinor(T, x), ecut)).max() < 1e-12


def _ref_hpsi_case(tag):
    g = np.load(GOLD.parent / "ref_hpsi.npz")
    nc = tuple(int(x) for x in g[f"{tag}_grid"])
    seed_cell, seed_v, seed_psi = (int(x) for x in g[f"{tag}_seeds"])
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, seed_cell)
    T, _ = pw.build_tables(L, z, pos, nc, tuple(2 * n for n in nc), seed_v=seed_v)
    psi = pw.random_orthonormal_psi(T.dm.ntot, int(g[f"{tag}_nband"]), seed_psi)
    return g, T, psi


@pytest.mark.parametrize("tag", ["c12", "c16"])
def test_oracle_hpsi_matches_reference_composition(tag):
    """The restated H*psi and Teter (oracle/pw.py) against the outputs of the
    reference's own Spinor::AddMultSpinorFineR2C / AddTeterPrecond compiled
    from its source (tests/golden/ref_hpsi.npz, make_golden.py hpsi): 1e-13."""
    g, T, psi = _ref_hpsi_case(tag)
    h = pw.mult_spinor(T, psi)
    ref = g[f"{tag}_hpsi"]
    assert np.abs(h - ref).max() / np.abs(ref).max() < 1e-13
    w = pw.add_teter_precond(T, psi)
    wr = g[f"{tag}_teter"]
    assert np.abs(w - wr).max() / np.abs(wr).max() < 1e-13


def test_oracle_hpsi_against_compiled_reference_other_grids():
    """Where the reference tree is present (the build container), the compiled
    composition on a non-cubic grid with uneven dimensions (24 x 16 x 20) and
    an fcc Al cell, against the restatement: 1e-13."""
    import ctypes as C

    from oracle import build_ref
    lib_path = build_ref.LIB_HPSI
    if not lib_path.exists():
        pytest.skip("reference composition not built here (oracle/_ref)")
    lib = C.CDLL(str(lib_path))
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    lib.ref_add_mult_spinor.argtypes = [ip, ip, dp, dp, dp, C.c_int, ip, ip, ip, dp, dp, C.c_int, dp, dp]
    for kind, a, nc in (("Si", 10.26, (24, 16, 20)), ("Al", 7.65, (12, 12, 12))):
        L, z, pos = pw.make_crystal(kind, (1, 1, 1), a, 0.02, 9)
        nf = tuple(2 * n for n in nc)
        T, _ = pw.build_tables(L, z, pos, nc, nf, seed_v=4)
        psi = pw.random_orthonormal_psi(T.dm.ntot, 2, 5)
        npts = np.array([len(at[0].idx) for at in T.pseudo], np.int32)
        nproj = np.array([len(at) for at in T.pseudo], np.int32)
        idx = np.concatenate([at[0].idx for at in T.pseudo]).astype(np.int32)
        beta = np.concatenate([pp.val[:, 0] for at in T.pseudo for pp in at]).astype(np.float64)
        wgt = np.array([pp.wgt for at in T.pseudo for pp in at], np.float64)
        h = np.zeros_like(psi)
        assert lib.ref_add_mult_spinor(np.array(nc, np.int32), np.array(nf, np.int32), np.array(L, np.float64),
                                       np.ascontiguousarray(T.ekin.ravel()), T.vtot, len(T.pseudo), npts, nproj, idx,
                                       beta, wgt, 2, np.ascontiguousarray(psi), h) == 0
        ref = pw.mult_spinor(T, psi)
        assert np.abs(h - ref).max() / np.abs(ref).max() < 1e-13, (kind, nc)


def test_compiled_reference_threaded_sweep_matches_restatement():
    """The multi-threaded form of the compiled composition (bands spread over
    OpenMP threads, one Fourier per thread) that the CPU baseline times: every
    band against the restatement, 1e-13."""
    import ctypes as C

    from oracle import build_ref
    lib_path = build_ref.LIB_HPSI
    if not lib_path.exists():
        pytest.skip("reference composition not built here (oracle/_ref)")
    lib = C.CDLL(str(lib_path))
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    lib.ref_add_mult_spinor_omp.argtypes = [ip, ip, dp, dp, dp, C.c_int, ip, ip, ip, dp, dp, C.c_int, dp, dp,
                                            C.c_int]
    nc = (16, 16, 16)
    nf = (32, 32, 32)
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 21)
    T, _ = pw.build_tables(L, z, pos, nc, nf, seed_v=22)
    psi = pw.random_orthonormal_psi(T.dm.ntot, 7, 23)
    npts = np.array([len(at[0].idx) for at in T.pseudo], np.int32)
    nproj = np.array([len(at) for at in T.pseudo], np.int32)
    idx = np.concatenate([at[0].idx for at in T.pseudo]).astype(np.int32)
    beta = np.concatenate([pp.val[:, 0] for at in T.pseudo for pp in at]).astype(np.float64)
    wgt = np.array([pp.wgt for at in T.pseudo for pp in at], np.float64)
    h = np.zeros_like(psi)
    assert lib.ref_add_mult_spinor_omp(np.array(nc, np.int32), np.array(nf, np.int32), np.array(L, np.float64),
                                       np.ascontiguousarray(T.ekin.ravel()), T.vtot, len(T.pseudo), npts, nproj, idx,
                                       beta, wgt, 7, np.ascontiguousarray(psi), h, 3) == 0
    ref = pw.mult_spinor(T, psi)
    assert np.abs(h - ref).max() / np.abs(ref).max() < 1e-13


def test_smearing_matches_reference_functions():
    """The occupation rate and -T S term of one state for both smearing schemes
    (Fermi-Dirac "FD", Gaussian "GB") against the reference's wgauss /
    getEntropy compiled from its source (ref_smearing.npz, 400 seeded points):
    the oracle's restatement and the band-distributed SCF's host copy."""
    from oracle import scf
    from pwdft_develop_b200.parallel import fermi_entropy
    g = np.load(Path(__file__).resolve().parent / "golden" / "ref_smearing.npz")
    ev, ef, tb, out = g["ev"], g["ef"], g["tbeta"], g["out"]
    for j, sm in enumerate(("FD", "GB")):
        w = np.array([scf.wgauss(ev[i], ef[i], tb[i], sm) for i in range(len(ev))])
        e = np.array([scf.entropy(np.array([ev[i]]), ef[i], tb[i], sm)[0] for i in range(len(ev))])
        assert np.abs(w - out[:, j]).max() <= 1e-15
        assert np.abs(e - out[:, 2 + j]).max() <= 1e-15 * max(1.0, np.abs(out[:, 2 + j]).max())
    e = np.array([fermi_entropy(np.array([ev[i]]), ef[i], tb[i])[0] for i in range(len(ev))])
    assert np.abs(e - out[:, 2]).max() <= 1e-15
    # the electron count the bisection fixes, either scheme
    eig = np.sort(np.random.default_rng(5).uniform(-0.3, 0.4, 24))
    for sm in ("FD", "GB"):
        occ, efermi = scf.occupations(eig, 16, 315774.67 / 3000.0, sm)
        assert abs(occ.sum() - 16) < 1e-10
