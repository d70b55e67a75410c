"""Sphere-cut (G-space) oracle (oracle/gspace.py) against the reference's
definitions and against published closed forms, on the CPU.

Tolerances: sphere maps exact; plane-wave and Hermiticity identities 1e-13;
the numerical Bessel transform of the HGH projectors against the closed-form
Gaussian transforms (Hartwigsen-Goedecker-Hutter 1998) 1e-7 relative; G-space
versus real-space (dual-grid) eigenvalues of the same V_tot 3e-3 Ha (two
different discretisations of one Hamiltonian)."""
import math

import numpy as np

from oracle import gspace as gs
from oracle import hgh, pw


def _si8(N=(32, 32, 32), ecut=10.0):
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 4)
    return L, z, pos, gs.sphere(L, N, ecut)


def test_sphere_maps_follow_the_reference_rules():
    L, z, pos, sp = _si8()
    m = sp.m
    # every stored point is in the R2C half with the G_x = 0 half-plane rule
    assert np.all((m[:, 0] > 0) | ((m[:, 0] == 0) & ((m[:, 1] > 0) | ((m[:, 1] == 0) & (m[:, 2] >= 0)))))
    assert sp.idx[0] == 0 and np.all(np.diff(sp.idx) > 0)      # G = 0 first, ascending R2C order
    # the stored half plus its mirror is the whole sphere, each point once
    full = {tuple(x) for x in m} | {tuple(-x) for x in m}
    assert len(full) == 2 * sp.ns - 1
    g = pw.gvec_full(pw.Domain(tuple(L), sp.N, sp.N)).reshape(-1, 3)
    assert len(full) == int(np.sum(0.5 * np.sum(g * g, axis=1) < sp.ecut))
    # padding pairs: G_x = 0 points with their mirror
    mm = gs.r2c_miller(sp.N)
    assert np.all(mm[sp.pad_dst] == -mm[sp.pad_src])
    assert np.all(mm[sp.pad_dst][:, 0] == 0)
    # ekin / Teter tables
    np.testing.assert_allclose(sp.ekin, 0.5 * np.sum(sp.g ** 2, axis=1), rtol=1e-15)
    a = 2 * sp.ekin
    b = 27 + a * (18 + a * (12 + 8 * a))
    np.testing.assert_allclose(sp.teter, b / (b + 16 * a ** 4), rtol=1e-15)


def test_plane_wave_in_constant_potential():
    L, z, pos, sp = _si8()
    v0 = 0.37
    for s in (0, 1, 17, sp.ns - 1):
        e = np.zeros((1, sp.ns), complex)
        e[0, s] = 1.0 if s == 0 else (0.6 - 0.8j)
        out = gs.hpsi(sp, np.full(sp.ntot, v0), e)
        np.testing.assert_allclose(out[0], e[0] * (sp.ekin + v0), atol=1e-13)


def test_hamiltonian_is_symmetric_in_the_real_gram():
    L, z, pos, sp = _si8()
    rng = np.random.Generator(np.random.Philox(3))
    vt = rng.uniform(-1, 0.5, sp.ntot)
    vn, w = gs.vnlc(sp, z, pos)
    x = gs.random_orthonormal_c(sp, 5, 1)
    y = gs.random_orthonormal_c(sp, 5, 2)
    A = np.real(x.conj() @ gs.hpsi(sp, vt, y, vn, w).T)
    B = np.real(gs.hpsi(sp, vt, x, vn, w).conj() @ y.T)
    assert np.abs(A - B).max() <= 1e-13 * np.abs(A).max()
    # the sqrt(2) convention: Re(c^H d) is the full-sphere inner product
    full = gs.c2r_unnormalised(sp, gs.to_r2c(sp, x))
    fully = gs.c2r_unnormalised(sp, gs.to_r2c(sp, y))
    np.testing.assert_allclose(full @ fully.T / sp.ntot, np.real(x.conj() @ y.T), atol=1e-13)


def test_bessel_and_simpson():
    x = np.array([0.0, 1e-3, 0.04, 0.3, 2.0, 7.5])
    j0 = np.where(x == 0, 1.0, np.sin(x) / np.where(x == 0, 1, x))
    np.testing.assert_allclose(gs.bessel(0, x), j0, rtol=1e-13)
    xs = x[1:]
    j1 = np.sin(xs) / xs ** 2 - np.cos(xs) / xs
    np.testing.assert_allclose(gs.bessel(1, xs), j1, rtol=1e-9, atol=1e-15)
    assert gs.bessel(1, np.array([0.0]))[0] == 0.0
    r = np.linspace(0, 2, 201)
    assert abs(gs.simpson(r ** 3, 0.01) - 4.0) < 1e-12


def test_projector_transform_matches_the_closed_form():
    """int r^2 p_i^l(r) j_l(q r) dr for the HGH Gaussians:
    i=1,l=0: sqrt(pi/2) a^3 e^{-q^2 a^2/2};  i=2,l=0: sqrt(pi/2) a^5 (3 - q^2 a^2) e^{-q^2a^2/2};
    i=1,l=1: sqrt(pi/2) a^5 q e^{-q^2a^2/2}; each times the HGH normalisation."""
    p = hgh._HGH_PARAMS[14]
    sp = hgh.hgh_table(14)
    tabs = gs.vq_tables(sp, 12.0)
    q = gs.DQ * np.arange(tabs[0][2].size)

    def closed(l, i, a):
        ex = l + (4 * i - 1) / 2.0
        norm = math.sqrt(2.0) / (a ** ex * math.sqrt(math.gamma(ex)))
        e = np.exp(-q * q * a * a / 2)
        if (l, i) == (0, 1):
            f = a ** 3 * e
        elif (l, i) == (0, 2):
            f = a ** 5 * (3 - q * q * a * a) * e
        elif (l, i) == (1, 1):
            f = a ** 5 * q * e
        else:
            raise ValueError
        return norm * math.sqrt(math.pi / 2) * f

    # channels are eigen-combinations of the radial functions (hgh_table)
    for k, (l, h, _, _) in enumerate(sp.proj):
        a = p["r0"] if l == 0 else p["r1"]
        # recover the combination from the table values at two radii
        r = np.array([0.3, 0.9])
        val = hgh.spl_eval(sp, ("val", k), r)
        fns = [hgh._proj_radial(l, i, a)[0] for i in (1, 2)]
        M = np.stack([f(r) for f in fns], axis=1)
        cf = np.linalg.solve(M, val) if l == 0 else np.array([val[0] / fns[0](r[:1])[0], 0.0])
        ref = cf[0] * closed(l, 1, a) + (cf[1] * closed(l, 2, a) if l == 0 else 0.0)
        got = tabs[k][2]
        assert np.abs(got - ref).max() <= 1e-7 * np.abs(ref).max(), (k, np.abs(got - ref).max())


def test_gspace_and_real_space_eigenvalues_agree():
    """The same V_tot through the sphere-cut H (N = 24) and the dual-grid H
    (12^3 coarse, 24^3 fine): the lowest eigenvalues agree to the
    discretisation difference."""
    L, z, pos, sp = _si8((24, 24, 24), 6.0)
    rng = np.random.Generator(np.random.Philox(7))
    vt = rng.uniform(-1, 0.5, sp.ntot)
    vn, w = gs.vnlc(sp, z, pos)
    keep = np.ones(2 * sp.ns, bool)
    keep[1] = False                        # Im c_0 is not a degree of freedom
    E = np.eye(2 * sp.ns)[keep]
    H = np.concatenate([gs.real_view(gs.hpsi(sp, vt, gs.complex_view(E[i:i + 256]), vn, w))
                        for i in range(0, E.shape[0], 256)])[:, keep]
    assert np.abs(H - H.T).max() <= 1e-13 * np.abs(H).max()
    eg = np.linalg.eigvalsh(0.5 * (H + H.T))[:12]
    T, _ = pw.build_tables(L, z, pos, (12, 12, 12), sp.N, vtot=vt)
    nc = T.dm.ntot
    I = np.eye(nc)
    Hr = np.concatenate([pw.mult_spinor(T, I[i:i + 512]) for i in range(0, nc, 512)])
    er = np.linalg.eigvalsh(0.5 * (Hr + Hr.T))[:12]
    assert np.abs(eg - er).max() <= 3e-3, np.abs(eg - er).max()


def test_gspace_exchange_matches_the_real_space_exchange():
    """Without the divergence correction the sphere-cut kernel (Fock set
    1/2|G|^2 < 4 Ecut) and the real-space kernel agree on every pair product of
    sphere functions (their spectra lie inside the Fock set), so the G-space
    V_x c equals the real-space V_x of the same functions on the same grid
    (oracle/exx.py, pinned against direct convolution) to 1e-13."""
    from oracle import exx
    L, z, pos, sp = _si8((24, 24, 24), 6.0)
    c = gs.random_orthonormal_c(sp, 6, 3)
    occ = np.linspace(1.0, 0.2, 6)
    dm = pw.Domain(tuple(L), sp.N, sp.N)
    psi_rs = gs.c2r_unnormalised(sp, gs.to_r2c(sp, c)) / math.sqrt(sp.ntot)
    for mu in (0.0, 0.106):
        k, _ = gs.exx_kernel(sp, 6.0, mu=mu, div_type=0)
        vg = gs.add_mult_spinor_exx(sp, c, gs.set_phi(sp, c), k, 0.25, occ)
        kr, _ = exx.exx_kernel_r2c(dm, 6.0, mu=mu, div_type=0)
        vr = exx.add_mult_spinor_exx(dm, psi_rs, exx.set_phi(dm, psi_rs), kr, 0.25, occ)
        ref = gs.from_r2c(sp, np.fft.rfftn(vr.reshape((-1,) + sp.N[::-1]), axes=(1, 2, 3))) / math.sqrt(sp.ntot)
        assert np.abs(vg - ref).max() <= 1e-13 * np.abs(vg).max()


def test_gspace_exchange_symmetric_negative_and_ace_exact():
    """Divergence type 1 (auxiliary function over eps < |G|^2 < 4 Ecut): the
    Gram Re(c^H V_x c) is symmetric and negative definite, Im (V_x c)_0 = 0,
    and the ACE operator built from the bands reproduces V_x on their span."""
    L, z, pos, sp = _si8((24, 24, 24), 6.0)
    c = gs.random_orthonormal_c(sp, 8, 5)
    occ = np.linspace(1.0, 0.1, 8)
    k, div = gs.exx_kernel(sp, 6.0, mu=0.106, div_type=1)
    assert div > 0
    v = gs.add_mult_spinor_exx(sp, c, gs.set_phi(sp, c), k, 0.25, occ)
    assert np.abs(v[:, 0].imag).max() == 0.0
    A = np.real(c.conj() @ v.T)
    assert np.abs(A - A.T).max() <= 1e-13 * np.abs(A).max()
    assert np.linalg.eigvalsh(0.5 * (A + A.T)).max() < 0
    W, X = gs.real_view(v), gs.real_view(c)
    M = -(X @ W.T)
    xi = np.linalg.solve(np.linalg.cholesky(0.5 * (M + M.T)), W)
    assert np.abs(-(X @ xi.T) @ xi - W).max() <= 1e-12 * np.abs(W).max()
