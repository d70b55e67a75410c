"""Sphere-cut (G-space) path on the device against the FP64 oracle
(oracle/gspace.py, restating src/SCF/spinor.cpp:528-680,
src/EigenSolver/eigensolver.cpp:471-515, src/SCF/fourier.cpp:542-640).

Tolerances: sphere tables exact (indices, Miller indices) and 1e-15 (ekin,
Teter); projector matrix 1e-12 relative; H c FP64 1e-12, FP32 1e-5
relative; Teter 1e-15 (FP64); density 1e-12 (FP64); fixed-potential
eigenvalues 1e-7 Ha against the dense oracle operator; SCF: mixed against FP64
1e-6 Ha/atom."""
import numpy as np
import pytest

from oracle import gspace as gs
from oracle import pw

pytestmark = pytest.mark.gpu


def _setup(N=(32, 32, 32), ecut=10.0, nb=11, seed_v=2):
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 4)
    sp = gs.sphere(L, N, ecut)
    rng = np.random.Generator(np.random.Philox(seed_v))
    vt = rng.uniform(-1.0, 0.5, sp.ntot)
    c = gs.random_orthonormal_c(sp, nb, 17)
    return L, z, pos, sp, vt, c


def _ctx(L, N, ecut, prec="f64", z=None, pos=None, vt=None):
    from pwdft_develop_b200 import Context
    cx = Context.gspace(L, N, ecut, precision=prec)
    if z is not None:
        cx.set_atoms([z] * len(pos), pos)
    if vt is not None:
        cx.set_vtot(vt)
    return cx


def _dev(cx, c):
    import torch
    return torch.tensor(gs.real_view(c), dtype=cx.torch_dtype, device="cuda")


def _host(x):
    return gs.complex_view(x.double().cpu().numpy())


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_sphere_tables_match_oracle():
    L, z, pos, sp, vt, c = _setup()
    cx = _ctx(L, sp.N, sp.ecut)
    assert cx.ns == sp.ns and cx.ntot == 2 * sp.ns and cx.ntotFine == sp.ntot
    idx, mil, ek, te = cx.gs_sphere()
    assert np.array_equal(idx, sp.idx) and np.array_equal(mil, sp.m)
    np.testing.assert_allclose(ek, sp.ekin, rtol=1e-15, atol=0)
    np.testing.assert_allclose(te, sp.teter, rtol=1e-15, atol=0)


def test_projectors_match_oracle():
    L, z, pos, sp, vt, c = _setup()
    vn, w = gs.vnlc(sp, z, pos)
    cx = _ctx(L, sp.N, sp.ecut, z=z, pos=pos)
    got, gw = cx.gs_get_projectors()
    assert got.shape == vn.shape
    assert _rel(got, vn) <= 1e-12
    np.testing.assert_allclose(gw, w, rtol=1e-14)


@pytest.mark.parametrize("prec,tol", [("f64", 1e-12), ("f32", 1e-5)])
def test_hpsi_matches_oracle(prec, tol):
    import torch
    L, z, pos, sp, vt, c = _setup()
    vn, w = gs.vnlc(sp, z, pos)
    ref = gs.hpsi(sp, vt, c, vn, w)
    cx = _ctx(L, sp.N, sp.ecut, prec, z, pos, vt)
    X = _dev(cx, c)
    assert _rel(_host(cx.hpsi(X)), ref) <= tol
    # accumulate adds to what is there (both components)
    acc = _host(cx.hpsi(X, out=torch.ones_like(X), accumulate=True))
    assert _rel(acc - (1 + 1j), ref) <= 10 * tol
    # caller-supplied NonlocalMultX table (pw_gs_set_projectors)
    vn2 = vn[:, ::2] * 1.3
    w2 = w[::2] * 0.7
    cx.gs_set_projectors(vn2, w2)
    assert _rel(_host(cx.hpsi(X)), gs.hpsi(sp, vt, c, vn2, w2)) <= tol
    # no projectors: local + kinetic only
    cx.gs_set_projectors(np.zeros((sp.ns, 0), complex), np.zeros(0))
    assert _rel(_host(cx.hpsi(X)), gs.add_mult_spinor_gspace(sp, vt, c)) <= tol


def test_hpsi_on_the_si64_grid():
    """96^3 G-space grid (the 48^3 slot box of the bench), Ecut 25 Ha, 6 bands."""
    L, z, pos = pw.make_crystal("Si", (2, 2, 2), 10.26, 0.02, 20261203 + 2)
    sp = gs.sphere(L, (96, 96, 96), 25.0)
    rng = np.random.Generator(np.random.Philox(4))
    vt = rng.uniform(-1.0, 0.5, sp.ntot)
    c = gs.random_orthonormal_c(sp, 6, 8)
    vn, w = gs.vnlc(sp, z, pos)
    ref = gs.hpsi(sp, vt, c, vn, w)
    for prec, tol in (("f64", 1e-12), ("f32", 1e-5)):
        cx = _ctx(L, sp.N, sp.ecut, prec, z, pos, vt)
        assert _rel(_host(cx.hpsi(_dev(cx, c))), ref) <= tol


def test_teter_and_density_match_oracle():
    L, z, pos, sp, vt, c = _setup()
    cx = _ctx(L, sp.N, sp.ecut, z=z, pos=pos, vt=vt)
    X = _dev(cx, c)
    assert _rel(_host(cx.teter(X)), gs.add_teter_precond(sp, c)) <= 1e-15
    occ = np.linspace(1.0, 0.3, c.shape[0])
    rho = cx.density(X, occ, 8).cpu().numpy()
    assert _rel(rho, gs.density(sp, c, occ, nocc=8)) <= 1e-12


@pytest.mark.parametrize("solver", ["lobpcg", "chebfsi", "davidson", "ppcg"])
def test_eigsolve_fixed_potential(solver):
    """Lowest eigenpairs of the sphere-cut H against the dense oracle operator
    (Si8, 24^3, Ecut 6 Ha: 739 real degrees of freedom)."""
    import torch
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 4)
    sp = gs.sphere(L, (24, 24, 24), 6.0)
    rng = np.random.Generator(np.random.Philox(5))
    vt = 0.3 * rng.uniform(-1.0, 0.5, sp.ntot)
    vn, w = gs.vnlc(sp, z, pos)
    keep = np.ones(2 * sp.ns, bool)
    keep[1] = False
    E = np.eye(2 * sp.ns)[keep]
    H = np.concatenate([gs.real_view(gs.hpsi(sp, vt, gs.complex_view(E[i:i + 256]), vn, w))
                        for i in range(0, E.shape[0], 256)])[:, keep]
    ref = np.linalg.eigvalsh(0.5 * (H + H.T))[:24]
    cx = _ctx(L, sp.N, sp.ecut, z=z, pos=pos, vt=vt)
    X = torch.tensor(gs.real_view(gs.random_orthonormal_c(sp, 24, 9)), device="cuda")
    maxit = {"chebfsi": 300, "ppcg": 500}.get(solver, 200)
    degree = {"chebfsi": 12, "ppcg": 4, "davidson": 3}.get(solver, 12)
    tol = 1e-12 if solver == "davidson" else 1e-9
    eig, res, it = cx.eigsolve(X, solver=solver, maxit=maxit, tol=tol, degree=degree)
    assert np.abs(eig[:16] - ref[:16]).max() < 1e-7, (eig[:16] - ref[:16], it)
    # Im c_0 stays zero and the Ritz vectors are orthonormal in Re(X^H X)
    Xh = X.cpu().numpy()
    assert np.abs(Xh[:, 1]).max() == 0.0
    G = Xh @ Xh.T
    assert np.abs(G - np.eye(24)).max() < 1e-10


def test_scf_gspace_fp64_and_mixed():
    """SCF::Iterate on a sphere-cut context: converges; the mixed form agrees
    with FP64; the energy is that of the dual-grid run of the same cell to the
    discretisation difference (5 mHa/atom)."""
    from pwdft_develop_b200 import Context
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)
    out = {}
    for mixed in (False, True):
        cx = _ctx(L, (32, 32, 32), 10.0, z=z, pos=pos)
        res, eig, rho = cx.scf(nocc=16, nextra=8, ecut=10.0, solver="chebfsi", mixed=mixed, tol_efree=1e-8,
                               eig_max_iter=4, eig_tol=1e-10, max_iter=80)
        assert res["converged"] == 1, res
        assert abs(rho.sum() * np.prod(L) / 32 ** 3 - 32.0) < 1e-8
        out[mixed] = (res["efree"], eig)
    nat = len(pos)
    assert abs(out[True][0] - out[False][0]) / nat < 1e-6
    assert np.abs(out[True][1][:16] - out[False][1][:16]).max() < 1e-6
    rs = Context(L, (16, 16, 16), (32, 32, 32))
    rs.set_atoms([z] * nat, pos)
    res, eig, rho = rs.scf(nocc=16, nextra=8, ecut=10.0, solver="chebfsi", tol_efree=1e-8, eig_max_iter=4,
                           eig_tol=1e-10, max_iter=80)
    assert abs(res["efree"] - out[False][0]) / nat < 5e-3, (res["efree"], out[False][0])


def test_real_space_only_entry_points_refuse():
    L, z, pos, sp, vt, c = _setup()
    cx = _ctx(L, sp.N, sp.ecut, z=z, pos=pos, vt=vt)
    with pytest.raises(RuntimeError, match="real-space"):
        cx.set_kpoint([0.1, 0.0, 0.0])


# bars of the sphere-cut exchange: kernel, V_x c, Fock energy (full / ACE), H c with exchange
EXX_TOL = {"f64": (1e-14, 1e-12, 1e-12, 1e-11, 1e-11), "f32": (1e-6, 2e-5, 1e-6, 1e-6, 2e-5)}


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("mu", [0.0, 0.106])
def test_exchange_matches_oracle(mu, prec):
    """Sphere-cut AddMultSpinorEXX (spinor.cpp:783-945) on the device against
    the FP64 oracle, FP64 and FP32 pair fields: kernel and exxDiv 1e-14 (FP32
    kernel 1e-6), V_x c 1e-12 (2e-5), the Fock energy with the full operator
    1e-12 (1e-6) and with ACE built from the same bands 1e-11 (1e-6), H c with
    the exchange term (full and ACE) 1e-11 (2e-5); batches cut by the scratch
    budget are invisible."""
    tk, tv, te, ta, th = EXX_TOL[prec]
    import torch
    from pwdft_develop_b200._lib import lib
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 4)
    sp = gs.sphere(L, (24, 24, 24), 6.0)
    c = gs.random_orthonormal_c(sp, 10, 11)
    occ = np.concatenate([np.ones(7), [0.6, 0.1, 0.0]])
    k, div = gs.exx_kernel(sp, 6.0, mu=mu, div_type=1)
    vx = gs.add_mult_spinor_exx(sp, c, gs.set_phi(sp, c), k, 0.25, occ)
    e_ref = float(np.sum(occ * np.real(np.sum(c.conj() * vx, axis=1))))
    rng = np.random.Generator(np.random.Philox(6))
    vt = rng.uniform(-1.0, 0.5, sp.ntot)
    cx = _ctx(L, sp.N, sp.ecut, prec, z=z, pos=pos, vt=vt)
    cx.exx_setup(0.25, mu, 1, 6.0)
    d, kern = cx.exx_kernel()
    assert abs(d - div) <= 1e-14 * abs(div)
    full = np.concatenate([k, np.conj(k[:, :, 1:-1][:, :, ::-1])], axis=2)   # even kernel: the full grid
    np.testing.assert_allclose(kern, full.real, rtol=tk, atol=tk * np.abs(k).max())
    X = _dev(cx, c)
    cx.exx_set_phi(X, occ)
    assert _rel(_host(cx.exx_apply(X)), vx) <= tv
    field = 3 * 24 ** 3 * (16 if prec == "f64" else 8)
    assert lib.pw_exx_set_scratch(cx.handle, field) == 0     # 3 pair fields per batch
    assert _rel(_host(cx.exx_apply(X)), vx) <= tv
    e_full = cx.exx_energy(X, occ)
    assert abs(e_full - e_ref) <= te * abs(e_ref)
    h0 = _host(cx.hpsi(X))
    cx.exx_set_mode("full")
    assert _rel(_host(cx.hpsi(X)), h0 + vx) <= th
    cx.ace_build(X)
    assert abs(cx.exx_energy(X, occ, use_ace=True) - e_ref) <= ta * abs(e_ref)
    assert _rel(_host(cx.hpsi(X)), h0 + vx) <= th


def test_scf_gspace_hse06():
    """The nested HSE06 hybrid SCF on a sphere-cut FP64 context (the
    reference's default mode): converges (dExx < 1e-8), the Fock energy is
    negative and equals the exchange energy of the final ACE on its own bands,
    and the total energy is below the PBE SCF of the same cell by the hybrid's
    exchange-correlation difference (a few 10 mHa/atom, sign only checked)."""
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)
    out = {}
    for xc in ("pbe", "hse06"):
        cx = _ctx(L, (24, 24, 24), 6.0, z=z, pos=pos)
        res, eig, rho = cx.scf(nocc=16, nextra=8, ecut=6.0, solver="chebfsi", tol_efree=1e-8, eig_max_iter=4,
                               eig_tol=1e-10, max_iter=80, xc=xc, phi_max_iter=20, phi_tol=1e-8)
        assert res["converged"] == 1, (xc, res)
        assert abs(rho.sum() * np.prod(L) / 24 ** 3 - 32.0) < 1e-8
        out[xc] = res
    h = out["hse06"]
    assert h["efock"] < 0 and h["dexx"] < 1e-8 and h["phi_iterations"] >= 1
    assert h["efree"] < out["pbe"]["efree"]


def test_scf_gspace_broyden_and_pbe():
    """Broyden mixing and PBE on a sphere-cut context: Broyden (converged on
    the density change) reaches the Anderson fixed point (E_free 1e-6
    Ha/atom), and the PBE SCF lands within the discretisation difference
    (5 mHa/atom) of the dual-grid PBE SCF of the same cell."""
    from pwdft_develop_b200 import Context
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)
    nat = len(pos)
    kw = dict(nocc=16, nextra=8, ecut=10.0, solver="chebfsi", eig_max_iter=4, eig_tol=1e-10, max_iter=80)
    cx = _ctx(L, (32, 32, 32), 10.0, z=z, pos=pos)
    ra, _, _ = cx.scf(tol_efree=1e-8, **kw)
    rb, _, _ = cx.scf(mix="broyden", tol_rho=1e-13, tol_efree=1e-8, **kw)
    assert ra["converged"] == 1 and rb["converged"] == 1
    assert abs(ra["efree"] - rb["efree"]) / nat < 1e-6, (ra["efree"], rb["efree"])
    rp, _, _ = cx.scf(xc="pbe", tol_efree=1e-8, **kw)
    rs = Context(L, (16, 16, 16), (32, 32, 32))
    rs.set_atoms([z] * nat, pos)
    rr, _, _ = rs.scf(xc="pbe", tol_efree=1e-8, **kw)
    assert rp["converged"] == 1 and rr["converged"] == 1
    assert abs(rp["efree"] - rr["efree"]) / nat < 5e-3, (rp["efree"], rr["efree"])
