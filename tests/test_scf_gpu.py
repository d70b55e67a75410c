"""Device eigensolvers, density and SCF against the FP64 oracle.
Tolerances: density 1e-12 relative (FP64), eigenvalues 1e-6 Ha, total energy
1e-6 Ha/atom (north-star parity bars)."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import pw, scf

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def _si8(nc=(16, 16, 16)):
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)
    return L, z, pos, nc, tuple(2 * n for n in nc)


def _ctx(L, z, pos, nc, nf, prec="f64"):
    from pwdft_develop_b200 import Context
    c = Context(L, nc, nf, precision=prec)
    c.set_atoms([z] * len(pos), pos)
    return c


@pytest.mark.parametrize("prec,tol", [("f64", 1e-12), ("f32", 1e-5)])
def test_density_matches_oracle(prec, tol):
    import torch
    L, z, pos, nc, nf = _si8()
    T, _ = pw.build_tables(L, z, pos, nc, nf, seed_v=3)
    psi = pw.random_orthonormal_psi(T.dm.ntot, 21, 4)
    occ = np.linspace(1.0, 0.2, 21)
    ref = scf.density(T, psi, occ, nocc=16)
    c = _ctx(L, z, pos, nc, nf, prec)
    rho = c.density(torch.tensor(psi, dtype=c.torch_dtype, device="cuda"), occ, 16).cpu().numpy()
    assert np.abs(rho - ref).max() / np.abs(ref).max() <= tol
    assert abs(rho.sum() * T.dm.vol / T.dm.ntotFine - 32.0) < 1e-9


@pytest.mark.parametrize("nc", [(16, 16, 16), (48, 48, 48)])
def test_hartree_and_xc_match_oracle(nc):
    import torch
    L, z, pos, _, _ = _si8()
    if nc[0] == 48:
        L, z, pos = pw.make_crystal("Si", (2, 2, 2), 10.26, 0.02, 7)
    nf = tuple(2 * n for n in nc)
    dm = pw.Domain(tuple(L), nc, nf)
    rng = np.random.default_rng(3)
    rho = rng.uniform(0.0, 0.1, dm.ntotFine)
    rps = rng.uniform(0.0, 0.1, dm.ntotFine)
    ref = scf.hartree(dm, rho, rps, 10.0)
    c = _ctx(L, z, pos, nc, nf)
    vh = c.hartree(torch.tensor(rho - rps, device="cuda"), 10.0).cpu().numpy()
    assert np.abs(vh - ref).max() / np.abs(ref).max() < 1e-12
    rho[::97] = 1e-12     # bad points
    e_ref, v_ref = scf.xc_teter93(rho)
    e, v = c.xc(torch.tensor(rho, device="cuda"))
    assert np.abs(e.cpu().numpy() - e_ref).max() < 1e-14 and np.abs(v.cpu().numpy() - v_ref).max() < 1e-14


def test_cholqr_orthonormalises():
    import torch
    L, z, pos, nc, nf = _si8()
    c = _ctx(L, z, pos, nc, nf)
    g = torch.Generator(device="cuda").manual_seed(1)
    X = torch.randn((24, c.ntot), dtype=torch.float64, device="cuda", generator=g)
    X0 = X.clone()
    c.cholqr(X)
    G = X @ X.T
    assert float((G - torch.eye(24, device="cuda", dtype=torch.float64)).abs().max()) < 1e-12
    # same span: projection of X0 onto span(X) reproduces X0
    assert float((X0 - (X0 @ X.T) @ X).abs().max() / X0.abs().max()) < 1e-10


@pytest.mark.parametrize("solver", ["lobpcg", "chebfsi", "ppcg", "davidson"])
def test_eigsolve_fixed_potential(solver):
    """Lowest 24 eigenpairs of H[V] against ARPACK on the oracle operator."""
    import torch
    L, z, pos, nc, nf = _si8()
    T, _ = pw.build_tables(L, z, pos, nc, nf, seed_v=5)
    T.vtot = 0.3 * (T.vtot - T.vtot.mean())
    ref, _ = scf._eigsh(T, 24, tol=1e-12)
    c = _ctx(L, z, pos, nc, nf)
    c.set_vtot(T.vtot)
    X = torch.tensor(pw.random_orthonormal_psi(T.dm.ntot, 24, 9), device="cuda")
    # PPCG's cheap sub-block sweeps (no locking, no periodic Rayleigh-Ritz, as in
    # the reference) need more iterations on the clustered spectrum
    maxit = {"chebfsi": 300, "ppcg": 500}.get(solver, 200)
    degree = {"chebfsi": 12, "ppcg": 4, "davidson": 3}.get(solver, 12)
    tol = 1e-12 if solver == "davidson" else 1e-9     # Davidson converges on the Ritz-value change
    eig, res, it = c.eigsolve(X, solver=solver, maxit=maxit, tol=tol, degree=degree)
    # the occupied states (the lowest 16 of the 24-wide block; the top of a
    # filtered block converges at the rate of the filter edge, which is why
    # the SCF carries extra states)
    assert np.abs(eig[:16] - ref[:16]).max() < 1e-6, (eig - ref, it)


def _gold(which):
    p = GOLD / f"si8_scf_{which}.json"
    if not p.exists():
        pytest.skip(f"{p.name} missing")
    return json.loads(p.read_text())


@pytest.mark.parametrize("solver,mixed", [("lobpcg", False), ("chebfsi", False), ("chebfsi", True), ("ppcg", False),
                                          ("davidson", False), ("ppcg", True)])
def test_scf_si8_small_matches_oracle(solver, mixed):
    g = _gold("small")
    L = np.array(g["length"])
    pos = np.array(g["positions"])
    nc = tuple(g["numGrid"])
    c = _ctx(L, g["znuc"], pos, nc, tuple(g["numGridFine"]))
    res, eig, rho = c.scf(nocc=16, nextra=8, ecut=g["ecut"], solver=solver, mixed=mixed, tol_efree=1e-8,
                          eig_max_iter=4, eig_tol=1e-10, max_iter=80, wfn_filter=False)
    assert res["converged"] == 1
    nat = len(pos)
    assert abs(res["efree"] - g["efree"]) / nat < 1e-6
    assert np.abs(eig[:16] - np.array(g["eig"][:16])).max() < 1e-6


@pytest.mark.parametrize("solver,mixed", [("lobpcg", False), ("chebfsi", False), ("chebfsi", True)])
def test_scf_si8_full_matches_oracle(solver, mixed):
    """The Si8 configuration at its stated size: 24^3 / 48^3 grids, Ecut 10 Ha,
    16 occupied + 8 extra bands, Anderson mixing, against the oracle's
    converged SCF: E_free within 1e-6 Ha/atom, occupied eigenvalues 1e-6 Ha."""
    g = _gold("full")
    L = np.array(g["length"])
    pos = np.array(g["positions"])
    c = _ctx(L, g["znuc"], pos, tuple(g["numGrid"]), tuple(g["numGridFine"]))
    res, eig, rho = c.scf(nocc=16, nextra=8, ecut=g["ecut"], solver=solver, mixed=mixed, tol_efree=1e-8,
                          eig_max_iter=4, eig_tol=1e-10, max_iter=80, cheby_degree=12, refine_threshold=1e-6,
                          wfn_filter=False)
    assert res["converged"] == 1
    nat = len(pos)
    assert abs(res["efree"] - g["efree"]) / nat < 1e-6, (res["efree"], g["efree"])
    assert np.abs(eig[:16] - np.array(g["eig"][:16])).max() < 1e-6
    c.close()


def _si64_gold(which):
    p = GOLD / f"si64_scf_{which}.json"
    if not p.exists():
        pytest.skip(f"{p.name} missing")
    return json.loads(p.read_text())


@pytest.mark.parametrize("which,mixed", [("plain", False), ("plain", True), ("filter", False), ("filter", True)])
def test_scf_si64_matches_oracle(which, mixed):
    """The Si64 configuration (48^3 / 96^3, Ecut 20 Ha, 128 + 32 bands, ChebFSI
    degree 10) against the oracle's converged FP64 SCF of the same operator:
    unfiltered (si64_scf_plain.json) and with CheFSI's wavefunction cut-off
    filter (si64_scf_filter.json); FP64 and mixed precision.  Bars:
    |E_free - E_oracle| / N_atom < 1e-6 Ha, occupied eigenvalues 1e-6 Ha.
    The device SCF stops at |E_free - E_Harris| / N_atom < 1e-10: the energy
    criterion is second order in the density error and the eigenvalues first
    order, and at 1e-8 a mixed run could stop where E_Harris crosses E_free
    with occupied eigenvalues still ~1e-5 Ha from the fixed point."""
    g = _si64_gold(which)
    L = np.array(g["length"])
    pos = np.array(g["positions"])
    c = _ctx(L, g["znuc"], pos, tuple(g["numGrid"]), tuple(g["numGridFine"]))
    res, eig, rho = c.scf(nocc=g["nocc"], nextra=g["nextra"], ecut=g["ecut"], solver="chebfsi", mixed=mixed,
                          cheby_degree=10, cheby_first_cycles=5, tol_efree=1e-10, refine_threshold=3e-6,
                          max_iter=100, graphs=True, wfn_filter=bool(g["wfn_filter"]))
    assert res["converged"] == 1
    nat = len(pos)
    assert abs(res["efree"] - g["efree"]) / nat < 1e-6, (res["efree"], g["efree"])
    nocc = g["nocc"]
    assert np.abs(eig[:nocc] - np.array(g["eig"][:nocc])).max() < 1e-6
    c.close()


@pytest.mark.parametrize("solver,mixed", [("chebfsi", False), ("lobpcg", False), ("chebfsi", True)])
def test_scf_al4_gaussian_smearing_matches_oracle(solver, mixed):
    """A metal with the reference's Gaussian smearing (Smearing_Scheme GB,
    wgauss / getEntropy of src/utility.cpp:4404-4444) at 3000 K: fcc Al4,
    16^3 / 32^3, Ecut 5 Ha, 6 + 4 bands, its threefold level at the Fermi
    energy two-thirds occupied; E_free within 1e-6 Ha/atom of the oracle
    (al4_scf_gb.json), the eigenvalues of the occupied and partly occupied
    levels 1e-6 Ha (the top extra bands are not converged by every solver),
    occupations 1e-5."""
    p = GOLD / "al4_scf_gb.json"
    g = json.loads(p.read_text())
    pos = np.array(g["positions"])
    c = _ctx(np.array(g["length"]), g["znuc"], pos, tuple(g["numGrid"]), tuple(g["numGridFine"]))
    res, eig, rho = c.scf(nocc=6, nextra=4, ecut=g["ecut"], solver=solver, mixed=mixed, temperature=3000.0,
                          smearing="GB", tol_efree=1e-8, eig_max_iter=4, eig_tol=1e-10, max_iter=80, wfn_filter=False)
    assert res["converged"] == 1
    nat = len(pos)
    assert abs(res["efree"] - g["efree"]) / nat < 1e-6, res["efree"] - g["efree"]
    ge = np.array(g["eig"])
    occd = np.array(g["occ"]) > 1e-12
    assert np.abs(eig[occd] - ge[occd]).max() < 1e-6
    # occupations from the device eigenvalues by the oracle's bisection, against the golden's
    occ, _ = scf.occupations(eig, 6, 315774.67 / 3000.0, "GB")
    assert np.abs(occ - np.array(g["occ"])).max() < 1e-5
