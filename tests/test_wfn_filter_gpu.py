"""The wavefunction cut-off filter of KohnSham::MultSpinor (the CheFSI path,
src/SCF/hamiltonian.cpp:316-321, 3090-3116, 3240-3265) on the device against
the FP64 oracle: the in-place filter P X, H*psi with the exit filter (P H psi,
dense and real-space projector modes, with ACE and with the full pair-FFT
exchange), the unfiltered accumulate call, the filtered eigenproblem and the
filtered ChebFSI SCF (tests/golden/si8_scf_small_filter.json).  Tolerances:
FP64 1e-12 and FP32 1e-5 relative; eigenvalues and E_free 1e-6 Ha (per atom)."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import exx, pw, scf

pytestmark = pytest.mark.gpu
TOL = {"f64": 1e-12, "f32": 1e-5}
ECUT = 10.0


def _setup(nc=(24, 24, 24), nb=9):
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)
    nf = tuple(2 * n for n in nc)
    T, _ = pw.build_tables(L, z, pos, nc, nf, seed_v=12)
    psi = pw.random_orthonormal_psi(T.dm.ntot, nb, 13)
    return L, z, pos, nc, nf, T, psi


def _ctx(L, z, pos, nc, nf, T, prec, mode="dense"):
    from pwdft_develop_b200 import Context
    c = Context(L, nc, nf, precision=prec)
    c.set_nonlocal_mode(mode)
    c.set_atoms([z] * len(pos), pos)
    c.set_vtot(T.vtot)
    return c


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_filter_in_place_matches_oracle(prec):
    import torch
    L, z, pos, nc, nf, T, psi = _setup()
    ref = pw.wfn_ecut_filter(T, psi, ECUT)
    c = _ctx(L, z, pos, nc, nf, T, prec)
    c.set_wfn_filter(ECUT)
    X = torch.tensor(psi, dtype=c.torch_dtype, device="cuda")
    c.wfn_filter(X)
    assert _rel(X.double().cpu().numpy(), ref) <= TOL[prec]
    # idempotent
    Y = X.clone()
    c.wfn_filter(Y)
    assert _rel(Y.double().cpu().numpy(), X.double().cpu().numpy()) <= TOL[prec]


@pytest.mark.parametrize("prec,mode", [("f64", "dense"), ("f32", "dense"), ("f64", "realspace"),
                                       ("f32", "realspace")])
def test_hpsi_exit_filter_matches_oracle(prec, mode):
    """a3 = P H psi for an unfiltered psi (the exit filter alone), and the
    accumulating call (AddMultSpinorFineR2C) stays unfiltered."""
    import torch
    L, z, pos, nc, nf, T, psi = _setup()
    ref = pw.mult_spinor(T, psi, wfn_ecut=ECUT)
    c = _ctx(L, z, pos, nc, nf, T, prec, mode)
    c.set_wfn_filter(ECUT)
    X = torch.tensor(psi, dtype=c.torch_dtype, device="cuda")
    got = c.hpsi(X).double().cpu().numpy()
    assert _rel(got, ref) <= TOL[prec]
    base = np.random.default_rng(1).standard_normal(psi.shape)
    Y = torch.tensor(base, dtype=c.torch_dtype, device="cuda")
    c.hpsi(X, out=Y, accumulate=True)
    assert _rel(Y.double().cpu().numpy(), base + pw.mult_spinor(T, psi)) <= TOL[prec]
    # switched off again: the plain operator
    c.set_wfn_filter(None)
    assert _rel(c.hpsi(X).double().cpu().numpy(), pw.mult_spinor(T, psi)) <= TOL[prec]


@pytest.mark.parametrize("prec,mode", [("f64", "ace"), ("f32", "ace"), ("f64", "full"), ("f32", "full")])
def test_hpsi_exit_filter_with_exchange(prec, mode):
    """P (H + V_x) psi with the ACE operator and with the full pair-FFT exchange."""
    import torch
    L, z, pos, nc, nf, T, psi = _setup(nc=(16, 16, 16), nb=8)
    occ = np.ones(6)
    kern, _ = exx.exx_kernel_r2c(T.dm, ECUT)
    phi = exx.set_phi(T.dm, psi[:6])
    if mode == "ace":
        xi = exx.ace_build(T.dm, psi[:6], phi, kern, 0.25, occ)
        vx = exx.ace_apply(xi, psi)
    else:
        vx = exx.add_mult_spinor_exx(T.dm, psi, phi, kern, 0.25, occ)
    ref = pw.wfn_ecut_filter(T, pw.mult_spinor(T, psi) + vx, ECUT)
    c = _ctx(L, z, pos, nc, nf, T, prec)
    c.exx_setup(0.25, 0.0, 1, ECUT)
    X = torch.tensor(psi, dtype=c.torch_dtype, device="cuda")
    c.exx_set_phi(X[:6].contiguous(), occ)
    if mode == "ace":
        c.ace_build(X[:6].contiguous())
    else:
        c.exx_set_mode("full")
    c.set_wfn_filter(ECUT)
    got = c.hpsi(X).double().cpu().numpy()
    assert _rel(got, ref) <= (1e-10 if prec == "f64" else 1e-5)


def test_eigsolve_filtered_operator_matches_oracle():
    """Lowest eigenpairs of the filtered operator (ChebFSI with the filter on)
    against ARPACK on the oracle's P H P restricted to the span of P."""
    import torch
    L, z, pos, nc, nf, T, _ = _setup(nc=(16, 16, 16))
    T.vtot = 0.3 * (T.vtot - T.vtot.mean())
    ref, _ = scf._eigsh(T, 24, tol=1e-12, wfn_ecut=5.0)
    c = _ctx(L, z, pos, nc, nf, T, "f64")
    c.set_wfn_filter(5.0)
    X = torch.tensor(pw.random_orthonormal_psi(T.dm.ntot, 24, 9), device="cuda")
    eig, res, it = c.eigsolve(X, solver="chebfsi", maxit=300, tol=1e-9, degree=12)
    assert np.abs(eig[:16] - ref[:16]).max() < 1e-6, (eig - ref, it)
    # the Ritz vectors lie in the span of P
    Y = X.clone()
    c.wfn_filter(Y)
    assert float((Y - X).abs().max()) < 1e-10


@pytest.mark.parametrize("mixed", [False, True])
def test_scf_chebfsi_filter_matches_oracle(mixed):
    """ChebFSI SCF with the reference's default filter against the oracle's
    filtered SCF (Si8 16^3 / 32^3, Ecut 5 Ha)."""
    from pwdft_develop_b200 import Context
    p = Path(__file__).resolve().parent / "golden" / "si8_scf_small_filter.json"
    g = json.loads(p.read_text())
    assert g["wfn_filter"]
    L, pos = np.array(g["length"]), np.array(g["positions"])
    c = Context(L, tuple(g["numGrid"]), tuple(g["numGridFine"]))
    c.set_atoms([g["znuc"]] * len(pos), pos)
    res, eig, rho = c.scf(nocc=16, nextra=8, ecut=g["ecut"], solver="chebfsi", mixed=mixed, tol_efree=1e-8,
                          max_iter=80, cheby_degree=12, refine_threshold=1e-6)
    assert res["converged"] == 1
    assert abs(res["efree"] - g["efree"]) / len(pos) < 1e-6, (res["efree"], g["efree"])
    assert np.abs(eig[:16] - np.array(g["eig"][:16])).max() < 1e-6
    # the unfiltered run of the same cell lands elsewhere (the filter matters here)
    r2, _, _ = c.scf(nocc=16, nextra=8, ecut=g["ecut"], solver="chebfsi", tol_efree=1e-8, max_iter=80,
                     cheby_degree=12, wfn_filter=False)
    assert abs(r2["efree"] - g["efree"]) / len(pos) > 1e-4
