"""Complex-band H(k) psi on the device against the FP64 oracle restatement of
Spinor::AddMultSpinorFine (complex; oracle/kpoints.py).  Tolerances: FP64
1e-12 relative, FP32 1e-5 relative (the H*psi parity bars)."""
import numpy as np
import pytest

from oracle import kpoints, pw

pytestmark = pytest.mark.gpu

KPTS = [(0.0, 0.0, 0.0), (0.11, -0.05, 0.23), (0.5 * 2 * np.pi / 10.26, 0.0, 0.25 * 2 * np.pi / 10.26)]


def _setup(nc=(16, 16, 16), nb=10):
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 3)
    nf = tuple(2 * n for n in nc)
    T, _ = pw.build_tables(L, z, pos, nc, nf, seed_v=6)
    psi = kpoints.random_complex_psi(T.dm.ntot, nb, 12)
    return L, z, pos, nc, nf, T, psi


def _ctx(L, z, pos, nc, nf, T, prec):
    from pwdft_develop_b200 import Context
    c = Context(L, nc, nf, precision=prec)
    c.set_atoms([z] * len(pos), pos)
    c.set_vtot(T.vtot)
    return c


@pytest.mark.parametrize("prec,tol", [("f64", 1e-12), ("f32", 1e-5)])
@pytest.mark.parametrize("k", KPTS)
def test_hpsi_k_matches_oracle(prec, tol, k):
    import torch
    L, z, pos, nc, nf, T, psi = _setup()
    ref = kpoints.mult_spinor_k(T, k, psi)
    c = _ctx(L, z, pos, nc, nf, T, prec)
    c.set_kpoint(k)
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    X = torch.tensor(psi, dtype=cdt, device="cuda")
    out = c.hpsi_k(X).cpu().numpy().astype(np.complex128)
    assert np.abs(out - ref).max() <= tol * np.abs(ref).max()
    ek, te = c.kpoint_tables()
    ek_ref, te_ref = kpoints.ekin_teter_k(T.dm, k)
    assert np.abs(ek - ek_ref).max() <= (1e-14 if prec == "f64" else 1e-6) * ek_ref.max()
    assert np.abs(te - te_ref).max() <= (1e-14 if prec == "f64" else 1e-6)


def test_hpsi_k_batches_and_accumulate():
    import torch
    L, z, pos, nc, nf, T, psi = _setup(nb=13)
    k = KPTS[1]
    ref = kpoints.mult_spinor_k(T, k, psi)
    c = _ctx(L, z, pos, nc, nf, T, "f64")
    c.set_band_batch(4)                          # two complex bands per internal batch
    c.set_kpoint(k)
    X = torch.tensor(psi, device="cuda")
    out = c.hpsi_k(X, out=torch.ones_like(X), accumulate=True).cpu().numpy()
    assert np.abs(out - 1.0 - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("prec,tol", [("f64", 1e-12), ("f32", 1e-5)])
def test_hpsi_kbatch_matches_per_k_oracle(prec, tol):
    """A 2x2x2 Monkhorst-Pack batch in one pass, batches straddling k-points."""
    import torch
    L, z, pos, nc, nf, T, psi = _setup(nb=6)
    b = 2 * np.pi / 10.26
    kpts = np.array([[i, j, l] for i in (0.25, -0.25) for j in (0.25, -0.25) for l in (0.25, -0.25)]) * b
    allpsi = np.stack([kpoints.random_complex_psi(T.dm.ntot, 6, 30 + i) for i in range(len(kpts))])
    c = _ctx(L, z, pos, nc, nf, T, prec)
    c.set_band_batch(10)                          # 5 complex bands per internal batch: straddles k boundaries
    c.set_kpoints(kpts)
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    out = c.hpsi_kbatch(torch.tensor(allpsi, dtype=cdt, device="cuda")).cpu().numpy().astype(np.complex128)
    for i, k in enumerate(kpts):
        ref = kpoints.mult_spinor_k(T, k, allpsi[i])
        assert np.abs(out[i] - ref).max() <= tol * np.abs(ref).max(), i
