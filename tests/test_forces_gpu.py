"""Atomic forces (KohnSham::CalculateForce, hamiltonian.cpp:2670-3056) on the
device against the FP64 oracle (oracle/forces.py), and against a central finite
difference of the device SCF free energy.  Tolerances: 1e-10 relative for the
oracle comparison (FP64 throughout); the finite-difference bar is stated at the
test."""
import numpy as np
import pytest

from oracle import forces, pw

pytestmark = pytest.mark.gpu


def _setup(nc=(16, 16, 16), seed=20261203 + 5):
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.05, seed)
    nf = tuple(2 * n for n in nc)
    return L, z, pos, nc, nf


def _ctx(L, z, pos, nc, nf, mode="dense"):
    from pwdft_develop_b200 import Context
    c = Context(L, nc, nf, precision="f64")
    if mode != "dense":
        c.set_nonlocal_mode(mode)
    c.set_atoms([z] * len(pos), pos)
    return c


@pytest.mark.parametrize("mode", ["dense", "realspace"])
def test_forces_match_oracle(mode):
    import torch
    L, z, pos, nc, nf = _setup()
    T, sp = pw.build_tables(L, z, pos, nc, nf, seed_v=1)
    dm = T.dm
    psi = pw.random_orthonormal_psi(dm.ntot, 21, 11)
    occ = np.linspace(1.0, 0.05, 21)
    rng = np.random.default_rng(7)
    rho = rng.uniform(0.0, 0.2, dm.ntotFine)
    sets = [pw.pseudo_charge(pw.Atom(z, p), dm, sp) for p in pos]
    rho_ps = np.zeros(dm.ntotFine)
    for idx, val in sets:
        rho_ps[idx] += val[:, 0]
    ref_loc = forces.local_force(dm, rho, rho_ps, [(idx, val[:, 0]) for idx, val in sets])
    ref_nl = forces.nonlocal_force(T, psi, occ)
    c = _ctx(L, z, pos, nc, nf, mode)
    F, Floc, Fnl = c.forces(torch.tensor(rho, device="cuda"), torch.tensor(psi, device="cuda"), occ)
    assert np.abs(Floc - ref_loc).max() <= 1e-10 * np.abs(ref_loc).max(), (Floc, ref_loc)
    assert np.abs(Fnl - ref_nl).max() <= 1e-10 * np.abs(ref_nl).max(), (Fnl, ref_nl)
    assert np.abs(F - (Floc + Fnl)).max() == 0.0


def test_forces_num_spin_and_occupation_scaling():
    """The nonlocal part is linear in numSpin * occ; the local part ignores both."""
    import torch
    L, z, pos, nc, nf = _setup()
    c = _ctx(L, z, pos, nc, nf)
    psi = torch.tensor(pw.random_orthonormal_psi(c.ntot, 10, 3), device="cuda")
    rho = torch.full((c.ntotFine,), 0.05, dtype=torch.float64, device="cuda")
    occ = np.ones(10)
    _, l2, n2 = c.forces(rho, psi, occ, num_spin=2)
    _, l1, n1 = c.forces(rho, psi, 0.5 * occ, num_spin=1)
    assert np.array_equal(l1, l2)
    assert np.abs(4 * n1 - n2).max() <= 1e-13 * np.abs(n2).max()


def test_scf_forces_finite_difference():
    """F_x of one atom against -(E_free(x+h) - E_free(x-h)) / 2h from two more
    converged SCF runs.  The analytic force is the reference's integration-by-
    parts form, exact in the continuum; on a 32^3 fine grid the pseudocharge
    sampling ("egg-box"), the O(h^2) difference error and the SCF tolerance
    leave ~4e-5 Ha/bohr (measured on a B200) against forces of ~1e-2 Ha/bohr;
    the bar is 2e-4 Ha/bohr."""
    L, z, pos, nc, nf = _setup()
    kw = dict(nocc=16, nextra=8, ecut=10.0, solver="chebfsi", wfn_filter=False, tol_efree=1e-10, eig_max_iter=4, eig_tol=1e-11,
              max_iter=120, cheby_degree=12)
    c = _ctx(L, z, pos, nc, nf)
    res, _, _ = c.scf(**kw)
    assert res["converged"] == 1
    F, Floc, Fnl = c.scf_forces()
    a, d, h = 3, 0, 0.02
    e = []
    for s in (+1, -1):
        p2 = np.array(pos, dtype=np.float64).copy()
        p2[a, d] += s * h
        c2 = _ctx(L, z, p2, nc, nf)
        r2, _, _ = c2.scf(**kw)
        assert r2["converged"] == 1
        e.append(r2["efree"])
    fd = -(e[0] - e[1]) / (2 * h)
    assert abs(F[a, d] - fd) < 2e-4, (F[a, d], fd, Floc[a, d], Fnl[a, d])
    # Newton's third law holds up to the same grid error (measured 2e-5)
    assert np.abs(F.sum(axis=0)).max() < 2e-4
