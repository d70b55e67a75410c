"""The adjoint/forces configuration at scale: Si216 (3x3x3 diamond cells,
a = 30.78 bohr, seeded +-0.05 bohr displacements, 72^3 / 144^3 grids, 432
occupied + 48 extra bands), mixed-precision ChebFSI SCF, then on the same SCF
state: forces (KohnSham::CalculateForce form), the band-energy backward
(d/dR of all 216 atoms through the projector derivatives, dE/dV_loc on the
density grid), checked by central differences with step 1e-4 bohr on 8
seeded atoms (bar 1e-5 Ha/bohr, the forces parity bar) and against the
reference-form nonlocal forces (bar 1e-7 Ha/bohr)."""
import numpy as np
import pytest

from oracle import pw

pytestmark = pytest.mark.gpu


def test_si216_forces_and_backward():
    import torch
    from pwdft_develop_b200 import Context
    L, z, pos = pw.make_crystal("Si", (3, 3, 3), 10.26, 0.05, 20261203 + 5)
    pos = np.asarray(pos, np.float64)
    nc, nf = (72, 72, 72), (144, 144, 144)
    c = Context(L, nc, nf, precision="f64")
    c.set_atoms([z] * len(pos), pos)
    res, eig, _ = c.scf(nocc=432, nextra=48, ecut=15.0, solver="chebfsi", mixed=True, cheby_degree=10,
                        tol_efree=1e-6, refine_threshold=3e-6, max_iter=80, graphs=True)
    assert res["converged"] == 1, res
    F, Floc, Fnl = c.scf_forces()
    assert F.shape == (216, 3)
    assert np.abs(F.sum(axis=0)).max() < 1e-3
    occ, psi, _ = c.scf_state()
    w = 2.0 * occ
    dv, dr = c.band_energy_backward(psi, w)
    # the reference-form nonlocal force and the analytic-derivative backward agree
    assert np.abs(-dr - Fnl).max() < 1e-7, np.abs(-dr - Fnl).max()
    # dE/dV_loc: the weighted band density, integrating to sum(w) N_c / N_f * N_f / N_c
    g = dv.cpu().numpy()
    assert g.min() >= 0.0 and abs(g.sum() - w.sum()) < 1e-6 * w.sum()
    # central differences of the band energy at fixed psi
    vt = np.zeros(int(np.prod(nf)))       # V_loc does not depend on R: any fixed potential will do
    h = 1e-4
    rng = np.random.default_rng(20261203 + 5)
    for a, d in zip(rng.choice(216, 8, replace=False), rng.integers(0, 3, 8)):
        e = []
        for s in (+1, -1):
            p2 = pos.copy()
            p2[a, d] += s * h
            c2 = Context(L, nc, nf, precision="f64")
            c2.set_atoms([z] * len(p2), p2)
            c2.set_vtot(vt)
            e.append(c2.band_energy(psi, w))
            c2.close()
        fd = (e[0] - e[1]) / (2 * h)
        assert abs(dr[a, d] - fd) < 1e-5, (a, d, dr[a, d], fd)
