"""Broyden potential mixing and the density-change convergence test of the
device SCF against the FP64 oracle (tests/golden/si8_scf_broyden.json, the
oracle's SCF::BroydenMix run converged to scfNorm < 1e-13).  Tolerances:
E_free 1e-6 Ha/atom, eigenvalues 1e-6 Ha."""
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("solver,mixed", [("chebfsi", False), ("lobpcg", False), ("chebfsi", True)])
def test_scf_broyden_matches_oracle(solver, mixed):
    from pwdft_develop_b200 import Context
    g = json.loads((GOLD / "si8_scf_broyden.json").read_text())
    L = np.array(g["length"])
    pos = np.array(g["positions"])
    c = Context(L, tuple(g["numGrid"]), tuple(g["numGridFine"]))
    c.set_atoms([g["znuc"]] * len(pos), pos)
    res, eig, rho = c.scf(nocc=16, nextra=8, ecut=g["ecut"], solver=solver, mixed=mixed, eig_max_iter=4,
                          eig_tol=1e-10, max_iter=80, mix="broyden", tol_rho=1e-12,
                          wfn_filter=False)
    assert res["converged"] == 1
    assert res["scf_norm"] < 1e-12
    nat = len(pos)
    assert abs(res["efree"] - g["efree"]) / nat < 1e-6, (res["efree"], g["efree"])
    assert np.abs(eig[:16] - np.array(g["eig"][:16])).max() < 1e-6


def test_anderson_with_the_density_criterion():
    """Anderson converged on scfNorm reaches the Anderson golden's energy."""
    from pwdft_develop_b200 import Context
    g = json.loads((GOLD / "si8_scf_small.json").read_text())
    L = np.array(g["length"])
    pos = np.array(g["positions"])
    c = Context(L, tuple(g["numGrid"]), tuple(g["numGridFine"]))
    c.set_atoms([g["znuc"]] * len(pos), pos)
    res, eig, rho = c.scf(nocc=16, nextra=8, ecut=g["ecut"], solver="chebfsi", eig_max_iter=4, eig_tol=1e-10,
                          max_iter=80, tol_rho=1e-12, wfn_filter=False)
    assert res["converged"] == 1 and res["scf_norm"] < 1e-12
    assert abs(res["efree"] - g["efree"]) / len(pos) < 1e-6
