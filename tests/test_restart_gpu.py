"""DEN / POT / WFN_<rank> restart files in the reference's serialize() layout
(include/utility.hpp:1183-1278; written by SCF::Iterate, src/SCF/scf.cpp:
1070-1145, read back at :164-178 and :296-330), parsed independently here, and
an SCF restarted from them.  Tolerances: bitwise round trips; the restarted
SCF reproduces E_free to 1e-8 Ha/atom within 3 iterations."""
import json
import struct
from pathlib import Path

import numpy as np
import pytest

from pwdft_develop_b200 import PwError

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def _vec(raw, off):
    (n,) = struct.unpack_from("=i", raw, off)
    return np.frombuffer(raw, np.float64, n, off + 4), off + 4 + 8 * n


def _ctx():
    from pwdft_develop_b200 import Context
    g = json.loads((GOLD / "si8_scf_small.json").read_text())
    L, pos = np.array(g["length"]), np.array(g["positions"])
    c = Context(L, tuple(g["numGrid"]), tuple(g["numGridFine"]))
    c.set_atoms([g["znuc"]] * len(pos), pos)
    return c, g


def test_layouts_and_round_trips(tmp_path):
    c, g = _ctx()
    N = g["numGridFine"]
    rng = np.random.default_rng(1)
    rho = rng.uniform(0, 0.1, c.ntotFine)
    c.write_density(tmp_path / "DEN", rho)
    raw = (tmp_path / "DEN").read_bytes()
    off = 0
    for d in range(3):
        gp, off = _vec(raw, off)
        assert np.array_equal(gp, np.arange(N[d]) / N[d])
    r2, off = _vec(raw, off)
    assert off == len(raw) and np.array_equal(r2, rho)
    assert np.array_equal(c.read_density(tmp_path / "DEN"), rho)
    c.write_potential(tmp_path / "POT", -rho)
    raw = (tmp_path / "POT").read_bytes()
    off = 0
    for d in range(3):
        _, off = _vec(raw, off)
    m, n = struct.unpack_from("=ii", raw, off)
    assert (m, n) == (c.ntotFine, 1)
    assert np.array_equal(np.frombuffer(raw, np.float64, m, off + 8), -rho)
    psi = rng.standard_normal((5, c.ntot))
    occ = np.array([1, 1, 1, 0.5, 0.0])
    c.write_wfn(tmp_path / "WFN_0", psi, occ)
    raw = (tmp_path / "WFN_0").read_bytes()
    m, n, p = struct.unpack_from("=iii", raw, 0)
    assert (m, n, p) == (c.ntot, 1, 5)
    assert np.array_equal(np.frombuffer(raw, np.float64, m * p, 12).reshape(p, m), psi)
    o2, off = _vec(raw, 12 + 8 * m * p)
    assert off == len(raw) and np.array_equal(o2, occ)
    x, o = c.read_wfn(tmp_path / "WFN_0")
    assert np.array_equal(x, psi) and np.array_equal(o, occ)


def test_mismatched_files_are_errors(tmp_path):
    from pwdft_develop_b200 import Context
    c, g = _ctx()
    c.write_density(tmp_path / "DEN", np.zeros(c.ntotFine))
    c.write_wfn(tmp_path / "WFN_0", np.zeros((2, c.ntot)), np.ones(2))
    other = Context(np.array(g["length"]), (24, 24, 24), (48, 48, 48))
    with pytest.raises(PwError, match="grid"):
        other.read_density(tmp_path / "DEN")
    with pytest.raises(PwError, match="layout"):
        other.read_wfn(tmp_path / "WFN_0")


def test_scf_restarts_from_den_and_wfn(tmp_path):
    c, g = _ctx()
    res, eig, rho = c.scf(nocc=16, nextra=8, ecut=g["ecut"], solver="chebfsi", tol_efree=1e-9, eig_max_iter=4,
                          eig_tol=1e-10, max_iter=80)
    assert res["converged"] == 1
    occ, psi, rho_d = c.scf_state()
    c.write_density(tmp_path / "DEN", rho_d.cpu().numpy())
    c.write_wfn(tmp_path / "WFN_0", psi.cpu().numpy(), occ)
    from pwdft_develop_b200.core import read_eig, write_eig
    write_eig(tmp_path / "EIG", eig)
    assert np.array_equal(read_eig(tmp_path / "EIG"), eig)
    c2, _ = _ctx()
    x, o = c2.read_wfn(tmp_path / "WFN_0")
    c2.scf_set_initial(rho=c2.read_density(tmp_path / "DEN"), psi=x)
    res2, eig2, _ = c2.scf(nocc=16, nextra=8, ecut=g["ecut"], solver="chebfsi", tol_efree=1e-9, eig_max_iter=4,
                           eig_tol=1e-10, max_iter=80)
    assert res2["converged"] == 1 and res2["iterations"] <= 3, res2["iterations"]
    assert abs(res2["efree"] - res["efree"]) / 8 < 1e-8
