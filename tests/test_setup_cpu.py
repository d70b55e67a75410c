"""The library's own HGH set-up (C++, host only) against the oracle:
projector index sets and VAL/DX/DY/DZ columns, weights, pseudocharge and
self energy."""
import numpy as np
import pytest

from oracle import hgh, pw
from pwdft_develop_b200 import core


@pytest.fixture(scope="module")
def crystal():
    return pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)


@pytest.mark.parametrize("znuc", [14, 13])
def test_species_constants(znuc):
    sp = hgh.hgh_table(znuc, with_splines=False)
    info = core.hgh_species(znuc)
    assert info["zion"] == sp.zion
    assert info["nproj"] == 5
    assert abs(info["eself"] - sp.eself) < 1e-12 * abs(sp.eself)
    assert info["rcut_nonlocal"] == sp.wavcut == 3.5


def test_unknown_species_rejected():
    from pwdft_develop_b200 import PwError
    with pytest.raises(PwError):
        core.hgh_species(6)


@pytest.mark.parametrize("atom", [0, 5])
def test_projectors_match_oracle(crystal, atom):
    L, z, pos = crystal
    nf = (48, 48, 48)
    dm = pw.Domain(tuple(L), (24, 24, 24), nf)
    sp = hgh.hgh_table(z)
    ref = pw.nonlocal_pp(pw.Atom(z, pos[atom]), dm, sp)
    idx, val, wgt = core.hgh_atom_projectors(L, nf, z, pos[atom])
    assert np.array_equal(idx, ref[0].idx)
    assert len(ref) == val.shape[0] == 5
    for q, pp in enumerate(ref):
        assert wgt[q] == pytest.approx(pp.wgt, rel=1e-13)
        # VAL to 1e-12 relative; derivative columns to 1e-10 (analytic vs spline derivative tables)
        s = np.abs(pp.val[:, 0]).max()
        assert np.abs(val[q, :, 0] - pp.val[:, 0]).max() <= 1e-12 * s
        sd = np.abs(pp.val[:, 1:]).max()
        assert np.abs(val[q, :, 1:] - pp.val[:, 1:]).max() <= 1e-10 * sd


def test_pseudocharge_matches_oracle(crystal):
    L, z, pos = crystal
    nf = (48, 48, 48)
    dm = pw.Domain(tuple(L), (24, 24, 24), nf)
    sp = hgh.hgh_table(z)
    ref = np.zeros(dm.ntotFine)
    for p in pos:
        idx, dv = pw.pseudo_charge(pw.Atom(z, p), dm, sp)
        np.add.at(ref, idx, dv[:, 0])
    got = core.hgh_pseudocharge(L, nf, [z] * len(pos), pos)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    q = got.sum() * dm.vol / dm.ntotFine
    assert abs(q - 4.0 * len(pos)) < 0.2
