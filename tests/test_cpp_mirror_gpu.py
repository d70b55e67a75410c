"""The C++ host mirror on the device: MultSpinor and AddTeterPrecond on host
blocks match the FP64 oracle (1e-12 relative) and LOBPCG through the mirror
finds the oracle's lowest eigenvalues (1e-6 Ha)."""
import subprocess

import numpy as np
import pytest

from cpp_mirror import build_demo
from oracle import pw, scf

pytestmark = pytest.mark.gpu


def test_mirror_demo_matches_oracle(tmp_path):
    exe = build_demo(tmp_path / "mirror_demo")
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)
    nc, nf = (16, 16, 16), (32, 32, 32)
    T, _ = pw.build_tables(L, z, pos, nc, nf, seed_v=5)
    T.vtot = 0.3 * (T.vtot - T.vtot.mean())
    nb = 24
    psi = pw.random_orthonormal_psi(T.dm.ntot, nb, 9)
    with open(tmp_path / "in.bin", "wb") as f:
        f.write(np.asarray(L, np.float64).tobytes())
        f.write(np.asarray(nc, np.int32).tobytes())
        f.write(np.asarray(nf, np.int32).tobytes())
        f.write(np.asarray([len(pos), nb], np.int32).tobytes())
        f.write(np.full(len(pos), z, np.int32).tobytes())
        f.write(np.asarray(pos, np.float64).ravel().tobytes())
        f.write(T.vtot.astype(np.float64).tobytes())
        f.write(psi.astype(np.float64).ravel().tobytes())
    subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], check=True, timeout=300)
    out = np.fromfile(tmp_path / "out.bin", dtype=np.float64)
    n = nb * T.dm.ntot
    hpsi, prec, eig = out[:n].reshape(nb, -1), out[n:2 * n].reshape(nb, -1), out[2 * n:]
    ref_h = pw.mult_spinor(T, psi)
    assert np.abs(hpsi - ref_h).max() <= 1e-12 * np.abs(ref_h).max()
    ref_t = pw.add_teter_precond(T, psi)
    assert np.abs(prec - ref_t).max() <= 1e-12 * np.abs(ref_t).max()
    ref_e, _ = scf._eigsh(T, nb, tol=1e-12)
    assert np.abs(eig[:16] - ref_e[:16]).max() < 1e-6
