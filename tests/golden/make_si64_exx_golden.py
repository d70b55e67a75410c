"""Regenerate the Si64 exchange-energy golden with the FP64 oracle (oracle/exx.py).

The hybrid-exchange configuration: the Si64 cell (2x2x2 diamond, a = 20.52
bohr, 48^3 coarse grid), 160 seeded Gaussian bands orthonormalised by
Cholesky-QR (oracle/pw.py random_orthonormal_psi, seed 20261203 + 4), the
first 128 occupied (occupation 1, numSpin 2), PBE0 (exchange fraction 0.25,
unscreened Coulomb kernel 4 pi / |G|^2, divergence type 1, Ecut 20 Ha).  The
exchange energy E_x = numSpin / 2 sum_j f_j <psi_j | V_x psi_j> needs V_x on the
occupied bands only: 128 x 128 pair products, split over a process pool.
Run from the repository root: ``python tests/golden/make_si64_exx_golden.py``.
"""
import json
import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import exx, pw  # noqa: E402

SEED = 20261203 + 4
NC = (48, 48, 48)
NB, NOCC = 160, 128
_G = {}


def _vx(rows):
    dm, phi, kern, occ = _G["dm"], _G["phi"], _G["kern"], _G["occ"]
    return exx.add_mult_spinor_exx(dm, rows, phi, kern, 0.25, occ)


def main():
    try:
        from threadpoolctl import threadpool_limits
    except ImportError:
        threadpool_limits = None
    L, z, pos = pw.make_crystal("Si", (2, 2, 2), 10.26, 0.02, 20261203 + 2)
    dm = pw.Domain(tuple(L), NC, tuple(2 * n for n in NC))
    t0 = time.time()
    psi = pw.random_orthonormal_psi(dm.ntot, NB, SEED)
    occ = np.zeros(NB)
    occ[:NOCC] = 1.0
    kern, div = exx.exx_kernel_r2c(dm, 20.0, mu=0.0, div_type=1)
    _G.update(dm=dm, phi=exx.set_phi(dm, psi), kern=kern, occ=occ)
    nproc = os.cpu_count() or 1
    chunks = np.array_split(psi[:NOCC], 4 * nproc)
    ctx = mp.get_context("fork")
    with ctx.Pool(nproc, initializer=(lambda: threadpool_limits(1)) if threadpool_limits else None) as pool:
        vx = np.concatenate(pool.map(_vx, chunks, chunksize=1))
    e = exx.exx_energy(vx, psi[:NOCC], occ[:NOCC], numSpin=2)
    out = dict(workload="Si64 48^3, 160 seeded bands (random_orthonormal_psi seed 20261203 + 4), 128 occupied, "
                        "PBE0 fraction 0.25, divergence type 1, Ecut 20 Ha",
               length=list(map(float, L)), numGrid=NC, nband=NB, nocc=NOCC, psi_seed=SEED, exx_fraction=0.25,
               screen_mu=0.0, divergence_type=1, ecut=20.0, exx_div=float(div), exchange_energy=e,
               natom=len(pos), seconds=time.time() - t0)
    path = Path(__file__).resolve().parent / "si64_exx_energy.json"
    path.write_text(json.dumps(out, indent=1))
    print(path, e, time.time() - t0)


if __name__ == "__main__":
    main()
