"""Regenerate the Si64 SCF golden fixtures with the FP64 oracle (oracle/scf.py).

Si64: the 2x2x2 diamond supercell (a = 20.52 bohr, seeded +-0.02 bohr
displacements, seed 20261203 + 2, Philox), HGH LDA Teter93, 48^3 / 96^3 grids,
Ecut 20 Ha, 128 occupied + 32 extra bands, 300 K, Anderson mixing (dim 8,
step 0.7), converged to |E_free - E_Harris| / N_atom < 1e-8.  The eigensolver
is scipy's block LOBPCG with the oracle's H*psi applied by a pool of worker
processes (one per host core); the fixed point does not depend on it.

Cases: ``plain`` (the unfiltered operator, as LOBPCG / PPCG / Davidson see it)
and ``filter`` (CheFSI's wavefunction cut-off filter at Ecut, the reference's
default for PW_Solver CheFSI).  Small-cell cases for checking the block path
against the ARPACK goldens: ``si8small`` / ``si8small_filter`` (16^3 / 32^3,
Ecut 5, 16 + 8 bands).  Run from the repository root:
``python tests/golden/make_si64_golden.py [plain|filter|si8small|si8small_filter]``
(about an hour per Si64 case on 8 cores).
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
from oracle import pw, scf  # noqa: E402

_G = {}


def _limit_threads():
    try:
        from threadpoolctl import threadpool_limits
        threadpool_limits(1)
    except ImportError:
        pass


def _apply(rows):
    return pw.mult_spinor(_G["T"], rows)


class PoolHx:
    """Block H*psi over a fork-started pool; the pool is started again when
    the potential changes (the children hold the tables of the fork)."""

    def __init__(self, nproc: int):
        self.nproc = nproc
        self.pool = None
        self.key = None

    def __call__(self, T, rows):
        key = (id(T.vtot), float(T.vtot.sum()), float(T.vtot[::997].sum()))
        if key != self.key:
            self.close()
            _G["T"] = T
            self.pool = mp.get_context("fork").Pool(self.nproc, initializer=_limit_threads)
            self.key = key
        chunks = [c for c in np.array_split(rows, min(len(rows), 2 * self.nproc)) if len(c)]
        return np.concatenate(self.pool.map(_apply, chunks, chunksize=1))

    def close(self):
        if self.pool is not None:
            self.pool.terminate()
            self.pool = None


CASES = {
    "plain": dict(reps=(2, 2, 2), seed=20261203 + 2, nc=(48, 48, 48), ecut=20.0, nocc=128, nextra=32, filt=False,
                  tol=1e-8, name="si64_scf_plain"),
    "filter": dict(reps=(2, 2, 2), seed=20261203 + 2, nc=(48, 48, 48), ecut=20.0, nocc=128, nextra=32, filt=True,
                   tol=1e-8, name="si64_scf_filter"),
    "si8small": dict(reps=(1, 1, 1), seed=20261203 + 1, nc=(16, 16, 16), ecut=5.0, nocc=16, nextra=8, filt=False,
                     tol=1e-9, name="si8_scf_small_lobpcg"),
    "si8small_filter": dict(reps=(1, 1, 1), seed=20261203 + 1, nc=(16, 16, 16), ecut=5.0, nocc=16, nextra=8,
                            filt=True, tol=1e-9, name="si8_scf_small_filter"),
}


def main(which):
    cs = CASES[which]
    L, z, pos = pw.make_crystal("Si", cs["reps"], 10.26, 0.02, cs["seed"])
    nc = cs["nc"]
    nf = tuple(2 * n for n in nc)
    hx = PoolHx(os.cpu_count() or 1)
    scf.set_block_hx(hx, tol=1e-9 if cs["reps"] == (1, 1, 1) else 1e-8)
    t0 = time.time()
    try:
        r = scf.scf(L, z, pos, nc, nf, nocc=cs["nocc"], nextra=cs["nextra"], ecut=cs["ecut"], tol_efree=cs["tol"],
                    verbose=True, max_iter=60, wfn_ecut=cs["ecut"] if cs["filt"] else None)
    finally:
        hx.close()
        scf.set_block_hx(None)
    out = dict(case=which, numGrid=nc, numGridFine=nf, ecut=cs["ecut"], xc="teter93", mix="anderson",
               nocc=cs["nocc"], nextra=cs["nextra"], temperature=300.0, wfn_filter=cs["filt"],
               length=list(map(float, L)), positions=pos.tolist(), znuc=int(z), tol_efree=cs["tol"],
               etot=r.etot, efree=r.efree, eharris=r.eharris, exc=r.exc, ehart=r.ehart, eself=r.eself,
               eig=r.eig.tolist(), occ=r.occ.tolist(), iterations=r.iterations, seconds=time.time() - t0,
               eigensolver="scipy lobpcg over a process-pool H*psi")
    path = Path(__file__).resolve().parent / f"{cs['name']}.json"
    path.write_text(json.dumps(out, indent=1))
    print(path, r.efree, r.iterations, time.time() - t0)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "plain")
