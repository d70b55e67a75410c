"""Regenerate the SCF golden fixtures with the FP64 oracle (oracle/scf.py).

Si8 diamond (a = 10.26 bohr, seeded +-0.02 bohr displacements, seed
20261203 + 1), HGH LDA, 16 occupied + 8 extra bands, 300 K, Anderson mixing
(dim 8, step 0.7), converged to |E_free - E_Harris| / N_atom < 1e-9.
Cases: 16^3 / 32^3 grids with Ecut 5 Ha, and the 24^3 / 48^3 grids with
Ecut 10 Ha (LDA Teter93); ``pbe``: the small case with PBE (the reference's
internal PBE path); ``broyden``: the small case with Broyden potential mixing;
``hse06``: the small case with the nested HSE06 hybrid scheme (PBE SCF, then
phi iterations with ACE until dExx < 1e-8); ``al4_gb``: an fcc Al4 metal with
Gaussian smearing at 3000 K (al4_scf_gb.json).  Run from the repository root:
``python tests/golden/make_scf_golden.py [small|full|pbe|broyden|hse06|al4_gb]``.
"""
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import pw, scf  # noqa: E402

CASES = {"small": ((16, 16, 16), (32, 32, 32), 5.0, "teter93"), "full": ((24, 24, 24), (48, 48, 48), 10.0, "teter93"),
         "al4_gb": ((16, 16, 16), (32, 32, 32), 5.0, "teter93"),
         "pbe": ((16, 16, 16), (32, 32, 32), 5.0, "pbe"), "broyden": ((16, 16, 16), (32, 32, 32), 5.0, "teter93"),
         "hse06": ((16, 16, 16), (32, 32, 32), 5.0, "hse06")}


def main(which):
    if which == "al4_gb":
        return al4_gb()
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)
    nc, nf, ecut, xc = CASES[which]
    t0 = time.time()
    mix = "broyden" if which == "broyden" else "anderson"
    # Broyden's mixed potential keeps only the density-sphere components, so its
    # |E_free - E_Harris| has a floor; it converges on the density change (scfNorm)
    tol_rho = 1e-13 if mix == "broyden" else None
    r = scf.scf(L, z, pos, nc, nf, nocc=16, nextra=8, ecut=ecut, tol_efree=1e-9, verbose=True, xc=xc, mix=mix,
                max_iter=80, tol_rho=tol_rho, phi_max_iter=20, phi_tol=1e-8)
    out = dict(case=which, numGrid=nc, numGridFine=nf, ecut=ecut, xc=xc, mix=mix, nocc=16, nextra=8,
               temperature=300.0,
               length=list(map(float, L)), positions=pos.tolist(), znuc=int(z),
               tol_rho=tol_rho, scf_norm=r.history[-1]["scf_norm"],
               etot=r.etot, efree=r.efree, eharris=r.eharris, exc=r.exc, ehart=r.ehart, eself=r.eself,
               eig=r.eig.tolist(), occ=r.occ.tolist(), iterations=r.iterations, seconds=time.time() - t0)
    if xc == "hse06":
        out.update(efock=r.efock, dexx=r.dexx, phi_iterations=r.phi_iterations, phi_tol=1e-8,
                   converged=bool(r.converged))
    path = Path(__file__).resolve().parent / f"si8_scf_{which}.json"
    path.write_text(json.dumps(out, indent=1))
    print(path, r.efree, r.iterations)


def al4_gb():
    """fcc Al4 (a = 7.65 bohr, seeded +-0.02 bohr displacements, seed
    20261203 + 3), HGH LDA, 16^3 / 32^3, Ecut 5 Ha, 6 occupied + 4 extra
    bands, Gaussian smearing (Smearing_Scheme GB) at 3000 K: a metal whose
    threefold level at the Fermi energy is two-thirds occupied."""
    L, z, pos = pw.make_crystal("Al", (1, 1, 1), 7.65, 0.02, 20261203 + 3)
    nc, nf, ecut, xc = CASES["al4_gb"]
    t0 = time.time()
    r = scf.scf(L, z, pos, nc, nf, nocc=6, nextra=4, ecut=ecut, temperature=3000.0, tol_efree=1e-9, verbose=True,
                max_iter=80, smearing="GB")
    out = dict(case="al4_gb", numGrid=nc, numGridFine=nf, ecut=ecut, xc=xc, mix="anderson", nocc=6, nextra=4,
               temperature=3000.0, smearing="GB", length=list(map(float, L)), positions=pos.tolist(), znuc=int(z),
               etot=r.etot, efree=r.efree, eharris=r.eharris, exc=r.exc, ehart=r.ehart, eself=r.eself,
               eig=r.eig.tolist(), occ=r.occ.tolist(), iterations=r.iterations, seconds=time.time() - t0)
    path = Path(__file__).resolve().parent / "al4_scf_gb.json"
    path.write_text(json.dumps(out, indent=1))
    print(path, r.efree, r.iterations)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "small")
