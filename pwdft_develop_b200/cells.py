"""Seeded batches of independent, uneven cells (Si diamond 8/16/64 atoms, fcc
Al 4/32 atoms) for the batched H*psi path: geometry, cut-off, grid and band
count per cell.  The grid of a cell is the smallest coarse grid built into the
library that resolves sqrt(2 Ecut) L / pi points per direction (at least 20);
one cell in four (seeded) is forced to a larger built grid, up to 60^3, so the
batch spans the 20^3 - 60^3 range."""
from __future__ import annotations

import math

import numpy as np

A_SI = 10.26
A_AL = 7.65
_SI_BASE = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                     [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
_AL_BASE = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]])
# kind -> (element Z, valence electrons per atom, lattice constant, base, repetitions)
KINDS = {
    "Si8": (14, 4, A_SI, _SI_BASE, (1, 1, 1)),
    "Si16": (14, 4, A_SI, _SI_BASE, (2, 1, 1)),
    "Si64": (14, 4, A_SI, _SI_BASE, (2, 2, 2)),
    "Al4": (13, 3, A_AL, _AL_BASE, (1, 1, 1)),
    "Al32": (13, 3, A_AL, _AL_BASE, (2, 2, 2)),
}
CUBIC = (20, 24, 30, 32, 36, 40, 48, 60)
ELONGATED = ((40, 20, 20), (48, 24, 24))


def _grid(L, ecut):
    need = [math.ceil(math.sqrt(2.0 * ecut) * l / math.pi) for l in L]
    if abs(L[0] - 2 * L[1]) < 1e-9 and abs(L[1] - L[2]) < 1e-9:
        for g in ELONGATED:
            if all(g[d] >= need[d] for d in range(3)):
                return g
        return ELONGATED[-1]
    for n in CUBIC:
        if n >= max(need):
            return (n, n, n)
    return (CUBIC[-1],) * 3


def uneven_cells(n: int = 48, seed: int = 20261203 + 3):
    """n cells drawn from the seed: kind uniform over KINDS, Ecut uniform in
    [8, 20] Ha, displacements uniform in [-0.02, 0.02] bohr."""
    rng = np.random.Generator(np.random.Philox(seed))
    kinds = list(KINDS)
    cells = []
    for _ in range(n):
        kind = kinds[int(rng.integers(len(kinds)))]
        z, zval, a, base, reps = KINDS[kind]
        ecut = float(rng.uniform(8.0, 20.0))
        pos = []
        for cz in range(reps[2]):
            for cy in range(reps[1]):
                for cx in range(reps[0]):
                    for f in base:
                        pos.append((np.array([cx, cy, cz]) + f) * a)
        pos = np.array(pos) + rng.uniform(-0.02, 0.02, size=(len(pos), 3))
        L = (a * reps[0], a * reps[1], a * reps[2])
        nc = _grid(L, ecut)
        if rng.random() < 0.25:
            # forced to a larger grid than the cut-off needs
            if nc in ELONGATED:
                nc = ELONGATED[-1]
            else:
                bigger = [g for g in CUBIC if g >= nc[0]]
                g = bigger[int(rng.integers(len(bigger)))]
                nc = (g, g, g)
        nocc = zval * len(pos) // 2
        nband = nocc + max(6, nocc // 4)
        nband += nband % 2
        cells.append({"kind": kind, "znuc": z, "length": L, "positions": pos, "ecut": ecut,
                      "numGrid": nc, "numGridFine": tuple(2 * x for x in nc), "nocc": nocc, "nband": nband})
    return cells
