"""Uneven cells applied together (pw_hpsi_batch on forked streams, and the
whole batch captured as one CUDA graph) reproduce each cell's own H*psi bit
for bit; the cells' grids and band counts differ, some are non-cubic."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _build(cells, precs):
    import torch
    from pwdft_develop_b200 import Context
    ctxs, psis, outs = [], [], []
    rng = np.random.default_rng(4)
    for cell, prec in zip(cells, precs):
        c = Context(cell["length"], cell["numGrid"], cell["numGridFine"], precision=prec)
        c.set_atoms([cell["znuc"]] * len(cell["positions"]), cell["positions"])
        c.set_vtot(rng.uniform(-1.0, 0.5, c.ntotFine))
        c.set_band_batch(cell["nband"])
        x = torch.tensor(rng.standard_normal((cell["nband"], c.ntot)) / np.sqrt(c.ntot), dtype=c.torch_dtype,
                         device="cuda")
        ctxs.append(c)
        psis.append(x)
        outs.append(torch.empty_like(x))
    return ctxs, psis, outs


def test_batch_and_graph_match_individual_calls():
    import torch
    from pwdft_develop_b200 import CellBatch
    from pwdft_develop_b200.cells import uneven_cells
    cells = uneven_cells(24)
    # a spread of grids: keep the first cell of each distinct grid, at most 7
    seen, pick = set(), []
    for c in cells:
        if c["numGrid"] not in seen and len(pick) < 7:
            seen.add(c["numGrid"])
            pick.append(c)
    assert any(c["numGrid"][0] != c["numGrid"][1] for c in pick) or len(pick) >= 3
    precs = ["f32" if i % 3 else "f64" for i in range(len(pick))]
    ctxs, psis, outs = _build(pick, precs)
    refs = [c.hpsi(x) for c, x in zip(ctxs, psis)]
    b = CellBatch(ctxs, psis, outs)
    b.hpsi()
    torch.cuda.synchronize()
    for o, r in zip(outs, refs):
        assert torch.equal(o, r)
    for o in outs:
        o.zero_()
    g = b.capture()
    for o in outs:
        o.zero_()
    g.replay()
    torch.cuda.synchronize()
    for o, r in zip(outs, refs):
        assert torch.equal(o, r)
    g.close()


def test_batch_cells_match_oracle():
    """Cells of the uneven batch, applied together, against the FP64 oracle
    (same cell, grid, potential and bands): FP64 1e-12, FP32 1e-5 relative."""
    import torch
    from pwdft_develop_b200 import CellBatch
    from pwdft_develop_b200.cells import uneven_cells

    from oracle import pw
    cells = uneven_cells(48)
    seen, pick = set(), []
    for c in cells:     # one cell of each kind, the smaller grids (oracle cost)
        if c["kind"] not in seen and c["numGrid"][0] <= 40:
            seen.add(c["kind"])
            pick.append(c)
    precs = ["f64" if i % 2 else "f32" for i in range(len(pick))]
    ctxs, psis, outs, refs = [], [], [], []
    from pwdft_develop_b200 import Context
    for i, (cell, prec) in enumerate(zip(pick, precs)):
        T, _ = pw.build_tables(cell["length"], cell["znuc"], cell["positions"], cell["numGrid"],
                               cell["numGridFine"], seed_v=31 + i)
        nb = min(cell["nband"], 10)
        psi = pw.random_orthonormal_psi(T.dm.ntot, nb, 41 + i)
        refs.append(pw.mult_spinor(T, psi))
        c = Context(cell["length"], cell["numGrid"], cell["numGridFine"], precision=prec)
        c.set_atoms([cell["znuc"]] * len(cell["positions"]), cell["positions"])
        c.set_vtot(T.vtot)
        x = torch.tensor(psi, dtype=c.torch_dtype, device="cuda")
        ctxs.append(c)
        psis.append(x)
        outs.append(torch.empty_like(x))
    CellBatch(ctxs, psis, outs).hpsi()
    torch.cuda.synchronize()
    for o, r, prec, cell in zip(outs, refs, precs, pick):
        err = np.abs(o.double().cpu().numpy() - r).max() / np.abs(r).max()
        assert err <= (1e-12 if prec == "f64" else 1e-5), (cell["kind"], cell["numGrid"], prec, err)
    for c in ctxs:
        c.close()
