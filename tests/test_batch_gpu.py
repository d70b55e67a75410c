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
