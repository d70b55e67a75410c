"""The distributed ChebFSI of pwdft_develop_b200.parallel on the device: one
rank whose apply_h is pw_hpsi (FP64) and whose local Gram, rotation and dense
steps run through the library (DeviceOps: pw_gram_rows, pw_rotate_rows,
pw_dense_*) reaches the lowest eigenvalues of the oracle operator (ARPACK,
oracle/scf.py) to 1e-9 Ha.  The multi-rank
transposes and reductions are covered by the two-rank gloo test on the CPU
(tests/test_parallel_cpu.py)."""
import numpy as np
import pytest

from oracle import pw, scf

pytestmark = pytest.mark.gpu


def test_chebfsi_dist_one_rank_on_device():
    import torch
    from pwdft_develop_b200.parallel import chebfsi_dist
    from tests.test_hpsi_gpu import make_ctx, make_system
    T = make_system((16, 16, 16))
    c = make_ctx(T, "f64")
    nband = 24
    X0 = torch.tensor(pw.random_orthonormal_psi(T.dm.ntot, nband, 7), device="cuda")
    lam, Xb, it, res = chebfsi_dist(lambda X: c.hpsi(X.contiguous()), X0, nband, degree=10, max_iter=200,
                                    tol=1e-9, nconv=16, ctx=c)
    ref, _ = scf._eigsh(T, nband, tol=1e-12)
    assert res < 1e-9, (it, res)
    assert np.abs(lam.cpu().numpy()[:16] - ref[:16]).max() < 1e-9
    G = (Xb @ Xb.T).cpu().numpy()
    assert np.abs(G - np.eye(nband)).max() < 1e-10


@pytest.mark.parametrize("prec,tol", [("f64", 1e-12), ("f32", 3e-5)])
def test_row_block_steps_on_device(prec, tol):
    """The local steps of the distributed eigensolver on a row block of the
    grid through the library (one rank: the whole reduction is local): Gram
    over the rows, Cholesky-QR and Rayleigh-Ritz of the row block, against
    torch FP64 on the same data."""
    import torch
    from pwdft_develop_b200 import Context
    from pwdft_develop_b200.parallel import cholqr_rows, gram_row_partitioned, rayleigh_ritz_rows
    c = Context((10.26,) * 3, (24, 24, 24), (48, 48, 48), precision=prec)
    dt = c.torch_dtype
    g = torch.Generator(device="cuda").manual_seed(5)
    nb, nr = 40, 4096                      # a block of 4096 grid rows
    X = torch.randn((nb, nr), device="cuda", generator=g).to(dt)
    Xd = X.double()
    G = gram_row_partitioned(X.T, X.T, ctx=c)
    ref = Xd @ Xd.T
    assert float((G - ref).abs().max() / ref.abs().max()) < tol
    Q = cholqr_rows(X, ctx=c).double()
    assert float((Q @ Q.T - torch.eye(nb, dtype=torch.float64, device="cuda")).abs().max()) < 50 * tol
    H = torch.randn((nr, nr), device="cuda", generator=g, dtype=torch.float64) / nr ** 0.5
    H = H + H.T
    HQ = (Q @ H).to(dt)
    lam, Xr, HXr = rayleigh_ritz_rows(Q.to(dt), HQ, ctx=c)
    A = Q @ H @ Q.T
    assert float((lam - torch.linalg.eigvalsh(0.5 * (A + A.T))).abs().max()) < 100 * tol
    c.close()


def test_scf_dist_one_rank_on_device_matches_golden():
    """The band-distributed SCF driver with its operators on the device
    (DeviceScfOps: pw_hpsi, the raw partial density of pw_density,
    pw_hartree, pw_xc_teter93; the local dense steps through the library) at
    one rank converges to the oracle's Si8 free energy (16^3 / 32^3, Ecut
    5 Ha, LDA) within 1e-6 Ha per atom.  Two ranks: the gloo test on the
    CPU."""
    import json
    from pathlib import Path

    import torch
    from pwdft_develop_b200 import Context
    from pwdft_develop_b200.parallel import DeviceScfOps, scf_dist
    g = json.loads((Path(__file__).resolve().parent / "golden" / "si8_scf_small.json").read_text())
    pos = np.array(g["positions"])
    c = Context(np.array(g["length"]), tuple(g["numGrid"]), tuple(g["numGridFine"]), precision="f64")
    c.set_atoms([g["znuc"]] * len(pos), pos)
    ops = DeviceScfOps(c, g["ecut"], g["znuc"], len(pos))
    nband = g["nocc"] + g["nextra"]
    X0 = torch.tensor(pw.random_orthonormal_psi(c.ntot, nband, 11), device="cuda")
    out, Xb = scf_dist(ops, X0, nband, g["nocc"], tol_efree=1e-8, max_iter=60, degree=10, ctx=c)
    assert out["converged"], out["iterations"]
    assert abs(out["efree"] - g["efree"]) / len(pos) < 1e-6, out["efree"] - g["efree"]
    assert np.abs(out["eig"][:g["nocc"]] - np.array(g["eig"][:g["nocc"]])).max() < 1e-6
    nel = float(out["rho"].sum()) * ops.vol / out["rho"].numel()
    assert abs(nel - 2 * g["nocc"]) < 1e-9
