"""The distributed ChebFSI of pwdft_develop_b200.parallel on the device: one
rank whose apply_h is pw_hpsi (FP64) reaches the lowest eigenvalues of the
oracle operator (ARPACK, oracle/scf.py) to 1e-9 Ha.  The multi-rank
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
                                    tol=1e-9, nconv=16)
    ref, _ = scf._eigsh(T, nband, tol=1e-12)
    assert res < 1e-9, (it, res)
    assert np.abs(lam.cpu().numpy()[:16] - ref[:16]).max() < 1e-9
    G = (Xb @ Xb.T).cpu().numpy()
    assert np.abs(G - np.eye(nband)).max() < 1e-10
