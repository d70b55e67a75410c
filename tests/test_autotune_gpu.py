"""Autotuner: picks a valid band batch and GEMM tiles, H*psi keeps its FP32
parity against the oracle under the chosen setting, and a second context of
the same shape takes the cached setting without timing runs."""
import numpy as np
import pytest

from oracle import pw

pytestmark = pytest.mark.gpu


def test_autotune_choice_keeps_parity_and_caches():
    import torch
    from pwdft_develop_b200 import Context
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)
    nc, nf = (16, 16, 16), (32, 32, 32)
    T, _ = pw.build_tables(L, z, pos, nc, nf, seed_v=2)
    psi = pw.random_orthonormal_psi(T.dm.ntot, 24, 5)
    ref = pw.mult_spinor(T, psi)
    c = Context(L, nc, nf, precision="f32")
    c.set_atoms([z] * len(pos), pos)
    c.set_vtot(T.vtot)
    r = c.autotune(24)
    assert r["cached"] == 0 and r["tried"] >= 2
    assert 2 <= r["band_batch"] <= 24 and r["ms_best"] <= r["ms_default"]
    assert r["gemm_bn"] in (0, 64, 96, 128, 160, 256) and r["gemm_bn_store"] in (0, 64, 128, 160, 256)
    out = c.hpsi(torch.tensor(psi, dtype=torch.float32, device="cuda")).double().cpu().numpy()
    assert np.abs(out - ref).max() <= 1e-5 * np.abs(ref).max()
    c2 = Context(L, nc, nf, precision="f32")
    c2.set_atoms([z] * len(pos), pos)
    c2.set_vtot(T.vtot)
    r2 = c2.autotune(24)
    assert r2["cached"] == 1 and r2["band_batch"] == r["band_batch"] and r2["gemm_bn"] == r["gemm_bn"]
