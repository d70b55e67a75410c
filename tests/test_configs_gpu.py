"""H*psi, Teter and Gram parity at the sizes of the benchmark configurations
that the smaller parity tests do not reach.

* every coarse grid built into the library besides the Si8 / Si64 ones, with
  the cells the uneven-cell batch draws them for (fcc Al 4 / 32 atoms, Si8,
  the elongated Si16 cell), against the FP64 oracle: FP64 1e-12 and FP32 1e-5
  relative (the H*psi parity bars); the 20^3 .. 60^3 range of the batched
  configuration, radix-3 and radix-5 FFT lengths included;
* the Si216 adjoint configuration (72^3 / 144^3, 216 atoms) on a 4-band block;
* the split-BF16 Gram at the LOBPCG block widths of Si64 (480 columns,
  K = 110,592) and Si216 (1440 columns, K = 373,248), against FP64 products,
  bound 3e-5 ||x_i|| ||x_j|| as in the small Gram tests.
"""
import numpy as np
import pytest

from oracle import pw

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 1e-5}

# (element, repetitions, lattice constant, coarse grid)
CELLS = [
    ("Al", (1, 1, 1), 7.65, (20, 20, 20)),
    ("Al", (1, 1, 1), 7.65, (30, 30, 30)),
    ("Al", (2, 2, 2), 7.65, (32, 32, 32)),
    ("Al", (2, 2, 2), 7.65, (36, 36, 36)),
    ("Si", (1, 1, 1), 10.26, (40, 40, 40)),
    ("Si", (2, 1, 1), 10.26, (40, 20, 20)),
    ("Si", (2, 1, 1), 10.26, (48, 24, 24)),
    ("Al", (2, 2, 2), 7.65, (60, 60, 60)),
    ("Si", (1, 1, 1), 10.26, (12, 12, 12)),
    ("Si", (1, 1, 1), 10.26, (24, 16, 20)),
]


def _check(kind, reps, a, nc, nb, seed, precs=("f64", "f32")):
    import torch
    from pwdft_develop_b200 import Context
    L, z, pos = pw.make_crystal(kind, reps, a, 0.02, seed)
    nf = tuple(2 * n for n in nc)
    T, _ = pw.build_tables(L, z, pos, nc, nf, seed_v=seed + 1)
    psi = pw.random_orthonormal_psi(T.dm.ntot, nb, seed + 2)
    ref = pw.mult_spinor(T, psi)
    tref = pw.add_teter_precond(T, psi)
    for prec in precs:
        c = Context(L, nc, nf, precision=prec)
        c.set_vtot(T.vtot)
        c.set_atoms([z] * len(pos), pos)
        x = torch.tensor(psi, dtype=c.torch_dtype, device="cuda")
        got = c.hpsi(x).double().cpu().numpy()
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err <= TOL[prec], (kind, nc, prec, "hpsi", err)
        w = c.teter(x).double().cpu().numpy()
        err = np.abs(w - tref).max() / np.abs(tref).max()
        assert err <= TOL[prec], (kind, nc, prec, "teter", err)
        c.close()


@pytest.mark.parametrize("kind,reps,a,nc", CELLS, ids=[f"{c[0]}{np.prod(c[1]) * (8 if c[0] == 'Si' else 4)}-"
                                                       f"{'x'.join(map(str, c[3]))}" for c in CELLS])
def test_hpsi_grid_matches_oracle(kind, reps, a, nc):
    # an odd band count exercises the unpaired last band of the band-pair pipeline
    _check(kind, reps, a, nc, 7, 20261203 + sum(nc))


def test_hpsi_si216_block_matches_oracle():
    _check("Si", (3, 3, 3), 10.26, (72, 72, 72), 4, 20261203 + 5)


@pytest.mark.parametrize("n,K", [(480, 48 ** 3), (1440, 72 ** 3)])
def test_gram_at_lobpcg_widths(n, K):
    import torch
    from pwdft_develop_b200 import Context
    g = int(round(K ** (1.0 / 3.0)))
    c = Context((10.26,) * 3, (g, g, g), (2 * g,) * 3, precision="f32")
    c.set_check_errors(True)
    gen = torch.Generator(device="cuda").manual_seed(n)
    X = torch.randn((n, c.ntot), device="cuda", generator=gen)
    S = c.gram(X)
    Xd = X.double()
    ref = Xd @ Xd.T
    nrm = Xd.norm(dim=1)
    bound = 3e-5 * nrm[:, None] * nrm[None, :]
    assert bool(((S - ref).abs() <= bound).all()), float(((S - ref).abs() / bound).max())
    # a rectangular block X^T Y of the [X W P] Gram shape
    Y = X[: n // 3].contiguous()
    G = c.gram(X, Y)
    assert bool(((G - ref[:, : n // 3]).abs() <= bound[:, : n // 3]).all())
    c.close()


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("kind,reps,a,nc", [("Si", (1, 1, 1), 10.26, (24, 24, 24)), ("Si", (2, 2, 2), 10.26, (48, 48, 48)),
                                            ("Al", (2, 2, 2), 7.65, (60, 60, 60)), ("Si", (2, 1, 1), 10.26, (48, 24, 24)),
                                            ("Si", (3, 3, 3), 10.26, (72, 72, 72))])
def test_hpsi_second_fft_decomposition_matches_oracle(kind, reps, a, nc, variant):
    """The fused fine-plane kernel in the autotuner's non-default forms (the
    default, variant 2, runs in every other test) against the oracle: the
    inter-stage twiddles read from shared-memory tables (variant 0) and the
    second radix decomposition (variant 1: 48 = 8 x 6, 96 = 12 x 8,
    120 = 12 x 10, 144 = 16 x 9); FP64 1e-12, FP32 1e-5."""
    import torch
    from pwdft_develop_b200 import Context
    L, z, pos = pw.make_crystal(kind, reps, a, 0.02, 77)
    nf = tuple(2 * n for n in nc)
    T, _ = pw.build_tables(L, z, pos, nc, nf, seed_v=78)
    psi = pw.random_orthonormal_psi(T.dm.ntot, 3, 79)
    ref = pw.mult_spinor(T, psi)
    for prec in ("f64", "f32"):
        c = Context(L, nc, nf, precision=prec)
        c.set_vtot(T.vtot)
        c.set_atoms([z] * len(pos), pos)
        c.set_fft_variant(variant)
        got = c.hpsi(torch.tensor(psi, dtype=c.torch_dtype, device="cuda")).double().cpu().numpy()
        assert np.abs(got - ref).max() / np.abs(ref).max() <= TOL[prec], (nc, prec)
        c.close()
