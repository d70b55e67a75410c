"""Tensor-core split-BF16 Gram GEMM (tcgen05) and FP64 Gram through pw_gram,
against torch FP64 products of the same inputs.  Tolerance for split-BF16
(3 products, FP32 accumulation): |G - G_ref| <= 3e-5 * ||x_i|| ||y_j||."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ctx(prec, n=(24, 24, 24)):
    from pwdft_develop_b200 import Context
    c = Context((10.26,) * 3, n, tuple(2 * x for x in n), precision=prec)
    c.set_check_errors(True)
    return c


@pytest.mark.parametrize("nx,ny", [(24, 24), (72, 72), (160, 160), (33, 7), (5, 130), (256, 96)])
def test_gram_split_bf16(nx, ny):
    import torch
    c = _ctx("f32")
    g = torch.Generator(device="cuda").manual_seed(nx * 1000 + ny)
    X = torch.randn((nx, c.ntot), device="cuda", generator=g)
    Y = torch.randn((ny, c.ntot), device="cuda", generator=g)
    G = c.gram(X, Y)
    ref = X.double() @ Y.double().T
    bound = 3e-5 * X.double().norm(dim=1)[:, None] * Y.double().norm(dim=1)[None, :]
    assert bool(((G - ref).abs() <= bound).all())
    # symmetric case, same buffer
    S = c.gram(X)
    refs = X.double() @ X.double().T
    assert float((S - refs).abs().max() / refs.abs().max()) < 3e-5


def test_gram_si64_grid_f32_and_f64():
    import torch
    for prec, tol in (("f32", 3e-5), ("f64", 1e-13)):
        c = _ctx(prec, (48, 48, 48))
        dt = torch.float32 if prec == "f32" else torch.float64
        g = torch.Generator(device="cuda").manual_seed(3)
        X = torch.randn((160, c.ntot), device="cuda", generator=g).to(dt)
        G = c.gram(X)
        ref = X.double() @ X.double().T
        assert float((G - ref).abs().max() / ref.abs().max()) < tol


def test_gram_empty():
    import torch
    c = _ctx("f32")
    X = torch.zeros((0, c.ntot), device="cuda")
    assert c.gram(X).shape == (0, 0)
