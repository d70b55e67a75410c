"""The library's small dense FP64 kernels (Cholesky, triangular inverse,
symmetric eigen-decomposition: tridiagonal form up to n = 160, Jacobi beyond;
SolveGenEig) through the C ABI, against torch.linalg
(cuSOLVER, used here only as the comparator) and against their defining
identities: U^T U = A, U Ui = I, A V = V diag(w) with V^T V = I, ascending
w, and the SolveGenEig result C^T B C = I, C^T A C = diag(eig).  Sizes cover
one block, block edges (31, 32, 33), the switch between the tridiagonal and
the Jacobi eigensolvers (160, 161), odd sizes, the LOBPCG Gram width 480, and clustered
(degenerate) spectra.  Tolerances: 1e-12 relative for factorisations and
eigenvalues, 1e-10 for eigenvector residuals."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 7, 31, 32, 33, 100, 160, 161, 480]


def _ctx():
    from pwdft_develop_b200 import Context
    return Context((10.26,) * 3, (12, 12, 12), (24, 24, 24), precision="f64")


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _spd(n, seed, cond=1e3):
    import torch
    g = torch.Generator().manual_seed(seed)
    Q, _ = torch.linalg.qr(torch.randn(n, n, generator=g, dtype=torch.float64))
    d = torch.logspace(0, np.log10(cond), n, dtype=torch.float64)
    return ((Q * d) @ Q.T).cuda()


@pytest.mark.parametrize("n", SIZES)
def test_potrf_and_trtri(n):
    import torch
    from pwdft_develop_b200._lib import check, lib
    c = _ctx()
    # a row-major torch buffer read as a column-major matrix is its transpose
    A = _spd(n, n)                        # symmetric: the same either way
    buf = A.clone()
    check(lib.pw_dense_potrf(c.handle, n, _ptr(buf), n))
    U = torch.triu(buf.T)
    assert float((U.T @ U - A).abs().max() / A.abs().max()) < 1e-12
    ref = torch.linalg.cholesky(A, upper=True)
    assert float((U - ref).abs().max() / ref.abs().max()) < 1e-10
    ubuf = U.T.contiguous()
    uibuf = torch.empty_like(U)
    check(lib.pw_dense_trtri(c.handle, n, _ptr(ubuf), n, _ptr(uibuf), n))
    Ui = uibuf.T
    I = torch.eye(n, dtype=torch.float64, device="cuda")
    assert float((U @ Ui - I).abs().max()) < 1e-10
    if n > 1:
        assert float(torch.tril(Ui, -1).abs().max()) == 0.0
    c.close()


def test_potrf_reports_indefinite():
    import torch
    from pwdft_develop_b200._lib import PW_ENUMERIC, lib
    c = _ctx()
    A = torch.eye(40, dtype=torch.float64, device="cuda")
    A[17, 17] = -1.0
    assert lib.pw_dense_potrf(c.handle, 40, _ptr(A), 40) == PW_ENUMERIC
    c.close()


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("kind", ["random", "clustered"])
def test_syev(n, kind):
    import torch
    from pwdft_develop_b200._lib import check, lib
    c = _ctx()
    g = torch.Generator().manual_seed(100 + n)
    if kind == "random":
        M = torch.randn(n, n, generator=g, dtype=torch.float64)
        A = (M + M.T).cuda()
    else:
        # threefold-degenerate clusters, as in the Rayleigh-Ritz matrices of symmetric cells
        Q, _ = torch.linalg.qr(torch.randn(n, n, generator=g, dtype=torch.float64))
        d = torch.repeat_interleave(torch.linspace(-0.3, 0.6, (n + 2) // 3, dtype=torch.float64), 3)[:n]
        d = d + 1e-12 * torch.randn(n, generator=g, dtype=torch.float64)
        A = ((Q * d) @ Q.T).cuda()
    V = A.clone()
    w = torch.empty(n, dtype=torch.float64, device="cuda")
    sw = C.c_int(0)
    check(lib.pw_dense_syev(c.handle, n, _ptr(V), n, _ptr(w), C.byref(sw)))
    ref = torch.linalg.eigvalsh(A)
    scale = float(A.abs().max())
    assert float((w - ref).abs().max()) < 1e-12 * max(scale, 1.0) * n ** 0.5
    assert bool((w[1:] >= w[:-1]).all())
    # V holds the eigenvectors in its columns (column-major), i.e. the rows of
    # the row-major torch view of the same memory
    E = V                         # E[j] = eigenvector j
    assert float((E @ E.T - torch.eye(n, dtype=torch.float64, device="cuda")).abs().max()) < 1e-10
    R = E @ A - w[:, None] * E
    assert float(R.abs().max()) < 1e-10 * max(scale, 1.0)
    # the tridiagonal path runs (no Jacobi sweeps): one CTA up to n = 160,
    # the cooperative reduction beyond
    assert sw.value == 0
    c.close()


@pytest.mark.parametrize("n", [40, 161, 480, 1440])
@pytest.mark.parametrize("kind", ["identity", "blocks"])
def test_syev_split_tridiagonal(n, kind):
    """Matrices whose tridiagonal form splits into blocks at negligible
    off-diagonals: the identity plus rounding-level noise (LOBPCG / Davidson
    overlap matrices of orthonormal blocks: n 1 x 1 blocks, all eigenvalues
    equal) and a block-diagonal matrix of three decoupled blocks sharing a
    threefold eigenvalue (degenerate across blocks).  Eigenvalues ascending,
    eigenvectors orthonormal and accurate."""
    import torch
    from pwdft_develop_b200._lib import check, lib
    c = _ctx()
    g = torch.Generator().manual_seed(11 * n)
    if kind == "identity":
        E = 1e-17 * torch.randn(n, n, generator=g, dtype=torch.float64)
        A = torch.eye(n, dtype=torch.float64) + E + E.T
    else:
        A = torch.zeros(n, n, dtype=torch.float64)
        sizes = [n // 3, n // 3, n - 2 * (n // 3)]
        o = 0
        for m in sizes:
            Q, _ = torch.linalg.qr(torch.randn(m, m, generator=g, dtype=torch.float64))
            d = torch.linspace(-1.0, 1.0, m, dtype=torch.float64)
            d[m // 2] = 0.25       # the eigenvalue every block shares
            A[o:o + m, o:o + m] = (Q * d) @ Q.T
            o += m
        A = 0.5 * (A + A.T)
        P = torch.randperm(n, generator=g)
        A = A[P][:, P]             # the blocks interleaved: the reduction has to find them
    A = A.cuda()
    V = A.clone()
    w = torch.empty(n, dtype=torch.float64, device="cuda")
    sw = C.c_int(-1)
    check(lib.pw_dense_syev(c.handle, n, _ptr(V), n, _ptr(w), C.byref(sw)))
    ref = torch.linalg.eigvalsh(A)
    assert float((w - ref).abs().max()) < 1e-12 * n ** 0.5
    assert bool((w[1:] >= w[:-1]).all())
    E = V
    assert float((E @ E.T - torch.eye(n, dtype=torch.float64, device="cuda")).abs().max()) < 1e-10
    R = E @ A - w[:, None] * E
    assert float(R.abs().max()) < 1e-10
    c.close()


@pytest.mark.parametrize("n", [161, 480, 1440])
@pytest.mark.parametrize("kind", ["overlap", "ritz"])
def test_syev_large_subspace(n, kind):
    """The cooperative tridiagonal path on the matrices of LOBPCG's 3n
    subspace: an overlap matrix S^T S of normalised, partly dependent columns
    (eigenvalues from ~1e-9 to ~3, dense near 1) and a Ritz matrix with
    threefold-degenerate levels spread like a band structure."""
    import torch
    from pwdft_develop_b200._lib import check, lib
    c = _ctx()
    g = torch.Generator().manual_seed(7 * n)
    if kind == "overlap":
        X = torch.linalg.qr(torch.randn(4 * n, n // 3, generator=g, dtype=torch.float64))[0].T
        W = X[torch.randint(0, n // 3, (n // 3,), generator=g)] + (0.3 / (4 * n) ** 0.5) * torch.randn(
            n // 3, 4 * n, generator=g, dtype=torch.float64)
        P = torch.randn(n - 2 * (n // 3), 4 * n, generator=g, dtype=torch.float64)
        P[0] = X[0] + 1e-5 * P[0]
        S = torch.cat([X, W, P], 0)
        S = S / S.norm(dim=1, keepdim=True)
        A = (S @ S.T).cuda()
    else:
        Q, _ = torch.linalg.qr(torch.randn(n, n, generator=g, dtype=torch.float64))
        d = torch.sort(torch.rand((n + 2) // 3, generator=g, dtype=torch.float64) * 1.8 - 0.3).values
        d = torch.repeat_interleave(d, 3)[:n] + 1e-13 * torch.randn(n, generator=g, dtype=torch.float64)
        A = ((Q * d) @ Q.T).cuda()
        A = 0.5 * (A + A.T)
    V = A.clone()
    w = torch.empty(n, dtype=torch.float64, device="cuda")
    sw = C.c_int(-1)
    check(lib.pw_dense_syev(c.handle, n, _ptr(V), n, _ptr(w), C.byref(sw)))
    assert sw.value == 0
    ref = torch.linalg.eigvalsh(A)
    scale = float(A.abs().max())
    assert float((w - ref).abs().max()) < 1e-12 * max(scale, 1.0) * n ** 0.5
    E = V
    assert float((E @ E.T - torch.eye(n, dtype=torch.float64, device="cuda")).abs().max()) < 1e-10
    R = E @ A - w[:, None] * E
    assert float(R.abs().max()) < 1e-10 * max(scale, 1.0)
    c.close()


@pytest.mark.parametrize("n,width", [(48, 16), (72, 24), (480, 160)])
def test_solve_gen_eig(n, width):
    """SolveGenEig on the [X W P] Gram pair of a LOBPCG step: B = S^T S of a
    block with a nearly dependent column (sigma cut), A = S^T H S."""
    import torch
    from pwdft_develop_b200._lib import check, lib
    c = _ctx()
    g = torch.Generator().manual_seed(n)
    K = 3 * n
    S = torch.randn(K, n, generator=g, dtype=torch.float64)
    S[:, -1] = S[:, 0] + 1e-9 * torch.randn(K, generator=g, dtype=torch.float64)   # dropped by the cut
    H = torch.randn(K, K, generator=g, dtype=torch.float64)
    H = H + H.T
    B = (S.T @ S).cuda()
    A = (S.T @ H @ S).cuda()
    A0, B0 = A.clone(), B.clone()
    eig = np.zeros(width)
    keep = C.c_int(0)
    # column-major on the device: torch's row-major (n, n) of a symmetric matrix is the same
    check(lib.pw_solve_gen_eig(c.handle, n, n, width, _ptr(A), _ptr(B), eig.ctypes.data_as(C.POINTER(C.c_double)),
                               C.byref(keep)))
    nk = keep.value
    assert width <= nk < n
    # C is column-major numCol x numKeep: its columns are the first nk rows of
    # the row-major view of the same memory
    Ct = A[:nk]
    G = Ct @ B0 @ Ct.T
    assert float((G - torch.eye(nk, dtype=torch.float64, device="cuda")).abs().max()) < 1e-8
    D = (Ct @ A0 @ Ct.T).cpu().numpy()
    amax = float(A0.abs().max())
    assert np.abs(D - np.diag(np.diag(D))).max() < 1e-8 * amax
    assert np.abs(np.diag(D)[:width] - eig).max() < 1e-8 * amax
    assert np.all(np.diff(eig) >= 0)
    c.close()


@pytest.mark.parametrize("prec,k,m", [("f64", 160, 160), ("f64", 33, 7), ("f32", 160, 160), ("f32", 480, 160),
                                      ("f32", 13, 5)])
def test_rotate_against_fp64(prec, k, m):
    """Out (+)= X C on the Si64 grid (K = 110,592 rows): FP64 kernel to 1e-13,
    split-BF16 tensor-core GEMM to 3e-5 relative of |X| |C| (the Gram bound),
    overwrite and accumulate."""
    import torch
    from pwdft_develop_b200 import Context
    from pwdft_develop_b200._lib import check, lib
    c = Context((20.52,) * 3, (48, 48, 48), (96, 96, 96), precision=prec)
    c.set_check_errors(True)
    dt = c.torch_dtype
    g = torch.Generator(device="cuda").manual_seed(k * 100 + m)
    X = torch.randn((k, c.ntot), device="cuda", generator=g).to(dt)
    Cm = torch.randn((m, k), dtype=torch.float64, device="cuda", generator=g)   # rows: columns of C (k x m)
    base = torch.randn((m, c.ntot), device="cuda", generator=g).to(dt)
    for acc in (0, 1):
        Out = base.clone()
        check(lib.pw_rotate(c.handle, _ptr(X), c.ntot, k, _ptr(Cm), k, m, _ptr(Out), c.ntot, acc, C.c_void_p(0)))
        torch.cuda.synchronize()
        ref = Cm @ X.double() + (base.double() if acc else 0)
        if prec == "f64":
            assert float((Out - ref).abs().max() / ref.abs().max()) < 1e-13
        else:
            bound = 3e-5 * (Cm.abs() @ X.double().abs())
            assert bool(((Out.double() - ref).abs() <= bound + 1e-6 * ref.abs()).all())
    c.close()
