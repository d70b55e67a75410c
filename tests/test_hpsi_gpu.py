"""GPU parity of the H*psi and Teter kernels against the FP64 oracle, called
through the C ABI.  Tolerances (relative, max-norm over the block):
H*psi <= 1e-12 in FP64 and <= 1e-5 in FP32; Teter the same."""
import numpy as np
import pytest

from oracle import pw

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 1e-5}


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def make_system(nc, reps=(1, 1, 1), a=10.26, seed=20261203 + 1, lengths=None):
    L, z, pos = pw.make_crystal("Si", reps, a, 0.02, seed)
    if lengths is not None:
        L = np.asarray(lengths, dtype=np.float64)
    nf = tuple(2 * n for n in nc)
    T, sp = pw.build_tables(L, z, pos, nc, nf, seed_v=seed + 100)
    return T


def make_ctx(T, prec, band_batch=None, mode="dense"):
    from pwdft_develop_b200 import Context
    c = Context(T.dm.length, T.dm.numGrid, T.dm.numGridFine, precision=prec)
    c.set_nonlocal_mode(mode)
    c.set_vtot(T.vtot)
    c.set_nonlocal([(a[0].idx, np.stack([pp.val[:, 0] for pp in a]), np.array([pp.wgt for pp in a]))
                    for a in T.pseudo])
    if band_batch:
        c.set_band_batch(band_batch)
    return c


@pytest.fixture(scope="module")
def si8():
    return make_system((24, 24, 24))


@pytest.mark.parametrize("mode", ["dense", "realspace"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_hpsi_parity_si8(si8, prec, mode):
    import torch
    T = si8
    psi = pw.random_orthonormal_psi(T.dm.ntot, 24, 5)
    ref = pw.mult_spinor(T, psi)
    c = make_ctx(T, prec, mode=mode)
    x = torch.tensor(psi, dtype=c.torch_dtype, device="cuda")
    y = c.hpsi(x)
    torch.cuda.synchronize()
    got = y.double().cpu().numpy()
    assert _rel(got, ref) <= TOL[prec]


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_teter_parity_si8(si8, prec):
    import torch
    T = si8
    rng = np.random.default_rng(9)
    r = rng.standard_normal((7, T.dm.ntot))
    ref = pw.add_teter_precond(T, r)
    c = make_ctx(T, prec)
    got = c.teter(torch.tensor(r, dtype=c.torch_dtype, device="cuda")).double().cpu().numpy()
    assert _rel(got, ref) <= TOL[prec]


@pytest.mark.parametrize("mode", ["dense", "realspace"])
def test_hpsi_noncubic_grid_f64(mode):
    """(24,16,20) coarse grid in a 10.26 x 7.0 x 8.5 cell."""
    import torch
    T = make_system((24, 16, 20), lengths=(10.26, 7.0, 8.5))
    psi = pw.random_orthonormal_psi(T.dm.ntot, 6, 8)
    ref = pw.mult_spinor(T, psi)
    c = make_ctx(T, "f64", mode=mode)
    got = c.hpsi(torch.tensor(psi, device="cuda")).cpu().numpy()
    assert _rel(got, ref) <= TOL["f64"]


@pytest.mark.parametrize("mode", ["dense", "realspace"])
@pytest.mark.parametrize("nband,batch", [(1, None), (5, None), (7, 2), (9, 4)])
def test_hpsi_odd_bands_and_batches(si8, nband, batch, mode):
    import torch
    T = si8
    psi = pw.random_orthonormal_psi(T.dm.ntot, nband, 11 + nband)
    ref = pw.mult_spinor(T, psi)
    c = make_ctx(T, "f64", band_batch=batch, mode=mode)
    got = c.hpsi(torch.tensor(psi, device="cuda")).cpu().numpy()
    assert _rel(got, ref) <= TOL["f64"]


def test_hpsi_accumulate_and_zero_bands(si8):
    import torch
    T = si8
    psi = pw.random_orthonormal_psi(T.dm.ntot, 4, 21)
    base = np.random.default_rng(2).standard_normal(psi.shape)
    ref = base + pw.mult_spinor(T, psi)
    c = make_ctx(T, "f64")
    out = torch.tensor(base, device="cuda")
    c.hpsi(torch.tensor(psi, device="cuda"), out=out, accumulate=True)
    assert _rel(out.cpu().numpy(), ref) <= TOL["f64"]
    empty = torch.zeros((0, T.dm.ntot), dtype=torch.float64, device="cuda")
    assert c.hpsi(empty).shape == (0, T.dm.ntot)


def test_hpsi_host_entry_matches_device(si8):
    import torch
    T = si8
    psi = pw.random_orthonormal_psi(T.dm.ntot, 6, 31)
    c = make_ctx(T, "f64")
    dev = c.hpsi(torch.tensor(psi, device="cuda")).cpu().numpy()
    host = c.hpsi_host(psi)
    # the projector scatter sums overlapping spheres with shared-memory atomics,
    # so two runs agree to rounding, not bit for bit
    assert _rel(host, dev) <= 1e-14


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_hpsi_host_pinned_chunks_match_device(si8, prec):
    """Page-locked host buffers take the chunked path (copies in and out on
    their own streams around each chunk's H*psi): 101 bands (chunks of 32 and a
    ragged, odd last one), leading dimension > ntot, overwrite and accumulate
    agree with the device entry to rounding; padding columns stay untouched."""
    import ctypes as C
    import torch
    from pwdft_develop_b200._lib import check, lib
    T = si8
    nb, nt = 101, T.dm.ntot
    ld = nt + 8
    c = make_ctx(T, prec)
    dt = torch.float64 if prec == "f64" else torch.float32
    X = torch.tensor(pw.random_orthonormal_psi(nt, nb, 33), dtype=dt)
    dev = c.hpsi(X.cuda()).cpu()
    Xh = torch.zeros((nb, ld), dtype=dt).pin_memory()
    Xh[:, :nt] = X
    for acc in (0, 1):
        Yh = torch.full((nb, ld), 1.0, dtype=dt).pin_memory()
        check(lib.pw_hpsi_host(c.handle, C.c_void_p(Xh.data_ptr()), ld, C.c_void_p(Yh.data_ptr()), ld, nb, acc))
        got = Yh[:, :nt] - (1.0 if acc else 0.0)
        tol = 1e-14 if prec == "f64" else 1e-6
        assert float((got - dev).abs().max() / dev.abs().max()) <= tol
        assert bool((Yh[:, nt:] == 1.0).all())


def test_hpsi_local_only_and_no_projectors(si8):
    import torch
    from pwdft_develop_b200 import Context
    T0 = pw.HamTables(si8.dm, si8.ekin, si8.teter, si8.vtot, [])
    psi = pw.random_orthonormal_psi(T0.dm.ntot, 4, 41)
    ref = pw.mult_spinor(T0, psi)
    c = Context(T0.dm.length, T0.dm.numGrid, T0.dm.numGridFine, "f64")
    c.set_vtot(T0.vtot)
    got = c.hpsi(torch.tensor(psi, device="cuda")).cpu().numpy()
    assert _rel(got, ref) <= TOL["f64"]


def test_hpsi_requires_potential(si8):
    import torch
    from pwdft_develop_b200 import Context, PwError
    c = Context(si8.dm.length, si8.dm.numGrid, si8.dm.numGridFine, "f64")
    with pytest.raises(PwError) as e:
        c.hpsi(torch.zeros((2, si8.dm.ntot), dtype=torch.float64, device="cuda"))
    assert e.value.code == -6


@pytest.fixture(scope="module")
def si64():
    return make_system((48, 48, 48), reps=(2, 2, 2))


@pytest.mark.parametrize("mode", ["dense", "realspace"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_hpsi_parity_si64_subset(si64, prec, mode):
    """Si64 (48^3 / 96^3, 320 projectors): a block of 6 bands vs the oracle."""
    import torch
    T = si64
    psi = pw.random_orthonormal_psi(T.dm.ntot, 6, 51)
    ref = pw.mult_spinor(T, psi)
    c = make_ctx(T, prec, mode=mode)
    got = c.hpsi(torch.tensor(psi, dtype=c.torch_dtype, device="cuda")).double().cpu().numpy()
    assert _rel(got, ref) <= TOL[prec]


def test_hpsi_si64_full_block_properties(si64):
    """160 bands: Hermiticity of psi^T H psi and linearity H(a x + y)."""
    import torch
    T = si64
    c = make_ctx(T, "f64", band_batch=160)
    g = torch.Generator(device="cuda").manual_seed(5)
    X = torch.randn((160, T.dm.ntot), dtype=torch.float64, device="cuda", generator=g)
    HX = c.hpsi(X)
    M = X @ HX.T
    assert float((M - M.T).abs().max() / M.abs().max()) < 1e-12
    Y = torch.randn((160, T.dm.ntot), dtype=torch.float64, device="cuda", generator=g)
    lhs = c.hpsi(2.5 * X + Y)
    rhs = 2.5 * HX + c.hpsi(Y)
    assert float((lhs - rhs).abs().max() / rhs.abs().max()) < 1e-12


@pytest.mark.parametrize("tag", ["c12", "c16"])
@pytest.mark.parametrize("prec,tol", [("f64", 1e-12), ("f32", 1e-5)])
@pytest.mark.parametrize("mode", ["dense", "realspace"])
def test_hpsi_matches_reference_compiled_composition(tag, prec, tol, mode):
    """Device H*psi and Teter against the outputs of the reference's own
    Spinor::AddMultSpinorFineR2C / AddTeterPrecond compiled from its source
    (tests/golden/ref_hpsi.npz): the device builds its projectors from the
    atoms (pw_set_atoms), the reference run used the oracle's restatement of
    CalculateNonlocalPP, so the projector set-up is checked too."""
    from pathlib import Path

    import torch
    from pwdft_develop_b200 import Context
    g = np.load(Path(__file__).resolve().parent / "golden" / "ref_hpsi.npz")
    nc = tuple(int(x) for x in g[f"{tag}_grid"])
    seed_cell, seed_v, seed_psi = (int(x) for x in g[f"{tag}_seeds"])
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, seed_cell)
    T, _ = pw.build_tables(L, z, pos, nc, tuple(2 * n for n in nc), seed_v=seed_v)
    psi = pw.random_orthonormal_psi(T.dm.ntot, int(g[f"{tag}_nband"]), seed_psi)
    c = Context(L, nc, tuple(2 * n for n in nc), precision=prec)
    c.set_nonlocal_mode(mode)
    c.set_atoms([z] * len(pos), pos)
    c.set_vtot(T.vtot)
    x = torch.tensor(psi, dtype=c.torch_dtype, device="cuda")
    h = c.hpsi(x).double().cpu().numpy()
    ref = g[f"{tag}_hpsi"]
    assert np.abs(h - ref).max() / np.abs(ref).max() <= tol
    w = c.teter(x).double().cpu().numpy()
    wr = g[f"{tag}_teter"]
    assert np.abs(w - wr).max() / np.abs(wr).max() <= tol
    c.close()


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_projector_overlap_same_result(prec):
    """The dense projector GEMMs on a second stream beside the FFT chain
    (pw_set_nl_overlap 1) give the same bits as after it for an overwriting
    H*psi, and agree to rounding when accumulating; both against the oracle."""
    import torch
    T = make_system((16, 16, 16))
    c = make_ctx(T, prec)
    psi = pw.random_orthonormal_psi(T.dm.ntot, 7, 31)
    X = torch.tensor(psi, dtype=c.torch_dtype, device="cuda")
    out = {}
    for ov in (0, 1):
        c.set_nl_overlap(ov)
        out[ov] = c.hpsi(X).clone()
        Y = torch.ones_like(X)
        c.hpsi(X, out=Y, accumulate=True)
        out[(ov, "acc")] = Y
    assert torch.equal(out[0], out[1])
    tol = 1e-12 if prec == "f64" else 1e-6
    assert float((out[(0, "acc")] - out[(1, "acc")]).abs().max()) <= tol * float(out[(0, "acc")].abs().max())
    ref = pw.mult_spinor(T, psi)
    got = out[1].double().cpu().numpy()
    assert np.abs(got - ref).max() / np.abs(ref).max() <= (1e-12 if prec == "f64" else 1e-5)
    c.close()
