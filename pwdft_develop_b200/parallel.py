"""Band sharding across ranks (one process per GPU, torch.distributed).

H*psi, the Teter preconditioner and the density are independent per band, so
a rank owns a contiguous block of bands and needs no exchange for them.  The
block sizes follow the reference's band distribution (numStateLocal =
nband / size, the first nband % size ranks one more; src/pwdft/pwdft.cpp:
179-195 and the Alltoall layouts of src/utility.cpp:1159-1197).  The Gram
blocks of the eigensolvers, when the grid is partitioned instead, are summed
over ranks (the reference's MPI_Allreduce after the local GEMM,
src/EigenSolver/lobpcg.cpp:683-687); device time of a step is reduced with
MAX over ranks.
"""
from __future__ import annotations


def band_range(nband: int, world: int, rank: int) -> tuple[int, int]:
    """(first band, number of bands) owned by `rank`."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    base, extra = divmod(nband, world)
    count = base + (1 if rank < extra else 0)
    start = rank * base + min(rank, extra)
    return start, count


def grid_range(ntot: int, world: int, rank: int) -> tuple[int, int]:
    """(first grid point, number of points) of the row partition used for Gram
    blocks: the band_range split in units of 8 points (16-byte rows of the FP32
    tensor-core operands); the last rank takes any remainder."""
    if ntot % 8:
        return band_range(ntot, world, rank)
    s, n = band_range(ntot // 8, world, rank)
    return 8 * s, 8 * n


def allreduce_sum_(t):
    """In-place sum over ranks of a tensor (FP64 Gram / overlap blocks)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t


def max_over_ranks(value: float, device=None) -> float:
    """Largest value of a per-rank scalar (device time of a step)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class DeviceOps:
    """The local steps of the distributed eigensolver on this rank's GPU, all
    through the library: Gram blocks and rotations over a row block of the
    grid (pw_gram_rows / pw_rotate_rows: split-BF16 tensor cores in FP32
    contexts), the upper Cholesky factor, the triangular inverse and the
    symmetric eigen-decomposition (pw_dense_potrf / _trtri / _syev).  Blocks
    are (bands, rows) tensors, i.e. column-major rows x bands matrices."""

    def __init__(self, ctx):
        self.ctx = ctx

    @staticmethod
    def _p(t):
        import ctypes as C
        return C.c_void_p(t.data_ptr())

    def gram(self, Xr, Yr):
        """Xr Yr^T (nx x ny, FP64) over this rank's rows."""
        import torch
        from ._lib import check, lib
        nx, nr = Xr.shape
        ny = Yr.shape[0]
        G = torch.empty((ny, nx), dtype=torch.float64, device=Xr.device)     # column-major nx x ny
        check(lib.pw_gram_rows(self.ctx.handle, nr, self._p(Xr), nr, nx, self._p(Yr), nr, ny, self._p(G), nx, None))
        return G.transpose(0, 1)

    def rotate(self, C, Xr):
        """C^T Xr: rows of X C for the column-major C (k x m, FP64)."""
        import torch
        from ._lib import check, lib
        k, nr = Xr.shape
        m = C.shape[1]
        Cc = C.transpose(0, 1).contiguous()            # column-major k x m
        out = torch.empty((m, nr), dtype=Xr.dtype, device=Xr.device)
        check(lib.pw_rotate_rows(self.ctx.handle, nr, self._p(Xr), nr, k, self._p(Cc), k, m, self._p(out), nr, 0,
                                 None))
        return out

    def cholesky_upper(self, S):
        """U with S = U^T U."""
        import torch
        from ._lib import check, lib
        n = S.shape[0]
        buf = S.contiguous().clone()                   # symmetric: the same in either layout
        check(lib.pw_dense_potrf(self.ctx.handle, n, self._p(buf), n))
        return torch.triu(buf.transpose(0, 1))

    def solve_upper_t(self, U, Xr):
        """U^-T Xr (rows of X U^-1)."""
        import torch
        from ._lib import check, lib
        n = U.shape[0]
        ub = U.transpose(0, 1).contiguous()            # column-major U
        ui = torch.empty_like(ub)
        check(lib.pw_dense_trtri(self.ctx.handle, n, self._p(ub), n, self._p(ui), n))
        return self.rotate(ui.transpose(0, 1), Xr)

    def eigh(self, A):
        """(ascending eigenvalues, column eigenvectors) of a symmetric A."""
        import ctypes as C

        import torch
        from ._lib import check, lib
        n = A.shape[0]
        buf = (0.5 * (A + A.transpose(0, 1))).contiguous()
        w = torch.empty(n, dtype=torch.float64, device=A.device)
        sw = C.c_int(0)
        check(lib.pw_dense_syev(self.ctx.handle, n, self._p(buf), n, self._p(w), C.byref(sw)))
        return w, buf.transpose(0, 1)


class HostOps:
    """The same local steps with torch on the CPU: the form the multi-process
    tests on CPU ranks (gloo) use to check the transposes and reductions."""

    def gram(self, Xr, Yr):
        return Xr @ Yr.transpose(0, 1)

    def rotate(self, C, Xr):
        return C.transpose(0, 1) @ Xr

    def cholesky_upper(self, S):
        import torch
        return torch.linalg.cholesky(0.5 * (S + S.transpose(0, 1)), upper=True)

    def solve_upper_t(self, U, Xr):
        import torch
        return torch.linalg.solve_triangular(U.transpose(0, 1), Xr, upper=False)

    def eigh(self, A):
        import torch
        return torch.linalg.eigh(0.5 * (A + A.transpose(0, 1)))


def local_ops(t, ctx=None):
    """DeviceOps for CUDA tensors (a library context is required: the product
    path has no fallback), HostOps for CPU tensors."""
    if t.is_cuda:
        if ctx is None:
            raise ValueError("device blocks need the rank's library context (ctx) for the local steps")
        return DeviceOps(ctx)
    return HostOps()


def gram_row_partitioned(X_rows, Y_rows, ctx=None):
    """X^T Y for blocks partitioned by grid rows (each rank holds rows of all
    bands; tensors (rows, bands)): local product then a sum over ranks."""
    Xb = X_rows.transpose(0, 1).contiguous()
    Yb = Y_rows.transpose(0, 1).contiguous()
    G = local_ops(Xb, ctx).gram(Xb, Yb)
    return allreduce_sum_(G.contiguous())


# ---------------------------------------------------------------------------
# Distributed eigensolver blocks.  Bands are sharded (band_range) for H*psi,
# which needs no exchange; the subspace steps need sums over the grid, so the
# block is transposed to grid rows (all bands of this rank's rows) with one
# all-to-all, reduced with an all-reduce of the n x n FP64 Gram, and
# transposed back -- the reference's AlltoallForward / AlltoallBackward
# (src/utility.cpp:1159-1197) around the local GEMM and MPI_Allreduce of
# EigenSolver (src/EigenSolver/lobpcg.cpp:683-687, eigensolver.cpp:301-384).
# With one rank (no process group) every collective is the identity.
# ---------------------------------------------------------------------------

def _world():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def band_to_rows(Xb, nband: int):
    """(this rank's bands x all grid points) -> (all bands x this rank's grid rows)."""
    import torch
    import torch.distributed as dist
    world, rank = _world()
    if world == 1:
        return Xb
    ntot = Xb.shape[1]
    bands = [band_range(nband, world, r) for r in range(world)]
    rows = [grid_range(ntot, world, r) for r in range(world)]
    assert Xb.shape[0] == bands[rank][1]
    send = torch.cat([Xb[:, s:s + n].reshape(-1) for s, n in rows])
    nr = rows[rank][1]
    recv = torch.empty(nband * nr, dtype=Xb.dtype, device=Xb.device)
    dist.all_to_all_single(recv, send, output_split_sizes=[b[1] * nr for b in bands],
                           input_split_sizes=[Xb.shape[0] * n for _, n in rows])
    return recv.view(nband, nr)


def rows_to_band(Xr, ntot: int):
    """Inverse of band_to_rows: (all bands x this rank's rows) -> (this rank's bands x all points)."""
    import torch
    import torch.distributed as dist
    world, rank = _world()
    if world == 1:
        return Xr
    nband = Xr.shape[0]
    bands = [band_range(nband, world, r) for r in range(world)]
    rows = [grid_range(ntot, world, r) for r in range(world)]
    nr = rows[rank][1]
    assert Xr.shape[1] == nr
    send = torch.cat([Xr[s:s + n].reshape(-1) for s, n in bands])
    nbm = bands[rank][1]
    recv = torch.empty(nbm * ntot, dtype=Xr.dtype, device=Xr.device)
    dist.all_to_all_single(recv, send, output_split_sizes=[nbm * n for _, n in rows],
                           input_split_sizes=[n * nr for _, n in bands])
    parts, off = [], 0
    for _, n in rows:
        parts.append(recv[off:off + nbm * n].view(nbm, n))
        off += nbm * n
    return torch.cat(parts, 1)


def _bcast_(t):
    import torch.distributed as dist
    if _world()[0] > 1:
        dist.broadcast(t, 0)
    return t


def cholqr_rows(Xr, ctx=None):
    """Cholesky-QR of a row-partitioned block (EigenSolver::Orthogonalize,
    src/EigenSolver/eigensolver.cpp:301-384): S = sum_ranks Xr Xr^T, S = U^T U
    (rank 0, broadcast), X <- X U^-1 (rows: Xr <- U^-T Xr)."""
    ops = local_ops(Xr, ctx)
    S = allreduce_sum_(ops.gram(Xr, Xr).contiguous())
    U = _bcast_(ops.cholesky_upper(S).contiguous())
    return ops.solve_upper_t(U, Xr)


def rayleigh_ritz_rows(Xr, HXr, ctx=None):
    """Rayleigh-Ritz on row-partitioned X and HX: A = sum_ranks Xr HXr^T,
    A = C diag(l) C^T (solved on rank 0 and broadcast, as the reference's
    rank-0 Syevd), X <- X C, HX <- HX C.  Returns (l, Xr, HXr)."""
    ops = local_ops(Xr, ctx)
    A = allreduce_sum_(ops.gram(Xr, HXr).contiguous())
    lam, C = ops.eigh(A)
    lam, C = _bcast_(lam.contiguous()), _bcast_(C.contiguous())
    return lam, ops.rotate(C, Xr), ops.rotate(C, HXr)


def chebyshev_filter(apply_h, X, degree: int, a: float, b: float, a0: float):
    """Scaled Chebyshev filter p_m(H) X damping [a, b] (Zhou, Saad, Tiago,
    Chelikowsky, J. Comput. Phys. 219, 172 (2006)); X: this rank's bands."""
    e = (b - a) / 2.0
    c = (b + a) / 2.0
    sigma = e / (a0 - c)
    sigma1 = sigma
    gamma = 2.0 / sigma1
    Y = (apply_h(X) - c * X) * (sigma1 / e)
    for _ in range(2, degree + 1):
        sigma2 = 1.0 / (gamma - sigma)
        Z = (apply_h(Y) - c * Y) * (2.0 * sigma2 / e) - (sigma * sigma2) * X
        X, Y = Y, Z
        sigma = sigma2
    return Y


def lanczos_upper_bound(apply_h, x0, steps: int = 16) -> float:
    """Upper bound of the spectrum from a k-step Lanczos run on one vector
    (rank 0's first band; the bound is broadcast): largest Ritz value plus
    the last off-diagonal magnitude."""
    import torch
    world, rank = _world()
    out = torch.zeros(1, dtype=torch.float64, device=x0.device)
    if rank == 0:
        v = x0[:1] / torch.linalg.norm(x0[:1])
        vprev = torch.zeros_like(v)
        al, be = [], [0.0]
        for k in range(steps):
            w = apply_h(v)
            a_ = float((w * v).sum())
            w = w - a_ * v - be[-1] * vprev
            b_ = float(torch.linalg.norm(w))
            al.append(a_)
            be.append(b_)
            if b_ == 0.0:
                break
            vprev, v = v, w / b_
        n = len(al)
        T = torch.zeros(n, n, dtype=torch.float64)
        for i in range(n):
            T[i, i] = al[i]
            if i + 1 < n:
                T[i, i + 1] = T[i + 1, i] = be[i + 1]
        out[0] = float(torch.linalg.eigvalsh(T)[-1]) + abs(be[-1])
    return float(_bcast_(out)[0])


def chebfsi_dist(apply_h, Xb, nband: int, degree: int = 10, max_iter: int = 100, tol: float = 1e-9,
                 nconv: int | None = None, ctx=None):
    """Distributed ChebFSI: Chebyshev-filtered subspace iteration over band
    shards (filter and H*psi local to each rank; Cholesky-QR and Rayleigh-Ritz
    on grid rows after an all-to-all transpose).  Xb: this rank's bands
    (band_range(nband, world, rank)) x all grid points, FP64; apply_h maps a
    block of this rank's bands to H times it (pw_hpsi on the rank's GPU).
    Returns (eigenvalues, Xb, iterations, max residual) with residuals
    ||H x - l x|| / max(1, |l|) of the lowest nconv (default all) pairs,
    gathered over ranks.  ctx: the rank's library context, required for
    device blocks (the local Gram, rotation and dense steps run through it)."""
    import torch
    world, rank = _world()
    ntot = Xb.shape[1]
    b_up = lanczos_upper_bound(apply_h, Xb)
    s, n = band_range(nband, world, rank)
    # first pass: orthonormalise and Rayleigh-Ritz the start block
    Xr = cholqr_rows(band_to_rows(Xb, nband), ctx)
    Xb = rows_to_band(Xr, ntot)
    lam, Xr, HXr = rayleigh_ritz_rows(Xr, band_to_rows(apply_h(Xb), nband), ctx)
    Xb = rows_to_band(Xr, ntot)
    res_max = float("inf")
    it = 0
    for it in range(1, max_iter + 1):
        Y = chebyshev_filter(apply_h, Xb, degree, float(lam[-1]), b_up, float(lam[0]))
        Yr = cholqr_rows(band_to_rows(Y, nband), ctx)
        Yb = rows_to_band(Yr, ntot)
        lam, Xr, HXr = rayleigh_ritz_rows(Yr, band_to_rows(apply_h(Yb), nband), ctx)
        Xb = rows_to_band(Xr, ntot)
        HXb = rows_to_band(HXr, ntot)
        loc = torch.linalg.norm(HXb - lam[s:s + n, None] * Xb, dim=1) / torch.clamp(lam[s:s + n].abs(), min=1.0)
        res = torch.zeros(nband, dtype=torch.float64, device=Xb.device)
        res[s:s + n] = loc
        res_max = float(allreduce_sum_(res)[:nconv or nband].max())
        if res_max < tol:
            break
    return lam, Xb, it, res_max


def gather_bands(Xb, nband: int):
    """All bands on every rank from the band shards (band_range order):
    (nband x ntot).  The exact-exchange orbitals are needed whole by every
    rank; the reference passes them round the ranks with MPI_Bcast
    (src/SCF/spinor.cpp:722-776), here one all-gather."""
    import torch
    import torch.distributed as dist
    world, rank = _world()
    if world == 1:
        return Xb
    ntot = Xb.shape[1]
    bands = [band_range(nband, world, r) for r in range(world)]
    nmax = max(n for _, n in bands)
    buf = torch.zeros((nmax, ntot), dtype=Xb.dtype, device=Xb.device)
    buf[:Xb.shape[0]] = Xb
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    return torch.cat([parts[r][:n] for r, (_, n) in enumerate(bands)], 0)


def exx_apply_dist(set_phi, apply_exx, Xb, occ, nband: int):
    """V_x of this rank's bands with the exchange orbitals of all ranks:
    set_phi(all bands, occ) then apply_exx(this rank's bands) -- on a GPU,
    Context.exx_set_phi and Context.exx_apply."""
    set_phi(gather_bands(Xb, nband), occ)
    return apply_exx(Xb)


# ---------------------------------------------------------------------------
# Distributed SCF (SCF::Iterate over band shards)
# ---------------------------------------------------------------------------
AU2K = 315774.67


def _wgauss(ev, ef, tbeta, smearing):
    import numpy as np
    x = np.clip(tbeta * (ef - ev), -700.0, 700.0)
    if smearing == "GB":
        from scipy.special import erfc
        return 0.5 * erfc(-x)
    return 1.0 / (1.0 + np.exp(-x))


def fermi_occupations(eig, nocc: int, tbeta: float, smearing: str = "FD"):
    """Occupation rates and Fermi level by bisection on the electron count
    (SCF::CalculateOccupationRate, src/SCF/scf.cpp:1780-1822) with wgauss
    (src/utility.cpp:4404-4420): smearing "FD" (Fermi-Dirac) or "GB"
    (Gaussian); eig: all bands, ascending.  numpy arrays."""
    import numpy as np
    ev = np.asarray(eig, dtype=np.float64)
    if ev.size == nocc:
        return np.ones(ev.size), float(ev[-1])
    lb, ub = float(ev.min()), float(ev.max())
    ef = 0.5 * (lb + ub)
    for _ in range(200):
        s = _wgauss(ev, ef, tbeta, smearing).sum()
        if abs(s - nocc) <= 1e-16:
            break
        if s < nocc:
            lb = ef
        else:
            ub = ef
        ef = 0.5 * (lb + ub)
    return _wgauss(ev, ef, tbeta, smearing), ef


def fermi_entropy(eig, ef: float, tbeta: float, smearing: str = "FD"):
    """Per-band -T S term of the free energy (getEntropy, src/utility.cpp:
    4422-4444; scf.cpp:1960-1984), numpy."""
    import numpy as np
    x = tbeta * (ef - np.asarray(eig, dtype=np.float64))
    if smearing == "GB":
        return -0.5 / tbeta * np.exp(-np.minimum(200.0, x * x)) / np.sqrt(np.pi)
    out = np.zeros_like(x)
    m = np.abs(x) <= 36.0
    f = 1.0 / (1.0 + np.exp(-x[m]))
    with np.errstate(divide="ignore", invalid="ignore"):
        out[m] = np.nan_to_num((f * np.log(f) + (1.0 - f) * np.log(1.0 - f)) / tbeta)
    return out


class AndersonMixer:
    """Anderson mixing of the potential (SCF::AndersonMix, src/SCF/scf.cpp:
    2299-2365): history of inputs and residuals, least-squares coefficients,
    the mixed input plus step times the mixed residual.  Every rank runs it on
    the same data (the potential is replicated), as the reference does."""

    def __init__(self, mix_dim: int = 8, step: float = 0.7):
        self.dim, self.step = mix_dim, step
        self.dv, self.df = [], []

    def __call__(self, vin, vout):
        import torch
        F = vout - vin
        if self.dv:
            difv = torch.stack([h - vin for h in self.dv], 1)
            diff = torch.stack([h - F for h in self.df], 1)
            theta = torch.linalg.solve(diff.T @ diff, diff.T @ F)
            xbar, fbar = vin - difv @ theta, F - diff @ theta
        else:
            xbar, fbar = vin, F
        self.dv.append(vin.clone())
        self.df.append(F.clone())
        if len(self.dv) > self.dim:
            self.dv.pop(0)
            self.df.pop(0)
        return xbar + self.step * fbar


def scf_dist(ops, Xb, nband: int, nocc: int, tol_efree: float = 1e-6, max_iter: int = 60, degree: int = 10,
             first_cycles: int = 5, mix_dim: int = 8, mix_step: float = 0.7, temperature: float = 300.0,
             ctx=None, verbose: bool = False, smearing: str = "FD"):
    """SCF::Iterate (src/SCF/scf.cpp:372-591) over band shards: each rank
    filters and holds its bands (band_range), the subspace steps run on grid
    rows (chebfsi_dist's Cholesky-QR and Rayleigh-Ritz), the density is the
    all-reduced sum of the ranks' partial densities, normalised once to
    2 nocc electrons (hamiltonian.cpp:2455-2600 with the reference's
    MPI_Allreduce), and the potentials, energies and Anderson mixing run on
    every rank on the same replicated data.  Converges when
    |E_free - E_Harris| / N_atom < tol_efree (efreeDifPerAtom, scf.cpp:464-471).

    ops: the rank's operators --
      set_vtot(vtot)          the local potential (fine grid, FP64 tensor)
      apply_h(Xb)             H times a block of this rank's bands
      density_raw(Xb, w)      sum_k w_k |psi_k,fine|^2 over this rank's bands
      potentials(rho)         (vh, vxc, eps): Hartree of rho - rho_ps and XC
      rho_ps, vol, natom, eself
    Xb: this rank's start bands (band_range(nband, world, rank) x all grid
    points).  Returns a dict (efree, etot, eharris, eig, occ, iterations,
    converged, rho, vtot) and the final bands of this rank."""
    import numpy as np
    import torch
    world, rank = _world()
    s, n = band_range(nband, world, rank)
    ntot = Xb.shape[1]
    rho_ps = ops.rho_ps
    nf = rho_ps.numel()
    w = ops.vol / nf
    tbeta = AU2K / temperature
    # initial density from the pseudocharge (scf.cpp:232-255)
    rho = torch.where(rho_ps > 1e-6, rho_ps, torch.full_like(rho_ps, 1e-6))
    rho = rho * (rho_ps.sum() / rho.sum())
    vh, vxc, eps = ops.potentials(rho)
    exc = float((eps * rho).sum()) * w
    vtot = vh + vxc
    mixer = AndersonMixer(mix_dim, mix_step)
    b_up = None
    lam = None
    out = dict(converged=False)
    for it in range(1, max_iter + 1):
        ops.set_vtot(vtot)
        if b_up is None:
            b_up = lanczos_upper_bound(ops.apply_h, Xb)
            Xr = cholqr_rows(band_to_rows(Xb, nband), ctx)
            Xb = rows_to_band(Xr, ntot)
            lam, Xr, _ = rayleigh_ritz_rows(Xr, band_to_rows(ops.apply_h(Xb), nband), ctx)
            Xb = rows_to_band(Xr, ntot)
            cycles = max(1, first_cycles)
        else:
            cycles = 1
        for _ in range(cycles):
            Y = chebyshev_filter(ops.apply_h, Xb, degree, float(lam[-1]), b_up, float(lam[0]))
            Yr = cholqr_rows(band_to_rows(Y, nband), ctx)
            Yb = rows_to_band(Yr, ntot)
            lam, Xr, _ = rayleigh_ritz_rows(Yr, band_to_rows(ops.apply_h(Yb), nband), ctx)
            Xb = rows_to_band(Xr, ntot)
        eig = lam.double().cpu().numpy()
        occ, ef = fermi_occupations(eig, nocc, tbeta, smearing)
        ent = float(np.sum(2.0 * fermi_entropy(eig, ef, tbeta, smearing)))
        ekin = float(np.sum(2.0 * eig * occ))
        # Harris energy with the input density and potentials (scf.cpp:1987-2140)
        ehart_h = float((0.5 * vh * (rho + rho_ps)).sum()) * w
        evxc = float((vxc * rho).sum()) * w
        eharris = ekin + (exc - evxc) - ehart_h - ops.eself + ent
        # new density: partial sums over the ranks' bands, then one normalisation
        part = ops.density_raw(Xb, torch.as_tensor(2.0 * occ[s:s + n], dtype=torch.float64))
        rho_out = allreduce_sum_(part.double().contiguous())
        rho_out = rho_out * (2.0 * nocc * nf / (ops.vol * float(rho_out.sum())))
        vh, vxc, eps = ops.potentials(rho_out)
        exc = float((eps * rho_out).sum()) * w
        vtot_new = vh + vxc
        # Kohn-Sham energy with the input potential (scf.cpp:1834-1984)
        ecor = -float((vtot * rho_out).sum()) * w + exc + float((0.5 * vh * (rho_out - rho_ps)).sum()) * w \
            - ops.eself
        etot = ekin + ecor
        efree = etot + ent
        dif = abs(efree - eharris) / ops.natom
        if verbose and rank == 0:
            print(f"scf_dist {it:3d} Efree {efree:.10f} Eharris {eharris:.10f} dif {dif:.3e}")
        out = dict(efree=efree, etot=etot, eharris=eharris, eig=eig, occ=occ, iterations=it, converged=False,
                   rho=rho_out, vtot=vtot)
        rho = rho_out
        if dif < tol_efree:
            out["converged"] = True
            break
        vtot = mixer(vtot, vtot_new)
    return out, Xb


class DeviceScfOps:
    """scf_dist's operators on this rank's GPU through the library: an FP64
    context with its atoms set (pw_set_atoms); H*psi pw_hpsi, the partial
    density pw_density without renormalisation, pw_hartree and pw_xc_teter93
    (LDA) on the fine grid."""

    def __init__(self, ctx, ecut: float, znuc, natom: int):
        import numpy as np
        import torch
        from .core import hgh_species
        self.ctx, self.ecut = ctx, float(ecut)
        dev = torch.device("cuda", ctx.device)
        self.rho_ps = torch.as_tensor(ctx.pseudocharge(), dtype=torch.float64, device=dev)
        L = np.asarray(ctx.length, dtype=np.float64)
        self.vol = float(L.prod())
        zs = np.broadcast_to(np.asarray(znuc), (natom,))
        self.natom = natom
        self.eself = float(sum(hgh_species(int(z))["eself"] for z in zs))

    def set_vtot(self, vtot):
        self.ctx.set_vtot(vtot.double().cpu().numpy())

    def apply_h(self, Xb):
        return self.ctx.hpsi(Xb)

    def density_raw(self, Xb, w):
        import numpy as np
        # pw_density takes occupation rates (it doubles them); nocc_total 0: no renormalisation
        return self.ctx.density(Xb, np.asarray(w.cpu().numpy()) / 2.0, 0)

    def potentials(self, rho):
        vh = self.ctx.hartree((rho - self.rho_ps).contiguous(), self.ecut)
        eps, vxc = self.ctx.xc(rho.contiguous())
        return vh, vxc, eps
