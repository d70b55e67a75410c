"""Band sharding and the rank reductions with two gloo ranks on the CPU:
every band owned exactly once with the reference's block sizes, the
row-partitioned Gram summed over ranks equals the full product, and the step
time reduction takes the maximum."""
import os
import socket

import numpy as np
import pytest

from pwdft_develop_b200.parallel import band_range


def test_band_range_covers_once():
    for nband in (1, 7, 24, 160, 480):
        for world in (1, 2, 3, 4, 8):
            seen = []
            for r in range(world):
                s, n = band_range(nband, world, r)
                seen.extend(range(s, s + n))
            assert seen == list(range(nband))
            sizes = [band_range(nband, world, r)[1] for r in range(world)]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    with pytest.raises(ValueError):
        band_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from pwdft_develop_b200.parallel import grid_range, gram_row_partitioned, max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(0)
    X = torch.tensor(rng.standard_normal((1000, 12)))
    Y = torch.tensor(rng.standard_normal((1000, 12)))
    s, n = grid_range(1000, world, rank)
    G = gram_row_partitioned(X[s:s + n], Y[s:s + n])
    t = max_over_ranks(1.0 + rank)
    if rank == 0:
        q.put((G.numpy(), (X.T @ Y).numpy(), t))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_two_ranks_gram_and_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    G, ref, t = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert np.abs(G - ref).max() <= 1e-12 * np.abs(ref).max()
    assert t == 2.0


def _eig_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from oracle import pw
    from pwdft_develop_b200.parallel import band_range, band_to_rows, chebfsi_dist, rows_to_band
    if world > 1:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
    T, _ = pw.build_tables(*_si8(), (12, 12, 12), (24, 24, 24), seed_v=4)
    nband = 20
    X0 = torch.tensor(pw.random_orthonormal_psi(T.dm.ntot, nband, 7))
    s, n = band_range(nband, world, rank)
    # the transposes are inverse to each other and lay out all bands of a row block
    Xr = band_to_rows(X0[s:s + n].clone(), nband)
    assert torch.equal(rows_to_band(Xr, T.dm.ntot), X0[s:s + n])

    def apply_h(X):
        return torch.from_numpy(pw.mult_spinor(T, X.numpy()))

    lam, Xb, it, res = chebfsi_dist(apply_h, X0[s:s + n].clone(), nband, degree=10, max_iter=200, tol=1e-9,
                                    nconv=14)
    if rank == 0:
        q.put((lam.numpy(), it, res))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _si8():
    from oracle import pw
    L, z, pos = pw.make_crystal("Si", (1, 1, 1), 10.26, 0.02, 20261203 + 1)
    return L, z, pos


def test_distributed_chebfsi_two_ranks_matches_one_rank_and_arpack():
    """ChebFSI over two gloo ranks (band shards, all-to-all transposes,
    all-reduced Gram and Rayleigh-Ritz) reaches the same lowest eigenvalues as
    one rank and as ARPACK on the oracle operator (1e-9 Ha)."""
    import torch.multiprocessing as mp
    from oracle import pw, scf
    ctx = mp.get_context("spawn")
    out = {}
    for world in (1, 2):
        q = ctx.Queue()
        port = _free_port()
        procs = [ctx.Process(target=_eig_worker, args=(r, world, port, q)) for r in range(world)]
        for p in procs:
            p.start()
        out[world] = q.get(timeout=600)
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
    T, _ = pw.build_tables(*_si8(), (12, 12, 12), (24, 24, 24), seed_v=4)
    ref, _ = scf._eigsh(T, 20, tol=1e-12)
    for world in (1, 2):
        lam, it, res = out[world]
        assert res < 1e-9, (world, it, res)
        assert np.abs(lam[:14] - ref[:14]).max() < 1e-9, (world, lam[:14] - ref[:14])


def _exx_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from oracle import exx, pw
    from pwdft_develop_b200.parallel import band_range, exx_apply_dist
    if world > 1:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
    T, _ = pw.build_tables(*_si8(), (12, 12, 12), (24, 24, 24), seed_v=4)
    nband = 9
    X = pw.random_orthonormal_psi(T.dm.ntot, nband, 13)
    occ = np.linspace(1.0, 0.2, nband)
    kern, _ = exx.exx_kernel_r2c(T.dm, 5.0, mu=0.106)
    s, n = band_range(nband, world, rank)
    state = {}

    def set_phi(phi, o):
        state["phi"] = exx.set_phi(T.dm, phi.numpy())
        state["occ"] = o

    def apply_exx(Xb):
        return torch.from_numpy(exx.add_mult_spinor_exx(T.dm, Xb.numpy(), state["phi"], kern, 0.25, state["occ"]))

    out = exx_apply_dist(set_phi, apply_exx, torch.tensor(X[s:s + n]), occ, nband)
    q.put((rank, s, out.numpy()))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def test_distributed_exchange_two_ranks_matches_one_rank():
    """V_x on band shards with the exchange orbitals all-gathered (two gloo
    ranks, uneven shards 5 + 4) equals the one-rank V_x bit for bit."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    res = {}
    for world in (1, 2):
        q = ctx.Queue()
        port = _free_port()
        procs = [ctx.Process(target=_exx_worker, args=(r, world, port, q)) for r in range(world)]
        for p in procs:
            p.start()
        parts = sorted(q.get(timeout=300) for _ in range(world))
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res[world] = np.concatenate([o for _, _, o in parts], 0)
    assert np.array_equal(res[1], res[2])


class _OracleScfOps:
    """scf_dist's operators on the CPU from the oracle: H*psi, the partial
    density sum_k w_k |psi_k,fine|^2 (the oracle's density before its
    normalisation), the Hartree potential and Teter93 LDA."""

    def __init__(self, L, z, pos, nc, nf, ecut):
        import torch
        from oracle import pw, scf
        self.pw, self.scf = pw, scf
        self.T, sp = pw.build_tables(L, z, pos, nc, nf)
        dm = self.T.dm
        rho_ps = np.zeros(dm.ntotFine)
        for p in pos:
            idx, dv = pw.pseudo_charge(pw.Atom(int(z), p), dm, sp)
            np.add.at(rho_ps, idx, dv[:, 0])
        self.rho_ps_np = rho_ps
        self.rho_ps = torch.from_numpy(rho_ps)
        self.vol, self.natom, self.eself, self.ecut = dm.vol, len(pos), sp.eself * len(pos), ecut
        self.gkk = scf.gkk_fine(dm)

    def set_vtot(self, vtot):
        self.T.vtot = vtot.numpy().copy()

    def apply_h(self, Xb):
        import torch
        return torch.from_numpy(self.pw.mult_spinor(self.T, Xb.numpy()))

    def density_raw(self, Xb, w):
        import torch
        pw, dm = self.pw, self.T.dm
        n0, n1, n2 = dm.numGrid
        N0, N1, N2 = dm.numGridFine
        p = Xb.numpy()
        Xc = pw.r2c(p.reshape(-1, n2, n1, n0), dm)
        Xf = self.T.ip.c2f(Xc.reshape(p.shape[0], -1)).reshape(p.shape[0], N2, N1, N0 // 2 + 1)
        pf = pw.c2r(Xf, dm, fine=True).reshape(p.shape[0], -1)
        return torch.from_numpy(np.einsum("b,bi->i", w.numpy(), pf * pf))

    def potentials(self, rho):
        import torch
        r = rho.numpy()
        vh = self.scf.hartree(self.T.dm, r, self.rho_ps_np, self.ecut, self.gkk)
        eps, vxc = self.scf.xc_teter93(r)
        return torch.from_numpy(vh), torch.from_numpy(vxc), torch.from_numpy(eps)


def _scf_worker(rank, world, port, q):
    import json
    from pathlib import Path

    import torch
    import torch.distributed as dist
    from oracle import pw
    from pwdft_develop_b200.parallel import band_range, scf_dist
    if world > 1:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
    g = json.loads((Path(__file__).resolve().parent / "golden" / "si8_scf_small.json").read_text())
    ops = _OracleScfOps(np.array(g["length"]), g["znuc"], np.array(g["positions"]), tuple(g["numGrid"]),
                        tuple(g["numGridFine"]), g["ecut"])
    nband = g["nocc"] + g["nextra"]
    X0 = torch.tensor(pw.random_orthonormal_psi(ops.T.dm.ntot, nband, 11))
    s, n = band_range(nband, world, rank)
    out, Xb = scf_dist(ops, X0[s:s + n].clone(), nband, g["nocc"], tol_efree=1e-7, max_iter=60, degree=10)
    if rank == 0:
        q.put((out["efree"], out["etot"], out["eig"], out["iterations"], out["converged"],
               out["rho"].numpy().sum() * ops.vol / out["rho"].numel()))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def test_distributed_scf_two_ranks_matches_one_rank_and_golden():
    """SCF over band shards (two gloo ranks: filtered bands split 12 + 12, the
    partial densities all-reduced, potentials and Anderson mixing replicated)
    follows the one-rank iteration and converges to the oracle's Si8 free
    energy (16^3 / 32^3, Ecut 5 Ha, LDA) within 1e-6 Ha per atom; the density
    holds 2 nocc electrons."""
    import json
    from pathlib import Path

    import torch.multiprocessing as mp
    g = json.loads((Path(__file__).resolve().parent / "golden" / "si8_scf_small.json").read_text())
    ctx = mp.get_context("spawn")
    out = {}
    for world in (1, 2):
        q = ctx.Queue()
        port = _free_port()
        procs = [ctx.Process(target=_scf_worker, args=(r, world, port, q)) for r in range(world)]
        for p in procs:
            p.start()
        out[world] = q.get(timeout=900)
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
    natom = len(g["positions"])
    for world in (1, 2):
        efree, etot, eig, it, conv, nel = out[world]
        assert conv, (world, it)
        assert abs(efree - g["efree"]) / natom < 1e-6, (world, efree - g["efree"])
        assert np.abs(eig[:g["nocc"]] - np.array(g["eig"][:g["nocc"]])).max() < 1e-5
        assert abs(nel - 2 * g["nocc"]) < 1e-9
    assert abs(out[1][0] - out[2][0]) / natom < 1e-8
