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
