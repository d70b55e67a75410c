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
