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
    """(first grid point, number of points) of the row partition used for Gram blocks."""
    return band_range(ntot, world, rank)


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


def gram_row_partitioned(X_rows, Y_rows):
    """X^T Y for blocks partitioned by grid rows (each rank holds rows of all
    bands): local product then a sum over ranks."""
    G = X_rows.transpose(0, 1) @ Y_rows
    return allreduce_sum_(G)
