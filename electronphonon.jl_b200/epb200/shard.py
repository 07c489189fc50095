"""Multi-GPU plumbing of the path: one process per GPU, k sharded, no data-path collective.

The path shards over outer k (the reference's `mpi_comm_k`, `src/calculator/run_eph_over_k_and_kq.jl:86-91`):
every k's outputs are independent, so each rank runs the whole pass on a contiguous k range. The only
exchanges are scalars and counts: the max-over-ranks step time, global sums for checksums, and, for the
energy-window filter, an all-gather of kept counts that turns each rank's local kept list into global
offsets (the reference's `mpi_allgather` of filtered counts, `src/filter.jl:76-100`).
"""
from __future__ import annotations


def shard_range(n: int, world: int, rank: int) -> tuple[int, int]:
    """[start, stop) of rank's share of n items: contiguous, sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of world {world}")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _dist():
    import torch.distributed as dist

    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(x: float, device="cpu") -> float:
    """Max of a scalar over all ranks (the step time of a weak-scaling run)."""
    import torch

    d = _dist()
    if d is None:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    d.all_reduce(t, op=d.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device="cpu") -> float:
    import torch

    d = _dist()
    if d is None:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    d.all_reduce(t, op=d.ReduceOp.SUM)
    return float(t.item())


def global_offsets(local_count: int, device="cpu") -> tuple[int, int]:
    """(offset of this rank's items in the global ascending list, global total) from an all-gather of
    the per-rank counts."""
    import torch

    d = _dist()
    if d is None:
        return 0, int(local_count)
    ws = d.get_world_size()
    t = torch.tensor([int(local_count)], dtype=torch.int64, device=device)
    out = [torch.zeros_like(t) for _ in range(ws)]
    d.all_gather(out, t)
    counts = [int(o.item()) for o in out]
    r = d.get_rank()
    return sum(counts[:r]), sum(counts)
