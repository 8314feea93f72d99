"""Multi-GPU sharding of the DFT subtract: one process per GPU, no data-path
collective.

Visibility records are independent given the component table (each output
(row, channel, IF) depends only on that row's u, v, w and the shared model), so
rows -- or, for a multi-facet job, whole facets -- are partitioned across ranks
and every rank updates its own records in place.  The only inter-rank traffic
is one broadcast of the component table from rank 0 before the first pass, and
the max-over-ranks reduction of the timing.

Reference for what is sharded: ObitSkyModelFTDFT splits rows over host
threads the same way (ObitSystem/Obit/src/ObitSkyModel.c:2298-2327), and
ObitGPUSkyModelDFTCalc takes whole buffers of rows
(ObitSystem/Obit/src/ObitGPUSkyModel.c:502-518).
"""
from __future__ import annotations

from typing import Sequence


def row_shard(nrows: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced [lo, hi) of `nrows` for `rank` of `world`: the
    first nrows % world ranks take one extra row."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    if nrows < 0:
        raise ValueError("negative row count")
    base, extra = divmod(nrows, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def facet_assignment(work: Sequence[float], world: int) -> list[list[int]]:
    """Whole facets to ranks, largest first onto the least-loaded rank
    (greedy LPT).  `work[i]` is facet i's cost (component-visibility evals).
    Returns, per rank, its facet indices in decreasing-work order.  Ties go to
    the lower rank and then the lower facet index, so every rank computes the
    same assignment without communication."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda k: (-float(work[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += float(work[i])
    return out


def broadcast_model(comps, group=None):
    """Replicate the component table (a torch tensor, same shape on every
    rank; device memory under NCCL, host memory under gloo) from rank 0."""
    import torch.distributed as dist

    dist.broadcast(comps, 0, group=group)
    return comps


def max_over_ranks(x: float, device=None, group=None) -> float:
    """Maximum of a per-rank scalar (a device-timed duration) over all ranks."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
