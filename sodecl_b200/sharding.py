"""Orbit sharding across ranks (one process per GPU).

Orbits are independent and the integrators have no exchange step, so N GPUs
split the orbits into contiguous ranges and integrate them with no collective
on the data path; the noise stream of an orbit is keyed by its global index
(the Threefry counter word 0), so results do not depend on the split.  The only
collectives are a barrier around timing and the max of the ranks' times.
"""
from __future__ import annotations


def shard(n_total: int, rank: int, world: int):
    """(first global orbit, number of orbits) of `rank`: contiguous ranges,
    sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world or n_total < 0:
        raise ValueError("bad shard request")
    base, extra = divmod(n_total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest `value` over all ranks (the whole job's time is its slowest
    rank's)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
