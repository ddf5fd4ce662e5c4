"""Particle sharding over ranks (one process per GPU).

The reference runs particles on every MPI rank over a replicated grid
(inputparmod.f:465-471) and sums the transport tallies on the way out
(reduce_gridtally / reduce_fluxtally / reduce_totals, mpimod_mpi.f:771-978).
Here each rank owns a contiguous range of particle slots (or creates its own
source particles) and the tallies are summed with one all-reduce per
timestep; particles never move between ranks, so there is no other exchange.
"""
from __future__ import annotations


def shard_range(npart: int, rank: int, world: int):
    """[lo, hi) particle slots of `rank` (sizes differ by at most one)."""
    base, extra = divmod(npart, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def rank_seed(seed: int, rank: int) -> int:
    """Per-rank stream key: ranks draw from disjoint Philox key spaces."""
    return (seed & 0xFFFFFFFF) | ((rank + 1) << 40)


def reduce_tallies(tensors, group=None):
    """Sum grid / flux tallies over all ranks in place (torch.distributed)."""
    import torch.distributed as dist
    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def reduce_counters(counters: dict, device, group=None) -> dict:
    """Sum the step/particle counters and take the max of nstepmax over ranks."""
    import torch
    import torch.distributed as dist
    keys = ("npckt", "nflux", "nstepimc", "nstepddmc", "nmethodswap", "nposwarn")
    v = torch.tensor([float(counters[k]) for k in keys], dtype=torch.float64, device=device)
    dist.all_reduce(v, op=dist.ReduceOp.SUM, group=group)
    m = torch.tensor([float(counters["nstepmax"])], dtype=torch.float64, device=device)
    dist.all_reduce(m, op=dist.ReduceOp.MAX, group=group)
    out = {k: int(x) for k, x in zip(keys, v.tolist())}
    out["nstepmax"] = int(m.item())
    return out
