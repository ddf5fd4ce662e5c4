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


def shard_cells(ncell: int, rank: int, world: int):
    """[lo, hi) shells whose opacity `rank` builds (the opacity of a shell
    depends on that shell alone: physical_opacity.f:94-247)."""
    return shard_range(ncell, rank, world)


def gather_cells(local, ncell: int, group=None):
    """All-gather per-shell rows: `local` holds this rank's shells
    shard_cells(ncell, rank, world) along dim 0 (e.g. gas_cap (n, ng) FP32,
    gas_sig / capgrey / capross (n,) FP64); returns the (ncell, ...) tensor on
    every rank, in shell order (the exchange of mpimod_mpi.f:668-711 after a
    cell-sharded opacity build).  Ranks' slices differ by at most one shell,
    so each is padded to the largest before one all_gather."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    sizes = [shard_cells(ncell, r, world) for r in range(world)]
    nmax = max(hi - lo for lo, hi in sizes)
    pad = torch.zeros((nmax,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:hi - lo] for p, (lo, hi) in zip(parts, sizes)], dim=0)
