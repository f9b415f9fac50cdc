"""Multi-GPU host logic: one process per GPU, independent volumes per rank.

The extraction shards by volume, never inside one: every rank builds and
traverses its own volumes with no collective on the data path (weak scaling).
The only communication is on the host side of the measurement -- the maximum
of the ranks' device times -- and, for a batch, the split of the volumes over
the ranks, which every rank computes identically from the volume sizes.
"""
from __future__ import annotations


def split_volumes(cells, world: int):
    """Greedy longest-first split of volumes (given their cell counts) over
    `world` ranks; returns one sorted index list per rank.  Deterministic: every
    rank computes the same split without communicating."""
    order = sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += int(cells[i])
    return [sorted(p) for p in parts]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar (a device time) over the process group;
    the value itself when no group is initialised."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    """Sum of a per-rank count (volumes, vertices) over the process group."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
