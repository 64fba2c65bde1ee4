"""Tube sharding across ranks (one process per GPU).

Flux tubes never interact in the reference -- species and tubes are the
outermost sequential loops around the time loop (_8_KineticSolver.f90:43-44)
-- so a multi-GPU run gives each rank a set of whole tubes and needs no
collective on the data path.  Only the results are gathered (per-tube moments
and counts to rank 0) and the timing is reduced as the maximum over ranks.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Sequence


def assign_tubes(particle_counts: Sequence[int], world: int) -> List[List[int]]:
    """Greedy largest-first assignment of tubes to ranks balancing the
    particle count per rank; deterministic (ties by tube index)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(particle_counts)), key=lambda k: (-particle_counts[k], k))
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda i: (load[i], i))
        out[r].append(k)
        load[r] += particle_counts[k]
    for lst in out:
        lst.sort()
    return out


def run_rank(rank: int, world: int, particle_counts: Sequence[int],
             run_tube: Callable[[int], Dict]) -> Dict[int, Dict]:
    """Advance this rank's tubes with `run_tube(tube_index) -> result dict`."""
    mine = assign_tubes(particle_counts, world)[rank]
    return {k: run_tube(k) for k in mine}


def gather_results(local: Dict[int, Dict], dist) -> Dict[int, Dict]:
    """All-gather the per-tube result dicts (object collective; results are
    small per-cell arrays) and merge them on every rank."""
    world = dist.get_world_size()
    bucket: List = [None] * world
    dist.all_gather_object(bucket, local)
    merged: Dict[int, Dict] = {}
    for part in bucket:
        merged.update(part)
    return merged


def max_over_ranks(value: float, dist, device=None) -> float:
    """Device time of a multi-rank step: the maximum over ranks."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
