"""Tube sharding across ranks (one process per GPU), and a tube split.

Flux tubes never interact in the reference -- species and tubes are the
outermost sequential loops around the time loop (_8_KineticSolver.f90:43-44)
-- so a multi-GPU run gives each rank a set of whole tubes and needs no
collective on the data path.  Only the results are gathered (per-tube moments
and counts to rank 0) and the timing is reduced as the maximum over ranks.

A tube larger than one GPU is split instead, as the reference's MPI ranks
split a tube's particles: every rank holds the tube's tables and a share of
its ions (`split_ions`), and the per-cell binning accumulators are summed
over the ranks before each set of moments (MPIReduceSumSub,
_9_MPIReduceSum.f90:25-55), here by one NCCL all-reduce of the handle's
accumulator block (`nccl_reduce_hook`, given to Solver.set_reduce).
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


def split_ions(n: int, world: int) -> List[range]:
    """Contiguous shares of n ions over `world` ranks (the first n % world
    ranks hold one more); rank r's ions keep their global ids."""
    base, extra = divmod(n, world)
    out, start = [], 0
    for r in range(world):
        m = base + (1 if r < extra else 0)
        out.append(range(start, start + m))
        start += m
    return out


class _DeviceCounters:
    """A device buffer of int32 counters seen through the CUDA array
    interface (the accumulators are uint32; every count fits in int32)."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<i4",
                                         "data": (int(ptr), False), "version": 3}


def nccl_reduce_hook(group=None):
    """A Solver.set_reduce hook: in-place sum of the accumulator block over
    the process group (NCCL on GPUs), ordered on the library's stream (the
    hook's `stream` argument), then wait for it."""
    import torch
    import torch.distributed as dist

    def hook(buf: int, count: int, stream: int) -> int:
        t = torch.as_tensor(_DeviceCounters(buf, count), device="cuda")
        s = torch.cuda.ExternalStream(int(stream)) if stream else torch.cuda.current_stream()
        with torch.cuda.stream(s):
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        s.synchronize()
        return 0

    return hook


def host_reduce_hook(group=None):
    """The same hook contract over HOST memory (a CPU process group such as
    gloo): in-place sum of `count` 32-bit counters at host address `buf`
    over the group.  For ranks that hold their accumulators on the host."""
    import ctypes

    import numpy as np
    import torch
    import torch.distributed as dist

    def hook(buf: int, count: int, stream: int) -> int:
        a = np.ctypeslib.as_array((ctypes.c_int32 * int(count)).from_address(int(buf)))
        dist.all_reduce(torch.from_numpy(a), op=dist.ReduceOp.SUM, group=group)
        return 0

    return hook
