"""Multi-rank path on CPU: world_size 2 over gloo (127.0.0.1).  Each rank
advances its share of tubes (here on the CPU oracle, the compute engine is a
callable), results are all-gathered and must equal a single-process run;
the step time is reduced as the maximum over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from kaos_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _tube_problem(k):
    from kaos_b200 import grids
    mi, spec, tube, vg = grids.config_small(n_particles=800 + 300 * k, nq=16 + 4 * k,
                                            steps_per_master=3)
    tube.nsnormCLB = 5.0
    return mi, spec, tube, vg


def _run_tube(k):
    from kaos_b200 import grids
    from kaos_b200.model_input import KAOS_M0, KAOS_M1PAR
    from oracle.oracle import Oracle
    mi, spec, tube, vg = _tube_problem(k)
    init = grids.initial_particles(tube, spec, mi, seed=50 + k)
    o = Oracle(mi, tube, vg)
    o.load(*init)
    o.step(7)
    return {"counts": o.counts(), "M0": o.moments(KAOS_M0),
            "M1par": o.moments(KAOS_M1PAR), "n": o.count()[0]}


def _worker(rank, world, port, counts, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = shard.run_rank(rank, world, counts, _run_tube)
        merged = shard.gather_results(local, dist)
        tmax = shard.max_over_ranks(1.0 + rank, dist)
        if rank == 0:
            q.put((merged, tmax, sorted(local)))
        else:
            q.put(("rank1", sorted(local)))
    finally:
        dist.destroy_process_group()


def _hook_worker(rank, world, port, q):
    """One rank of a split tube: its accumulator block (uint32 counters in
    host memory) is summed over the ranks in place through the hook
    contract the library calls (fn(buf_ptr, count, stream_ptr) -> 0)."""
    import ctypes

    import torch.distributed as dist
    from kaos_b200.lib import REDUCE_FN
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 1 + 3 * 4099                     # ncell x (1 + n|| + n1 + n2) counters
        buf = (ctypes.c_uint32 * n)()
        for i in range(n):
            buf[i] = (i * 7 + rank * 1000003) % 65536
        hook = shard.host_reduce_hook()
        cb = REDUCE_FN(lambda ctx, p, count, stream: int(hook(p, count, stream)))
        rc = cb(None, ctypes.addressof(buf), n, None)
        q.put((rank, rc, list(buf)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_split_tube_hook_sums_accumulators_in_place():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_hook_worker, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    n = len(res[0][2])
    want = [sum((i * 7 + r * 1000003) % 65536 for r in range(world)) for i in range(n)]
    for rank, rc, got in res:
        assert rc == 0
        assert got == want


def test_assign_tubes_balances_and_covers():
    counts = [10, 200, 30, 150, 90, 5]
    a = shard.assign_tubes(counts, 3)
    flat = sorted(k for r in a for k in r)
    assert flat == list(range(len(counts)))
    loads = [sum(counts[k] for k in r) for r in a]
    assert max(loads) - min(loads) <= max(counts)
    assert shard.assign_tubes(counts, 3) == a  # deterministic
    assert shard.assign_tubes(counts, 1) == [list(range(len(counts)))]


@pytest.mark.timeout(300)
def test_two_ranks_gloo_match_single_process():
    ntubes = 3
    counts = [800 + 300 * k for k in range(ntubes)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, counts, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    r0 = next(r for r in res if r[0] != "rank1")
    r1 = next(r for r in res if r[0] == "rank1")
    merged, tmax, mine0 = r0
    assert tmax == 2.0
    assert sorted(mine0 + r1[1]) == list(range(ntubes))
    assert sorted(merged) == list(range(ntubes))
    for k in range(ntubes):
        ref = _run_tube(k)
        np.testing.assert_array_equal(merged[k]["counts"], ref["counts"])
        np.testing.assert_array_equal(merged[k]["M0"], ref["M0"])
        assert merged[k]["n"] == ref["n"]


def test_split_ions_and_conversion_shares():
    """A split tube: contiguous shares that cover every ion once, and the
    per-rank shares floor((N + r) / R) of a cell's conversions sum to N."""
    from kaos_b200.shard import split_ions
    for n, world in ((10, 3), (7, 7), (5, 8), (123457, 4)):
        sh = split_ions(n, world)
        assert sum(len(s) for s in sh) == n
        assert [i for s in sh for i in s] == list(range(n))
        for N in (0, 1, 2, 5, 17, 1000):
            assert sum((N + r) // world for r in range(world)) == N
