"""One tube split over two ranks (the reference's MPI particle split): two
handles on one GPU, each with half of the ions and disjoint id ranges, whose
binning accumulators are summed by a reduction hook before every set of
moments.  With wave heating on and no injection or charge exchange, each
share reproduces its slice of the unsplit run bit for bit, and both ranks
get the unsplit moments."""
import threading

import numpy as np
import pytest
import torch

from kaos_b200 import build as kbuild
from kaos_b200 import grids
from kaos_b200.lib import Solver
from kaos_b200.model_input import KAOS_EAMAG, KAOS_M0, KAOS_M2, KAOS_M2PAR
from kaos_b200.shard import _DeviceCounters, split_ions

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _build():
    kbuild.build()


class PairReduce:
    """Sums the accumulator blocks of two handles stepping in two threads:
    both hooks meet at a barrier, one adds, both continue."""

    def __init__(self):
        self.barrier = threading.Barrier(2, timeout=60)
        self.bufs = [None, None]
        self.calls = 0

    def hook(self, rank):
        def fn(buf, count, stream):
            self.bufs[rank] = torch.as_tensor(_DeviceCounters(buf, count), device="cuda")
            self.barrier.wait()
            if rank == 0:
                tot = self.bufs[0] + self.bufs[1]
                self.bufs[0].copy_(tot)
                self.bufs[1].copy_(tot)
                torch.cuda.synchronize()
                self.calls += 1
            self.barrier.wait()
            return 0
        return fn


def test_split_tube_matches_unsplit():
    mi, spec, tube, vg = grids.config_small(n_particles=6000, three_d=True,
                                            steps_per_master=4, heating=True)
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=21)
    steps = 11
    ref = Solver(mi, [tube], vg)
    ref.load(0, q, vpar, v1, v2)
    ref.step(steps)
    shares = split_ions(len(q), 2)
    red = PairReduce()
    solvers = []
    for r, sh in enumerate(shares):
        s = Solver(mi, [tube], vg)
        s.set_id_base(0, sh.start)
        s.set_rank(r, 2)
        s.set_reduce(red.hook(r))
        s.load(0, q[sh.start:sh.stop], vpar[sh.start:sh.stop],
               v1[sh.start:sh.stop], v2[sh.start:sh.stop])
        solvers.append(s)
    errors = []

    def run(s):
        try:
            s.step(steps)
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(e)
            red.barrier.abort()

    th = [threading.Thread(target=run, args=(s,)) for s in solvers]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=120)
    assert not errors, errors
    assert red.calls >= 3  # step 1 and the master steps 4 and 8
    pr = ref.particles()
    for r, (s, sh) in enumerate(zip(solvers, shares)):
        ps = s.particles()
        for k in ("z", "rho", "vpar", "vperp1", "vperp2"):
            np.testing.assert_array_equal(ps[k], pr[k][sh.start:sh.stop], err_msg=f"{r} {k}")
        for m in (KAOS_M0, KAOS_M2, KAOS_M2PAR, KAOS_EAMAG):
            np.testing.assert_array_equal(s.moments(m), ref.moments(m), err_msg=f"{r} {m}")
        np.testing.assert_array_equal(s.counts(), ref.counts())


def test_nccl_hook_on_a_one_rank_group(tmp_path):
    """shard.nccl_reduce_hook as a Solver.set_reduce hook on a one-rank NCCL
    process group: the all-reduce runs on the library's stream at every
    statistics step (here the identity) and the run equals the unhooked one
    bit for bit.  (The two-rank sum is checked by the host-barrier hook
    above and, over gloo on host memory, by the CPU tests.)"""
    import torch.distributed as dist
    from kaos_b200.shard import nccl_reduce_hook
    mi, spec, tube, vg = grids.config_small(n_particles=3000, three_d=True,
                                            steps_per_master=4, heating=True)
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=22)
    ref = Solver(mi, [tube], vg)
    ref.load(0, q, vpar, v1, v2)
    ref.step(9)
    store = dist.FileStore(str(tmp_path / "pg"), 1)
    dist.init_process_group("nccl", store=store, rank=0, world_size=1)
    try:
        inner = nccl_reduce_hook()
        calls = []

        def hook(buf, count, stream):
            calls.append(stream)
            return inner(buf, count, stream)

        s = Solver(mi, [tube], vg)
        s.set_rank(0, 1)
        s.set_reduce(hook)
        s.load(0, q, vpar, v1, v2)
        s.step(9)
        assert len(calls) >= 3 and all(calls)  # step 1, master steps 4 and 8
        np.testing.assert_array_equal(s.counts(), ref.counts())
        for m in (KAOS_M0, KAOS_M2, KAOS_M2PAR, KAOS_EAMAG):
            np.testing.assert_array_equal(s.moments(m), ref.moments(m))
        s.close()
    finally:
        dist.destroy_process_group()
    ref.close()
