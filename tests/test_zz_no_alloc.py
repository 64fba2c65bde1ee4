"""The allocation-free statistics entry point (kaos_moments_noalloc).

Callers that cannot allocate device memory (a host with its own fixed
device pool, a GPU shared under a memory cap) get the start-of-step counts and moments from this entry point, whose
scratch histograms live in a static device array.  This test drives it
through the C-ABI on device buffers the test owns, twice in a row (the
second call must clear what the first left behind), and checks both results
against the existing path (kaos_step of a handle, then kaos_get_moments /
kaos_get_counts) on the same ions: counts bit-exact, moments within 1e-10
relative, the tolerance of the other GPU parity tests.

It is collected last so that a run stopping at the first failure has already
run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from kaos_b200 import build as kbuild
from kaos_b200 import grids
from kaos_b200 import lib as klib
from kaos_b200.model_input import KAOS_NQ

pytestmark = pytest.mark.gpu
MOM_TOL = 1e-10


def test_noalloc_matches_handle_path_twice():
    import torch
    kbuild.build()
    L = klib.load()
    mi, spec, tube, vg = grids.config_small(n_particles=5000, three_d=True)
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=17)
    # existing path: first step statistics of a handle
    s = klib.Solver(mi, [tube], vg)
    s.load(0, q, vpar, v1, v2)
    s.step(1)
    ref = np.stack([s.moments(k) for k in range(KAOS_NQ + 1)])
    ref_counts = s.counts()
    s.close()
    # allocation-free path on device buffers owned by the caller (here torch)
    dev = torch.device("cuda:0")
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    edges = t(np.append(tube.qGL, tube.qGH[-1]))
    d3x = t(tube.d3xC)
    dq, dvp, dv1, dv2 = t(q), t(vpar), t(v1), t(v2)
    nq = tube.nq
    pc, vgc = mi.to_c(), vg.to_c()
    for call in range(2):
        out = torch.full((KAOS_NQ + 1, nq), -1.0, dtype=torch.float64, device=dev)
        cnt = torch.full((nq,), -1, dtype=torch.int64, device=dev)
        rc = L.kaos_moments_noalloc(C.addressof(pc), C.addressof(vgc), nq,
                                    edges.data_ptr(), d3x.data_ptr(),
                                    tube.nsnormfac, dq.data_ptr(), dvp.data_ptr(),
                                    dv1.data_ptr(), dv2.data_ptr(), len(q),
                                    out.data_ptr(), cnt.data_ptr(), None)
        assert rc == 0, call
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_array_equal(cnt.cpu().numpy(), ref_counts)
        for k in range(KAOS_NQ + 1):
            scale = max(np.max(np.abs(ref[k])), 1e-300)
            assert np.max(np.abs(got[k] - ref[k])) / scale <= MOM_TOL, (call, k)


def test_noalloc_rejects_oversize_grid():
    kbuild.build()
    L = klib.load()
    mi, spec, tube, vg = grids.config_small(n_particles=100, three_d=True)
    pc, vgc = mi.to_c(), vg.to_c()
    dummy = C.c_double(0.0)
    # 513 cells exceed the static array: rejected before any device work
    rc = L.kaos_moments_noalloc(C.addressof(pc), C.addressof(vgc), 513,
                                C.addressof(dummy), C.addressof(dummy), 1.0,
                                None, None, None, None, 0, C.addressof(dummy),
                                None, None)
    assert rc == 2  # KAOS_ERR_CAPACITY
    # a 3D grid needs the Vperp2 array whenever there are ions to bin
    rc = L.kaos_moments_noalloc(C.addressof(pc), C.addressof(vgc), tube.nq,
                                C.addressof(dummy), C.addressof(dummy), 1.0,
                                C.addressof(dummy), C.addressof(dummy),
                                C.addressof(dummy), None, 1, C.addressof(dummy),
                                None, None)
    assert rc == 1  # KAOS_ERR_PARAM
