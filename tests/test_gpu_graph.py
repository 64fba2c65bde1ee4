"""Steps replayed from CUDA graphs (kaos_set_graph) give bit-identical
results to directly launched steps: same particles, ENAs, counts, moments
and boundary counters, across master steps, compaction buffer swaps,
injection and charge exchange, and across several kaos_step calls."""
import numpy as np
import pytest

from kaos_b200 import build as kbuild
from kaos_b200 import grids
from kaos_b200.lib import Solver
from kaos_b200.model_input import (KAOS_M0, KAOS_M2PAR, KAOS_NUPOI, KAOS_PREC_FP64,
                                   KAOS_PREC_MIXED, KAOS_PREC_MIXED_K64)

PRECISIONS = [KAOS_PREC_FP64, KAOS_PREC_MIXED, KAOS_PREC_MIXED_K64]

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _build():
    kbuild.build()


def _run(prec, graph, export, chunks):
    mi, spec, tube, vg = grids.config_small(n_particles=6000, three_d=True,
                                            steps_per_master=4, heating=True,
                                            collisions=True)
    mi.precision = prec
    tube.nsnormCLB = 30.0
    init = grids.initial_particles(tube, spec, mi, seed=11)
    s = Solver(mi, [tube], vg)
    s.load(0, *init)
    s.set_graph(graph)
    if export:
        s.set_export(True)
    for c in chunks:
        s.step(c)
    out = {"p": s.particles(), "e": s.enas(), "cnt": s.counts(),
           "b": s.boundary(), "n": s.count(),
           "m": [s.moments(k) for k in (KAOS_M0, KAOS_M2PAR, KAOS_NUPOI)]}
    if export:
        out["h"] = s.counts(full=True)
    s.close()
    return out


@pytest.mark.parametrize("prec", PRECISIONS)
def test_graph_replay_bit_identical(prec):
    chunks = (1, 6, 19, 3, 12)  # 41 steps: ten master steps, uneven calls
    a = _run(prec, False, False, chunks)
    b = _run(prec, True, False, chunks)
    assert a["n"] == b["n"]
    assert a["n"][1] > 0  # charge exchange produced ENAs
    for k in a["p"]:
        np.testing.assert_array_equal(a["p"][k], b["p"][k], err_msg=k)
    for k in a["e"]:
        np.testing.assert_array_equal(a["e"][k], b["e"][k], err_msg=k)
    np.testing.assert_array_equal(a["cnt"], b["cnt"])
    np.testing.assert_array_equal(a["b"], b["b"])
    for x, y in zip(a["m"], b["m"]):
        np.testing.assert_array_equal(x, y)


def test_graph_replay_with_export():
    chunks = (9, 8)
    a = _run(KAOS_PREC_FP64, False, True, chunks)
    b = _run(KAOS_PREC_FP64, True, True, chunks)
    np.testing.assert_array_equal(a["h"], b["h"])
    for k in a["p"]:
        np.testing.assert_array_equal(a["p"][k], b["p"][k], err_msg=k)


def _run_shape(prec, shape):
    mi, spec, tube, vg = grids.config_small(n_particles=9000, three_d=True,
                                            steps_per_master=4, heating=True,
                                            collisions=True)
    mi.precision = prec
    tube.nsnormCLB = 30.0
    init = grids.initial_particles(tube, spec, mi, seed=5)
    s = Solver(mi, [tube], vg)
    s.load(0, *init)
    if shape is not None:
        s.set_launch(*shape)
    s.step(13)
    out = {"p": s.particles(), "e": s.enas(), "cnt": s.counts(),
           "launch": s.launch()}
    s.close()
    return out


@pytest.mark.parametrize("prec", PRECISIONS)
def test_launch_shapes_bit_identical(prec):
    """Every push launch shape (ions per work item, one block per item or a
    persistent grid, register budget and block size) and the autotuner's
    choice give the same particles, ENAs and counts, in every precision
    mode."""
    ref = _run_shape(prec, (2048, 0))
    shapes = [(1024, 1), (4096, 0), None]
    if prec != KAOS_PREC_FP64:
        # bits 3-4: the master-step variant's budget + 1 (64 with 80, 72 with 64)
        shapes += [(1024, 2), (4096, 3), (2048, 4), (1024, 5), (2048, 2 | 8), (4096, 24)]
    for sh in shapes:
        o = _run_shape(prec, sh)
        if sh is not None:
            assert o["launch"] == sh
        else:
            assert o["launch"][0] in (1024, 2048, 4096)
        for k in ref["p"]:
            np.testing.assert_array_equal(ref["p"][k], o["p"][k], err_msg=f"{sh} {k}")
        for k in ref["e"]:
            np.testing.assert_array_equal(ref["e"][k], o["e"][k], err_msg=f"{sh} {k}")
        np.testing.assert_array_equal(ref["cnt"], o["cnt"])


def test_launch_mode_out_of_range_rejected():
    from kaos_b200.lib import KaosError
    mi, spec, tube, vg = grids.config_small(n_particles=500, three_d=True)
    mi.precision = KAOS_PREC_MIXED
    s = Solver(mi, [tube], vg)
    for chunk, mode in ((4096, 6), (3000, 0)):
        with pytest.raises(KaosError):
            s.set_launch(chunk, mode)
    s.set_launch(1024, 5)
    assert s.launch() == (1024, 5)
    s.close()


@pytest.mark.parametrize("tight", [False, True])
def test_graph_replay_with_escapes_and_deferred_packing(tight):
    """Mixed path on a tube losing ~40 ions per master step: escaped ions
    are marked dead in place and the arrays packed every few master steps
    (or when the capacity is tight); graph replay and direct launches give
    the same ions, counts and escape counts."""
    def run(graph):
        mi, spec, tube, vg = grids.config_escaping()
        mi.precision = KAOS_PREC_MIXED
        init = grids.initial_particles(tube, spec, mi, seed=29)
        if tight:
            tube.capacity = len(init[0]) + 70
        s = Solver(mi, [tube], vg)
        s.load(0, *init)
        s.set_graph(graph)
        bnd = []
        for c in (3, 6, 9, 4):  # 22 steps
            s.step(c)
            bnd.append(s.boundary())
        out = {"p": s.particles(), "cnt": s.counts(), "n": s.count(), "b": bnd}
        s.close()
        return out
    a, b = run(False), run(True)
    assert a["n"] == b["n"]
    for k in a["p"]:
        np.testing.assert_array_equal(a["p"][k], b["p"][k], err_msg=k)
    np.testing.assert_array_equal(a["cnt"], b["cnt"])
    np.testing.assert_array_equal(np.array(a["b"]), np.array(b["b"]))
    assert sum(x[0] + x[1] for x in a["b"]) > 50


@pytest.mark.parametrize("mixed", [False, True])
def test_state_reads_between_steps_change_nothing(mixed):
    """kaos_get_particles stages through the spare particle buffers, which
    the packing and the autotuner also use inside a step: reading the state
    between steps (across a master step with packing and the autotuner's
    first step) leaves the run bit-identical to one that never reads it."""
    def run(read):
        mi, spec, tube, vg = grids.config_escaping()
        if mixed:
            mi.precision = KAOS_PREC_MIXED
        init = grids.initial_particles(tube, spec, mi, seed=37)
        s = Solver(mi, [tube], vg)
        s.load(0, *init)
        for c in (1, 1, 3, 5, 6, 4):  # 20 steps, master every 2
            s.step(c)
            if read:
                s.particles()
        out = {"p": s.particles(), "cnt": s.counts(), "b": s.boundary()}
        s.close()
        return out
    a, b = run(False), run(True)
    for k in a["p"]:
        np.testing.assert_array_equal(a["p"][k], b["p"][k], err_msg=k)
    np.testing.assert_array_equal(a["cnt"], b["cnt"])
    np.testing.assert_array_equal(a["b"], b["b"])
