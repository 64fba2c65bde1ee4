"""F_alg: FP64 flop-equivalents per ion particle-step of the reference
formulation, counted by the op-counting build of the oracle
(oracle/op_count.cpp: kaos_oracle.c compiled with a counting double).

The weights are fixed (add/mul 1, div/sqrt 4, each transcendental call
20) and so is the count: the tests pin the per-ion breakdown of the push on
the 256-cell precision A/B tube, and the bench reports the FP64 path's
flop-equivalent rate with the same number.  The counted build must compute
exactly what the plain oracle computes, or its counts would describe other
arithmetic."""
import numpy as np
import pytest

import bench
from kaos_b200 import grids
from oracle import oracle as O

# per ion, one ordinary step of the push (KineticRK4UpdateSub with
# KineticUpdateA/B/C, WaveHeatingSub and the quartic re-projection)
F_ALG_CLASSES = {"add": 176, "mul": 554, "div": 158, "sqrt": 22,
                 "transcendental": 41}
F_ALG = 2270


def _push_counts(mi, tube, vg, spec, n_first=1, seed=5):
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=seed)
    o = O.Oracle(mi, tube, vg, counted=True)
    o.load(q, vpar, v1, v2)
    o.step(n_first)
    ni, _ = o.count()
    O.ops_reset()
    o.step(1)
    return O.ops_get(), ni


def test_weights_are_fixed():
    assert O.OPS_CLASSES == ("add", "mul", "div", "sqrt", "transcendental")
    assert O.OPS_WEIGHTS == (1, 1, 4, 4, 20)
    assert O.ops_weighted(F_ALG_CLASSES) == F_ALG


@pytest.mark.parametrize("collisions", [True, False])
def test_f_alg_of_the_precision_tube(collisions):
    mi, spec, tube, vg = grids.config_c2(n_particles=1500, collisions=collisions)
    c, ni = _push_counts(mi, tube, vg, spec)
    per_ion = {k: v / ni for k, v in c["push_ion"].items()}
    assert per_ion == pytest.approx(F_ALG_CLASSES, abs=1e-12)
    assert O.ops_weighted(c["push_ion"]) == F_ALG * ni
    # an ordinary step: no ENA, no charge exchange, no master-step work
    assert O.ops_weighted(c["master"]) == 0
    assert bench.F_ALG == F_ALG


def test_heating_costs_its_formula():
    """Without wave heating the push loses WaveHeatingSub's arithmetic:
    the Box-Muller log/cos/sin, four pow and the diffusion algebra."""
    mi, spec, tube, vg = grids.config_c2(n_particles=1000, heating=False)
    c, ni = _push_counts(mi, tube, vg, spec)
    per_ion = {k: v / ni for k, v in c["push_ion"].items()}
    assert per_ion["transcendental"] == F_ALG_CLASSES["transcendental"] - 7
    assert O.ops_weighted(c["push_ion"]) < F_ALG * ni


def test_counted_build_computes_what_the_oracle_computes():
    """Heating, charge exchange to ENAs, removal, injection and master
    steps: particles, ENAs, moments and counts bit-identical."""
    mi, spec, tube, vg = grids.config_small(n_particles=1500, heating=True,
                                            collisions=True, steps_per_master=5)
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=3)
    runs = []
    for counted in (False, True):
        o = O.Oracle(mi, tube, vg, counted=counted)
        o.load(q, vpar, v1, v2)
        o.step(17)
        runs.append((o.particles(), o.enas(),
                     [o.moments(k) for k in range(10)], o.counts(full=True)))
    (pa, ea, ma, ca), (pb, eb, mb, cb) = runs
    assert len(ea["x"]) > 0
    for k in pa:
        assert np.array_equal(pa[k], pb[k]), k
    for k in ea:
        assert np.array_equal(ea[k], eb[k]), k
    for a, b in zip(ma, mb):
        assert np.array_equal(a, b)
    assert np.array_equal(ca, cb)


def test_ena_push_is_cheaper_than_the_ion_push():
    """ENAs fly ballistically under gravity (no heating, no quartic)."""
    mi, spec, tube, vg = grids.config_small(n_particles=1500, heating=True,
                                            collisions=True, steps_per_master=5)
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=3)
    o = O.Oracle(mi, tube, vg, counted=True)
    o.load(q, vpar, v1, v2)
    o.step(12)
    ni, ne = o.count()
    assert ne > 0
    O.ops_reset()
    o.step(1)
    c = O.ops_get()
    assert 0 < O.ops_weighted(c["push_ena"]) / ne < F_ALG
    assert O.ops_weighted(c["charge_exchange"]) > 0
