"""The benchmark configurations built on the host (kaos_b200.grids): the
sizes and parameter ranges each one states."""
import numpy as np

from kaos_b200 import grids
from kaos_b200.model_input import MH, MO, RE


def test_batched_uneven_tubes_config():
    mi, specs, tubes, vg = grids.config_c4()
    assert len(tubes) == 256
    assert all(2.0 <= s.L <= 8.0 for s in specs)
    assert all(64 <= t.nq <= 512 for t in tubes)
    n = np.array([int(t._counts.sum()) for t in tubes])
    assert 4e7 < n.sum() < 8e7
    assert n.min() > 5e3 and n.max() < 2e6
    assert all(t.capacity > c for t, c in zip(tubes, n))
    assert (vg.n1, vg.n2, vg.npar) == (48, 48, 64)
    assert mi.ICRflag == 1 and mi.QEXCHANGEflag == 0


def test_species_ena_convection_config():
    mi, specs, tubes, vg, evg = grids.config_c5()
    assert len(tubes) == 128
    assert [s.ms for s in specs[:4]] == [MO, MH, MO, MH]
    assert all(3.0 <= s.L <= 7.0 and s.nq == 256 for s in specs)
    assert all(specs[2 * k].L == specs[2 * k + 1].L for k in range(64))
    n = sum(int(t._counts.sum()) for t in tubes)
    assert abs(n - 2e7) < 1e5
    o = sum(int(t._counts.sum()) for t in tubes[0::2])
    assert abs(o / n - 0.8) < 0.01  # O+ : H+ = 4 : 1
    assert mi.QEXCHANGEflag == 1 and mi.mNeut == MH
    # 0.5 km/s over a master interval of 50 steps of 5 ms, in Earth radii
    assert abs(grids.CONV_C5_DL * RE - 500.0 * 0.25) < 1e-9
    moved = grids.moved_tube(specs[0], mi, tubes[0], specs[0].L + grids.CONV_C5_DL)
    np.testing.assert_array_equal(moved.qGL, tubes[0].qGL)
    assert moved.pG == specs[0].L + grids.CONV_C5_DL


def test_large_tube_config():
    mi, spec, tube, vg = grids.config_c3(n_particles=1_000_000)
    assert tube.nq == 512 and spec.L == 6.0
    assert (vg.n1, vg.n2, vg.npar) == (64, 64, 96)
    # heating, collisions, and LB injection sampled from the Maxwellian flux
    assert mi.ICRflag == 1 and mi.QEXCHANGEflag == 1 and mi.FLUXINJECTIONflag == 1
    assert mi.LBCONDITIONflag == 1 and tube.nsnormCLB > 0
    assert abs(grids.conv_c5_dl(10) * RE - 500.0 * 10 * 0.005) < 1e-9


def test_heating_rate_calibration():
    """S0 is set so that the base cell's Maxwellian ions gain 1e-3 eV/s under
    the reference's stochastic kick: the oracle's kick variance over 40 steps
    of the precision A/B tube gives that rate within 10 %."""
    from oracle.oracle import Oracle
    mi, spec, tube, vg = grids.config_c2(n_particles=100_000, heating=True,
                                         collisions=False, ndatfac=1000)
    tube.nsnormCLB = 0.0
    o = Oracle(mi, tube, vg)
    o.load(*grids.initial_particles(tube, spec, mi, seed=3))
    p0 = o.particles()
    o.step(40)
    p1 = o.particles()
    base = p0["qind"] == 0
    d2 = (p1["vperp1"] - p0["vperp1"]) ** 2 + (p1["vperp2"] - p0["vperp2"]) ** 2
    rate = 0.5 * mi.ms * d2[base].mean() / 1.602e-19 / (40 * mi.h)
    assert abs(rate - 1e-3) < 1e-4, rate
