"""Edge cases of the CUDA path against the oracle: the largest tube (2048
cells) and velocity grid (128 bins per axis) the library accepts, and
batches holding an empty entry and a single-ion entry (injection fills
the empty one)."""
import numpy as np
import pytest

from kaos_b200 import build as kbuild
from kaos_b200 import grids
from kaos_b200.grids import TubeSpec, make_tube, make_vgrid
from kaos_b200.lib import KaosError, Solver
from kaos_b200.model_input import (KAOS_M0, KAOS_M1PAR, KAOS_M2, KAOS_M2PAR,
                                   KAOS_PREC_MIXED, ModelInput)
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

TRAJ_TOL = 1e-12
MOM_TOL = 1e-10


@pytest.fixture(scope="module", autouse=True)
def _build():
    kbuild.build()


def rel_norm(a, b):
    scale = max(np.max(np.abs(b)), 1e-300)
    return np.max(np.abs(a - b)) / scale


def _compare(s, k, o):
    assert s.count(k) == o.count(), k
    po, ps = o.particles(), s.particles(k)
    for key in ("z", "vpar", "vperp1", "vperp2"):
        if len(po[key]):
            assert rel_norm(ps[key], po[key]) < TRAJ_TOL, (k, key)
    np.testing.assert_array_equal(s.counts(k), o.counts())
    for m in (KAOS_M0, KAOS_M1PAR, KAOS_M2, KAOS_M2PAR):
        assert rel_norm(s.moments(m, k), o.moments(m)) < MOM_TOL, (k, m)


def _run_one(mi, spec, vg, steps, seed=1):
    t = make_tube(spec, mi)
    init = grids.initial_particles(t, spec, mi, seed=seed)
    s = Solver(mi, [t], vg)
    s.load(0, *init)
    s.step(steps)
    o = Oracle(mi, t, vg)
    o.load(*init)
    o.step(steps)
    return s, o


def test_largest_tube_2048_cells():
    mi = ModelInput(h=0.01, ndatfac=3, ION2VPERPflag=1, ICRflag=1, QEXCHANGEflag=1)
    spec = TubeSpec(L=4.0, nq=2048, n_particles=20000, q_ub=1e-3, H=900e3,
                    heat_rate_eV_s=5.0, neut_n0=3e18, neut_H=300e3)
    vg = make_vgrid(True, 16, 16, 24, 8e3)
    s, o = _run_one(mi, spec, vg, 7)
    _compare(s, 0, o)
    # the mixed path runs the same tube (shared tables of 2048 cells)
    mi.precision = KAOS_PREC_MIXED
    t = make_tube(spec, mi)
    init = grids.initial_particles(t, spec, mi, seed=1)
    m = Solver(mi, [t], vg)
    m.load(0, *init)
    m.step(7)
    assert rel_norm(m.moments(KAOS_M0), o.moments(KAOS_M0)) < 2e-2


def test_largest_velocity_grid_128_bins():
    mi = ModelInput(h=0.01, ndatfac=3, ION2VPERPflag=1)
    spec = TubeSpec(L=4.0, nq=12, n_particles=5000, q_ub=0.3, H=600e3)
    vg = make_vgrid(True, 128, 128, 128, 6e3)
    s, o = _run_one(mi, spec, vg, 7)
    _compare(s, 0, o)


def test_limits_rejected():
    mi = ModelInput(h=0.01, ndatfac=3, ION2VPERPflag=1)
    vg = make_vgrid(True, 16, 16, 24, 8e3)
    t = make_tube(TubeSpec(nq=2049, n_particles=1000, q_ub=1e-3), mi)
    with pytest.raises(KaosError):
        Solver(mi, [t], vg)
    t = make_tube(TubeSpec(nq=16, n_particles=1000, q_ub=0.2), mi)
    with pytest.raises(KaosError):
        Solver(mi, [t], make_vgrid(True, 130, 16, 24, 8e3))
    # a tube shorter than the moment filter's window (11 cells)
    t = make_tube(TubeSpec(nq=10, n_particles=1000, q_ub=0.2), mi)
    with pytest.raises(KaosError):
        Solver(mi, [t], vg)


def test_empty_and_single_ion_entries():
    mi = ModelInput(h=0.01, ndatfac=3, ION2VPERPflag=1, ICRflag=1, QEXCHANGEflag=1)
    vg = make_vgrid(True, 16, 16, 24, 8e3)
    common = dict(L=4.0, nq=20, q_ub=0.15, H=600e3, heat_rate_eV_s=5.0,
                  neut_n0=3e18, neut_H=300e3)
    specs = [TubeSpec(n_particles=600, **common), TubeSpec(n_particles=600, **common),
             TubeSpec(n_particles=600, **common)]
    tubes = [make_tube(sp, mi) for sp in specs]
    tubes[0].nsnormCLB = 12.0  # the empty entry fills by injection
    full = grids.initial_particles(tubes[2], specs[2], mi, seed=3)
    inits = [tuple(np.zeros(0) for _ in range(4)),
             tuple(a[:1].copy() for a in full), full]
    s = Solver(mi, tubes, vg)
    for k in range(3):
        s.load(k, *inits[k])
    s.step(10)
    for k in range(3):
        o = Oracle(mi, tubes[k], vg)
        o.load(*inits[k])
        o.step(10)
        _compare(s, k, o)
    assert s.count(0)[0] > 0


@pytest.mark.parametrize("mixed", [False, True])
def test_state_export_skips_converted_slots(mixed):
    """kaos_get_particles (device export) between master steps, while slots
    converted to ENAs are still in the ion arrays: the live ions in order,
    the same into caller-provided arrays, and n must equal the live count."""
    mi, spec, tube, vg = grids.config_small(n_particles=6000, three_d=True,
                                            steps_per_master=5, collisions=True)
    if mixed:
        mi.precision = KAOS_PREC_MIXED
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=17)
    s = Solver(mi, [tube], vg)
    s.load(0, q, vpar, v1, v2)
    s.step(8)  # master step at 5; conversions at 6..8 leave dead slots
    ni, ne = s.count()
    assert ne > 0
    a = s.state()
    assert len(a["q"]) == ni
    assert np.all(a["qind"] >= -2)
    out = {k: np.full(ni + 7, np.nan) for k in ("q", "vpar", "vperp1", "vperp2")}
    out["qind"] = np.full(ni + 7, 99, dtype=np.int32)
    b = s.state(out=out)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert np.isnan(out["q"][ni]) and out["qind"][ni] == 99  # nothing past n
    from kaos_b200.lib import load
    import ctypes as C
    buf = np.zeros(ni + 1)
    rc = load().kaos_get_particles(s.h, 0, buf.ctypes.data_as(C.c_void_p), None,
                                   None, None, None, ni + 1)
    assert rc != 0
    s.close()


def test_mixed_bins_equal_host_binning():
    """The mixed push's start-of-step velocity bins (a lookup table plus a
    walk over the FP32 edges) and cells equal a plain search on the host:
    the full histogram of a master step against the host's count of the
    same ions (the state after the step before it)."""
    mi, spec, tube, vg = grids.config_small(n_particles=20000, three_d=True,
                                            steps_per_master=4)
    mi.precision = KAOS_PREC_MIXED
    tube.nsnormCLB = 0.0  # no injected ions in the master step's counts
    init = grids.initial_particles(tube, spec, mi, seed=41)
    s = Solver(mi, [tube], vg)
    s.load(0, *init)
    s.set_export(True)
    s.step(3)
    P = s.particles()
    s.step(1)  # master step 4 bins the state P
    H = s.counts(full=True)
    s.close()
    qGL, qGH = np.asarray(tube.qGL), np.asarray(tube.qGH)
    sgn = 1.0 if qGL[0] <= 0.0 else -1.0
    E = sgn * np.append(qGL, qGH[-1])
    sq = sgn * P["q"]
    cell = np.searchsorted(E, sq, side="left") - 1
    cell[sq == E[0]] = 0
    cell[(sq < E[0]) | (sq > E[-1])] = -1

    def vbin(e, v):
        e32, v32 = np.asarray(e, np.float32), np.asarray(v, np.float32)
        b = np.searchsorted(e32, v32, side="left") - 1
        b[v32 == e32[0]] = 0
        b[(v32 < e32[0]) | (v32 > e32[-1])] = -1
        return b
    b1, b2, bp = vbin(vg.e1, P["vperp1"]), vbin(vg.e2, P["vperp2"]), vbin(vg.epar, P["vpar"])
    ok = (cell >= 0) & (b1 >= 0) & (b2 >= 0) & (bp >= 0)
    idx = ((cell * vg.n1 + b1) * vg.n2 + b2) * vg.npar + bp
    Hh = np.bincount(idx[ok], minlength=len(qGL) * vg.n1 * vg.n2 * vg.npar)
    assert Hh.sum() > 10000
    np.testing.assert_array_equal(H, Hh)


def test_moments_all_equals_each_selector():
    """kaos_get_moments_all (every selector in one copy) equals
    kaos_get_moments selector by selector, ion and ENA moments alike."""
    from kaos_b200.model_input import KAOS_NMOMENTS
    mi, spec, tube, vg = grids.config_small(n_particles=3000, three_d=True,
                                            steps_per_master=3, collisions=True)
    s = Solver(mi, [tube], vg)
    s.load(0, *grids.initial_particles(tube, spec, mi, seed=19))
    s.step(7)
    A = s.moments_all()
    assert A.shape == (KAOS_NMOMENTS, tube.nq)
    assert np.max(A[KAOS_M0]) > 0
    for m in range(KAOS_NMOMENTS):
        np.testing.assert_array_equal(A[m], s.moments(m), err_msg=str(m))
    with pytest.raises(ValueError):
        s.moments_all(out=np.zeros((3, tube.nq)))
    s.close()
