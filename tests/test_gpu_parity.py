"""Parity of the CUDA path against the CPU oracle on identical seeded
initial particles.  Tolerances: FP64 trajectories
1e-12 relative (norm-wise over the particle set), per-cell integer counts
bit-exact, moments 1e-10 relative; mixed precision: moments 1e-6 relative
to the FP64 oracle's scale (stated per moment)."""
import numpy as np
import pytest

from kaos_b200 import build as kbuild
from kaos_b200 import grids
from kaos_b200.lib import Solver
from kaos_b200.model_input import (KAOS_M0, KAOS_M1PAR, KAOS_M1PERP,
                                   KAOS_M1PERP1, KAOS_M1PERP2, KAOS_M2,
                                   KAOS_M2PAR, KAOS_M2PERP, KAOS_M2PERP1,
                                   KAOS_M2PERP2, KAOS_NQ, KAOS_EAMAG,
                                   KAOS_M0FILT, KAOS_PREC_MIXED)
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

TRAJ_TOL = 1e-12
MOM_TOL = 1e-10


@pytest.fixture(scope="module", autouse=True)
def _build():
    kbuild.build()


def run_pair(mi, spec, tube, vg, steps, seed=3, export=False, at_centre=False):
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=seed,
                                              at_centre=at_centre)
    o = Oracle(mi, tube, vg)
    o.load(q, vpar, v1, v2)
    s = Solver(mi, [tube], vg)
    s.load(0, q, vpar, v1, v2)
    if export:
        s.set_export(True)
    o.step(steps)
    s.step(steps)
    return o, s


def rel_norm(a, b):
    scale = max(np.max(np.abs(b)), 1e-300)
    return np.max(np.abs(a - b)) / scale


def moment_list(three_d):
    base = [KAOS_NQ, KAOS_M0, KAOS_M1PAR, KAOS_M2, KAOS_M2PAR, KAOS_EAMAG,
            KAOS_M0FILT]
    if three_d:
        return base + [KAOS_M1PERP1, KAOS_M1PERP2, KAOS_M2PERP1, KAOS_M2PERP2]
    return base + [KAOS_M1PERP, KAOS_M2PERP]


@pytest.mark.parametrize("three_d", [True, False])
def test_fp64_trajectories_counts_moments(three_d):
    mi, spec, tube, vg = grids.config_small(n_particles=3000, three_d=three_d,
                                            steps_per_master=5)
    tube.nsnormCLB = 25.0
    steps = 23  # crosses four master steps (n = 5, 10, 15, 20)
    o, s = run_pair(mi, spec, tube, vg, steps)
    po, ps = o.particles(), s.particles()
    assert len(po["q"]) == len(ps["q"])
    for k in ("rho", "z", "vpar", "vperp1", "vperp2"):
        assert rel_norm(ps[k], po[k]) < TRAJ_TOL, k
    assert rel_norm(ps["q"], po["q"]) < TRAJ_TOL
    np.testing.assert_array_equal(s.counts(), o.counts())
    np.testing.assert_array_equal(ps["qind"], po["qind"])
    for m in moment_list(three_d):
        a, b = s.moments(m), o.moments(m)
        assert rel_norm(a, b) < MOM_TOL, (m, rel_norm(a, b))
    np.testing.assert_array_equal(s.boundary(), o.boundary())


def test_fp64_full_histogram_bit_exact():
    mi, spec, tube, vg = grids.config_small(n_particles=3000, three_d=True,
                                            steps_per_master=4)
    o, s = run_pair(mi, spec, tube, vg, 8, export=True)
    np.testing.assert_array_equal(s.counts(full=True), o.counts(full=True))


def test_fp64_heating_same_random_stream():
    mi, spec, tube, vg = grids.config_small(n_particles=2000, three_d=True,
                                            steps_per_master=5, heating=True)
    o, s = run_pair(mi, spec, tube, vg, 12)
    po, ps = o.particles(), s.particles()
    for k in ("vperp1", "vperp2", "vpar", "z"):
        assert rel_norm(ps[k], po[k]) < TRAJ_TOL, k
    assert np.max(np.abs(po["vperp1"])) > 0


@pytest.mark.parametrize("tight", [False, True])
def test_fp64_escape_and_injection_order(tight):
    """Ions leaving through both boundaries are removed in order and new
    ions appended at the LB cell centre (stable pack + injection).  The
    library marks escaped ions dead at each master step and packs the arrays
    only every few master steps, or when the tube's capacity could not take
    the next injection (tight: capacity = initial ions + 70, so the occupied
    slots are read back and packing is forced); the oracle packs at every
    master step.  Escape counts per master step, the ions in order and the
    counts agree."""
    mi, spec, tube, vg = grids.config_escaping()
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=23)
    if tight:
        tube.capacity = len(q) + 70
    o = Oracle(mi, tube, vg)
    o.load(q, vpar, v1, v2)
    s = Solver(mi, [tube], vg)
    s.load(0, q, vpar, v1, v2)
    escaped = 0
    for _ in range(11):  # 22 steps, 11 master steps
        o.step(2)
        s.step(2)
        bo = o.boundary()
        np.testing.assert_array_equal(s.boundary(), bo)
        assert s.count() == o.count()
        escaped += bo[0] + bo[1]
    assert escaped > 200
    po, ps = o.particles(), s.particles()
    for k in ("z", "vpar", "vperp1", "vperp2"):
        assert rel_norm(ps[k], po[k]) < TRAJ_TOL, k
    np.testing.assert_array_equal(ps["qind"], po["qind"])
    np.testing.assert_array_equal(s.counts(), o.counts())
    for m in (KAOS_M0, KAOS_M2PAR):
        assert rel_norm(s.moments(m), o.moments(m)) < MOM_TOL, m


ALL_ION_MOMENTS = [KAOS_M0, KAOS_M1PERP1, KAOS_M1PERP2, KAOS_M1PAR, KAOS_M2,
                   KAOS_M2PERP1, KAOS_M2PERP2, KAOS_M2PAR, KAOS_NQ, KAOS_EAMAG,
                   KAOS_M0FILT]
MIXED_MOM_TOL = 1e-6  # every moment within 1e-6 of the FP64 oracle's scale


@pytest.mark.parametrize("heat", [False, True])
def test_mixed_precision_every_moment_vs_oracle(heat):
    """Mixed path (FP32 arithmetic on FP64 state) against the FP64 oracle on
    the precision A/B geometry (L = 4, 256 cells, 48x48x64 grid) with 2e4
    ions, collisions on, heating off and on, three master steps: every
    moment selector within 1e-6 of the oracle's scale, state within the
    FP32 increments' precision."""
    mi, spec, tube, vg = grids.config_c2(n_particles=20000, heating=heat,
                                         collisions=True, precision=KAOS_PREC_MIXED,
                                         ndatfac=10)
    o, s = run_pair(mi, spec, tube, vg, 31)
    assert s.count() == o.count()
    po, ps = o.particles(), s.particles()
    assert rel_norm(ps["vpar"], po["vpar"]) < 1e-6
    assert rel_norm(ps["q"], po["q"]) < 1e-9
    np.testing.assert_array_equal(s.counts(), o.counts())
    for m in ALL_ION_MOMENTS:
        err = rel_norm(s.moments(m), o.moments(m))
        assert err < MIXED_MOM_TOL, (m, err)


def test_mixed_kick64_heating_matches_fp64():
    """KAOS_PREC_MIXED_K64 -- the mixed path with the WaveHeatingSub kick in
    FP64 (the FP64 path's formula and Philox draw on the FP64 state) --
    against the FP64 oracle on the precision A/B geometry, 2e4 ions, heating
    and collisions on, three master steps: Vperp within 1e-9 (measured
    5e-11: the kick's inputs differ from the oracle's only by the mixed
    path's position and V|| rounding) and a thousand times closer than with
    the FP32 kick of KAOS_PREC_MIXED (measured 2e-6), counts bit-exact,
    every moment within 1e-6."""
    from kaos_b200.model_input import KAOS_PREC_MIXED_K64
    import dataclasses
    mi, spec, tube, vg = grids.config_c2(n_particles=20000, heating=True,
                                         collisions=True, precision=KAOS_PREC_MIXED_K64,
                                         ndatfac=10)
    o, s = run_pair(mi, spec, tube, vg, 31)
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=3)
    f = Solver(dataclasses.replace(mi, precision=KAOS_PREC_MIXED), [tube], vg)
    f.load(0, q, vpar, v1, v2)
    f.step(31)
    assert s.count() == o.count() == f.count()
    po, ps, pf = o.particles(), s.particles(), f.particles()
    e64 = max(rel_norm(ps[k], po[k]) for k in ("vperp1", "vperp2"))
    e32 = max(rel_norm(pf[k], po[k]) for k in ("vperp1", "vperp2"))
    assert e64 < 1e-9 and e64 < 1e-3 * e32, (e64, e32)
    assert rel_norm(ps["vpar"], po["vpar"]) < 1e-6
    np.testing.assert_array_equal(s.counts(), o.counts())
    for m in ALL_ION_MOMENTS:
        err = rel_norm(s.moments(m), o.moments(m))
        assert err < MIXED_MOM_TOL, (m, err)
    f.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed", "k64"])
def test_heated_2d_grid_every_precision(prec):
    """Wave heating on a 2D (V||, |Vperp|) velocity grid, where an ion whose
    speed leaves the grid keeps its previous bins, in every precision mode
    against the oracle (23 steps, four master steps, charge exchange on):
    FP64 states 1e-12, counts and escapes exact, moments 1e-10;
    KAOS_PREC_MIXED_K64 Vperp 1e-9, counts exact, moments 1e-6; the FP32
    kick of KAOS_PREC_MIXED moments 1e-6."""
    from kaos_b200.model_input import KAOS_PREC_MIXED_K64
    mi, spec, tube, vg = grids.config_small(n_particles=4000, three_d=False,
                                            steps_per_master=5, heating=True,
                                            collisions=True)
    if prec != "fp64":
        mi.precision = KAOS_PREC_MIXED if prec == "mixed" else KAOS_PREC_MIXED_K64
    o, s = run_pair(mi, spec, tube, vg, 23, seed=13)
    assert s.count() == o.count()
    po, ps = o.particles(), s.particles()
    if prec == "fp64":
        for k in ("z", "rho", "vpar", "vperp1", "vperp2"):
            assert rel_norm(ps[k], po[k]) < TRAJ_TOL, k
    elif prec == "k64":
        for k in ("vperp1", "vperp2"):
            assert rel_norm(ps[k], po[k]) < 1e-9, (k, rel_norm(ps[k], po[k]))
    if prec != "mixed":
        np.testing.assert_array_equal(s.counts(), o.counts())
    tol = MOM_TOL if prec == "fp64" else MIXED_MOM_TOL
    for m in moment_list(False):
        err = rel_norm(s.moments(m), o.moments(m))
        assert err < tol, (m, err)


ENA_MOMENTS = list(range(15, 24))  # KAOS_ENA_NQ .. KAOS_ENA_M2PHI


def test_ena_statistics_match_oracle():
    """ENA counts by start-of-step cell and (Vp, Vq, Vphi) bins and the ENA
    moments (ZerothENAMoment .. SecondPHIENAMoment) on a separate ENA grid,
    FP64 path against the oracle."""
    from kaos_b200.grids import make_vgrid
    mi, spec, tube, vg = grids.config_small(n_particles=3000, three_d=True,
                                            steps_per_master=3, collisions=True)
    evg = make_vgrid(True, 12, 20, 18, 7e3)
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=3)
    o = Oracle(mi, tube, vg)
    o.set_ena_grid(evg)
    o.load(q, vpar, v1, v2)
    s = Solver(mi, [tube], vg)
    s.set_ena_grid(evg)
    s.load(0, q, vpar, v1, v2)
    o.step(16)
    s.step(16)  # master steps at 3, 6, ..., 15
    assert s.count() == o.count()
    assert np.max(o.moments(16)) > 0  # ENAs were binned
    for m in ENA_MOMENTS:
        a, b = s.moments(m), o.moments(m)
        assert rel_norm(a, b) < MOM_TOL, (m, rel_norm(a, b))


@pytest.mark.parametrize("mixed", [False, True])
def test_charge_exchange_and_ena_push(mixed):
    """Ion -> ENA conversion of the first N ions per cell in index order
    (Poisson N from the model-A collision frequency) and the ballistic ENA
    push: same ions converted, same ENA trajectories (FP64 to 1e-12)."""
    mi, spec, tube, vg = grids.config_small(n_particles=3000, three_d=True,
                                            steps_per_master=4, collisions=True)
    if mixed:
        mi.precision = KAOS_PREC_MIXED
    o, s = run_pair(mi, spec, tube, vg, 14)
    ni_o, ne_o = o.count()
    ni_s, ne_s = s.count()
    assert ne_o > 5
    if mixed:
        # FP64 state: the same bins, hence the same moments, Poisson means,
        # collision counts and converted ions; the ENA states come from the
        # FP32 q of the k4 point
        assert (ni_s, ne_s) == (ni_o, ne_o)
        np.testing.assert_array_equal(s.moments(14), o.moments(14))  # nuPoi
        return
    assert (ni_s, ne_s) == (ni_o, ne_o)
    np.testing.assert_array_equal(s.moments(14), o.moments(14))  # nuPoi
    # the oracle keeps ENAs in place among the ions (index order); the
    # library appends them per step (step, then index order): match by z
    eo, es = o.enas(), s.enas()
    io, is_ = np.argsort(eo["z"]), np.argsort(es["z"])
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        a, b = es[k][is_], eo[k][io]
        scale = max(np.max(np.abs(eo["z"])) if k in "xyz" else np.max(np.abs(eo["vz"])), 1.0)
        assert np.max(np.abs(a - b)) / scale < TRAJ_TOL, k


@pytest.mark.parametrize("mixed", [False, True])
def test_charge_exchange_idle_then_active(mixed):
    """A thin exosphere: the master steps at 1 and 4 list no converting cell
    and leave no ENA, so steps 2-8 run idle (no selection, conversion or ENA
    push; no Qindk1 or k4 stores at the ordinary steps); the master steps
    still count Qindk1 into cleared rows, and the Poisson draw at 8 lists
    two cells: conversions start at step 9.  The converted ions, the ENA
    states and every count match the oracle, which selects at every step."""
    from kaos_b200.grids import TubeSpec, make_tube, make_vgrid
    from kaos_b200.model_input import ModelInput
    mi = ModelInput(h=0.01, ndatfac=4, ION2VPERPflag=1, QEXCHANGEflag=1, ICRflag=1)
    if mixed:
        mi.precision = KAOS_PREC_MIXED
    vg = make_vgrid(True, 16, 16, 24, 8e3)
    sp = TubeSpec(L=4.0, nq=32, n_particles=3000, q_ub=0.15, H=600e3, neut_n0=3e16,
                  neut_H=300e3, heat_rate_eV_s=200.0)
    tube = make_tube(sp, mi)
    init = grids.initial_particles(tube, sp, mi, seed=9)
    o = Oracle(mi, tube, vg)
    o.load(*init)
    s = Solver(mi, [tube], vg)
    s.load(0, *init)
    seen = []
    for _ in range(6):  # master steps at 4, 8, ..., 24
        o.step(4)
        s.step(4)
        assert s.count() == o.count()
        np.testing.assert_array_equal(s.moments(14), o.moments(14))  # nuPoi
        seen.append(o.count()[1])
    assert seen[:2] == [0, 0] and seen[-1] > 0  # idle first, converting later
    if mixed:
        return
    eo, es = o.enas(), s.enas()
    io, is_ = np.argsort(eo["z"]), np.argsort(es["z"])
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        a, b = es[k][is_], eo[k][io]
        scale = max(np.max(np.abs(eo["z"])) if k in "xyz" else np.max(np.abs(eo["vz"])), 1.0)
        assert np.max(np.abs(a - b)) / scale < TRAJ_TOL, k


@pytest.mark.parametrize("mixed", [False, True])
def test_charge_exchange_many_tubes(mixed):
    """300 small tubes with a dense exosphere in one solver: most cells
    convert ions every step (several per cell: the ranked selection), the
    scan and conversion kernels work on many tubes at once, and the ENA
    push builds its per-tube unit prefix over more tubes than it has
    threads (two tubes a thread).  Each tube matches its own oracle run:
    the ion and ENA counts and the Poisson means exactly, the ENA states to
    1e-12 (FP64 path)."""
    from kaos_b200.grids import TubeSpec, make_tube, make_vgrid
    from kaos_b200.model_input import ModelInput
    mi = ModelInput(h=0.01, ndatfac=4, ION2VPERPflag=1, QEXCHANGEflag=1)
    if mixed:
        mi.precision = KAOS_PREC_MIXED
    vg = make_vgrid(True, 16, 16, 24, 8e3)
    nt = 300
    specs = [TubeSpec(L=3.0 + 3.0 * k / nt, nq=16, n_particles=300, q_ub=0.15,
                      H=600e3, neut_n0=3e18, neut_H=300e3) for k in range(nt)]
    tubes = [make_tube(sp, mi) for sp in specs]
    s = Solver(mi, tubes, vg)
    inits = []
    for k, (sp, t) in enumerate(zip(specs, tubes)):
        init = grids.initial_particles(t, sp, mi, seed=500 + k)
        inits.append(init)
        s.load(k, *init)
    s.step(10)
    total_enas = 0
    for k, (sp, t) in enumerate(zip(specs, tubes)):
        o = Oracle(mi, t, vg)
        o.load(*inits[k])
        o.step(10)
        assert s.count(k) == o.count(), k
        np.testing.assert_array_equal(s.moments(14, k), o.moments(14))  # nuPoi
        total_enas += o.count()[1]
        if mixed:
            continue
        eo, es = o.enas(), s.enas(k)
        io, is_ = np.argsort(eo["z"]), np.argsort(es["z"])
        for key in ("x", "y", "z", "vx", "vy", "vz"):
            a, b = es[key][is_], eo[key][io]
            scale = max(np.max(np.abs(eo["z"])) if key in "xyz" else np.max(np.abs(eo["vz"])), 1.0)
            assert np.max(np.abs(a - b)) / scale < TRAJ_TOL, (k, key)
    assert total_enas > 100 * nt


def test_batched_uneven_tubes_one_launch():
    """Several tubes of different L-shell, cell count and particle count
    advance together (one launch per kernel over a (tube, chunk) map); each
    tube matches its own oracle run."""
    from kaos_b200.grids import TubeSpec, make_tube, make_vgrid
    from kaos_b200.model_input import ModelInput
    mi = ModelInput(h=0.01, ndatfac=4, ION2VPERPflag=1, ICRflag=1)
    vg = make_vgrid(True, 16, 16, 24, 8e3)
    specs = [TubeSpec(L=3.0, nq=24, n_particles=1500, q_ub=0.2, H=500e3, heat_rate_eV_s=5.0),
             TubeSpec(L=5.0, nq=40, n_particles=2500, q_ub=0.1, H=700e3, heat_rate_eV_s=1.0),
             TubeSpec(L=7.0, nq=12, n_particles=700, q_ub=0.05, H=900e3, heat_rate_eV_s=0.0)]
    tubes = [make_tube(sp, mi) for sp in specs]
    for t in tubes:
        t.nsnormCLB = 15.0
    s = Solver(mi, tubes, vg)
    inits = []
    for k, (sp, t) in enumerate(zip(specs, tubes)):
        init = grids.initial_particles(t, sp, mi, seed=100 + k)
        inits.append(init)
        s.load(k, *init)
    s.step(10)
    for k, (sp, t) in enumerate(zip(specs, tubes)):
        o = Oracle(mi, t, vg)
        o.load(*inits[k])
        o.step(10)
        po, ps = o.particles(), s.particles(k)
        assert len(po["q"]) == len(ps["q"]), k
        for key in ("z", "vpar", "vperp1"):
            assert rel_norm(ps[key], po[key]) < TRAJ_TOL, (k, key)
        np.testing.assert_array_equal(s.counts(k), o.counts())
        a, b = s.moments(KAOS_M0, k), o.moments(KAOS_M0)
        assert rel_norm(a, b) < MOM_TOL, k


def test_two_species_as_separate_entries():
    """H+ and O+ of one flux tube as two entries of one batched solver (the
    reference runs species as independent outer loops, each with its own
    ambipolar field): each matches its own oracle run in FP64, with wave
    heating and charge exchange on."""
    from kaos_b200.grids import TubeSpec, make_tube, make_vgrid
    from kaos_b200.model_input import MH, MO, ModelInput
    mi = ModelInput(h=0.01, ndatfac=4, ION2VPERPflag=1, ICRflag=1, QEXCHANGEflag=1)
    vg = make_vgrid(True, 16, 16, 24, 3e4)
    common = dict(L=4.0, nq=24, q_ub=0.15, H=600e3, heat_rate_eV_s=5.0,
                  neut_n0=3e18, neut_H=300e3)
    specs = [TubeSpec(n_particles=800, ms=MH, **common),
             TubeSpec(n_particles=3200, ms=MO, **common)]
    tubes = [make_tube(sp, mi) for sp in specs]
    s = Solver(mi, tubes, vg)
    inits = []
    for k, (sp, t) in enumerate(zip(specs, tubes)):
        inits.append(grids.initial_particles(t, sp, mi, seed=40 + k))
        s.load(k, *inits[k])
    s.step(10)
    for k, (sp, t) in enumerate(zip(specs, tubes)):
        o = Oracle(mi, t, vg)
        o.load(*inits[k])
        o.step(10)
        assert s.count(k) == o.count(), k
        po, ps = o.particles(), s.particles(k)
        for key in ("z", "vpar", "vperp1", "vperp2"):
            assert rel_norm(ps[key], po[key]) < TRAJ_TOL, (k, key)
        np.testing.assert_array_equal(s.counts(k), o.counts())
        for m in moment_list(True):
            assert rel_norm(s.moments(m, k), o.moments(m)) < MOM_TOL, (k, m)
    # the species differ: lighter ions are faster
    assert np.std(s.particles(0)["vpar"]) > 2 * np.std(s.particles(1)["vpar"])


@pytest.mark.parametrize("mixed", [False, True])
def test_device_initial_ions_match_oracle(mixed):
    """kaos_init_particles draws the same initial ions as the oracle's
    generator (Maxwellian core plus a kappa = 3 tail), and the runs started
    from them agree (FP64: 1e-12 after 9 steps with heating and charge
    exchange)."""
    mi, spec, tube, vg = grids.config_small(n_particles=5000, three_d=True,
                                            steps_per_master=4, heating=True,
                                            collisions=True)
    if mixed:
        mi.precision = KAOS_PREC_MIXED
    T_tail = 5.0 * 1.602e-19 / 138e-25
    kw = dict(tail_fraction=0.1, kappa=3.0, tail_T=T_tail, seed=99)
    o = Oracle(mi, tube, vg)
    o.init(tube._counts, **kw)
    s = Solver(mi, [tube], vg)
    s.init_particles(0, tube._counts, **kw)
    po, ps = o.particles(), s.particles()
    tol = 1e-6 if mixed else 1e-13
    for k in ("q", "vpar", "vperp1", "vperp2"):
        assert rel_norm(ps[k], po[k]) < tol, k
    np.testing.assert_array_equal(ps["qind"], po["qind"])
    if mixed:
        return
    o.step(9)
    s.step(9)
    assert s.count() == o.count()
    po, ps = o.particles(), s.particles()
    for k in ("z", "vpar", "vperp1", "vperp2"):
        assert rel_norm(ps[k], po[k]) < TRAJ_TOL, k
    np.testing.assert_array_equal(s.counts(), o.counts())


@pytest.mark.parametrize("flux,static", [(1, 0), (0, 1)])
def test_injection_variants(flux, static):
    """Flux-weighted injection (extension) and STATICINJECTIONflag at both
    boundaries match the oracle (FP64, 1e-12; counts exact)."""
    mi, spec, tube, vg = grids.config_small(n_particles=3000, three_d=True,
                                            steps_per_master=3)
    mi.FLUXINJECTIONflag, mi.STATICINJECTIONflag, mi.UBCONDITIONflag = flux, static, 1
    tube.nsnormCLB, tube.nsnormCUB = 40.0, 15.0
    o, s = run_pair(mi, spec, tube, vg, 13)
    assert o.count() == s.count()
    np.testing.assert_array_equal(s.boundary(), o.boundary())
    po, ps = o.particles(), s.particles()
    for k in ("z", "vpar", "vperp1", "vperp2"):
        assert rel_norm(ps[k], po[k]) < TRAJ_TOL, k
    np.testing.assert_array_equal(s.counts(), o.counts())


@pytest.mark.parametrize("mixed", [False, True])
def test_convection_to_new_lshell(mixed):
    """A tube moved to a new L-shell (ConvectionSub, applied first at the
    next master step: q and V|| kept, magnetic moment kept) matches the
    oracle: FP64 1e-12 / exact counts / moments 1e-10; mixed within its
    precision."""
    from kaos_b200.grids import moved_tube
    mi, spec, tube, vg = grids.config_small(n_particles=3000, three_d=True,
                                            steps_per_master=3, heating=True)
    if mixed:
        mi.precision = KAOS_PREC_MIXED
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=8)
    o = Oracle(mi, tube, vg)
    o.load(q, vpar, v1, v2)
    s = Solver(mi, [tube], vg)
    s.load(0, q, vpar, v1, v2)
    o.step(4)
    s.step(4)
    new = moved_tube(spec, mi, tube, 4.05)
    o.update_tube(new)
    s.update_tube(0, new)
    o.step(7)  # the move at n = 6, another master step at n = 9
    s.step(7)
    assert o.count() == s.count()
    po, ps = o.particles(), s.particles()
    if mixed:
        assert rel_norm(ps["vperp1"], po["vperp1"]) < 1e-4
        assert rel_norm(ps["z"], po["z"]) < 1e-6
        return
    for k in ("z", "rho", "vpar", "vperp1", "vperp2"):
        assert rel_norm(ps[k], po[k]) < TRAJ_TOL, k
    np.testing.assert_array_equal(s.counts(), o.counts())
    for m in (KAOS_M0, KAOS_M2, KAOS_M2PAR, KAOS_EAMAG):
        assert rel_norm(s.moments(m), o.moments(m)) < MOM_TOL, m


def test_ena_escapes_per_master_step():
    """Escaped LB/UB ENA counts of every master step (kaos_get_boundary_ena)
    equal the oracle's, with ions and ENAs leaving through both ends."""
    mi, spec, tube, vg = grids.config_escaping(neut_n0=3e16)
    tube.nsnormCLB = 30.0
    q, vpar, v1, v2 = grids.initial_particles(tube, spec, mi, seed=3)
    o = Oracle(mi, tube, vg)
    o.load(q, vpar, v1, v2)
    s = Solver(mi, [tube], vg)
    s.load(0, q, vpar, v1, v2)
    o.step(1)
    s.step(1)
    tot = np.zeros(2, dtype=np.int64)
    for _ in range(10):
        o.step(2)
        s.step(2)
        np.testing.assert_array_equal(s.boundary(), o.boundary())
        be = o.boundary_ena()
        np.testing.assert_array_equal(s.boundary_ena(), be)
        assert s.count() == o.count()
        tot += be
    assert tot[0] > 20 and tot[1] > 20
    po, ps = o.particles(), s.particles()
    for k in ("z", "vpar", "vperp1", "vperp2"):
        assert rel_norm(ps[k], po[k]) < TRAJ_TOL, k


def test_fp64_charge_exchange_across_packing():
    """Charge exchange every step over ten master steps (slots converted to
    ENAs and escaped ions both marked dead, the arrays packed at the eighth
    master step): ions, ENA count, counts and moments equal the oracle's."""
    mi, spec, tube, vg = grids.config_small(n_particles=4000, three_d=True,
                                            steps_per_master=2, collisions=True)
    tube.nsnormCLB = 12.0
    o, s = run_pair(mi, spec, tube, vg, 21)
    assert s.count() == o.count()
    assert o.count()[1] > 10
    po, ps = o.particles(), s.particles()
    for k in ("z", "vpar", "vperp1", "vperp2"):
        assert rel_norm(ps[k], po[k]) < TRAJ_TOL, k
    np.testing.assert_array_equal(ps["qind"], po["qind"])
    np.testing.assert_array_equal(s.counts(), o.counts())
    for m in (KAOS_M0, KAOS_M2PAR):
        assert rel_norm(s.moments(m), o.moments(m)) < MOM_TOL, m
