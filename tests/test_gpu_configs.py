"""Parity on the benchmark configurations, beyond the small test tube.

* The plain FP64 configuration in full: L = 4 from 1000 km to |q| = 1e-3,
  128 cells, 2D grid 64 x 32 up to 30 km/s, 1e5 O+, gravity + mirror +
  ambipolar field, dt 0.01 s, 200 steps (ten master steps): FP64 states
  within 1e-12 of the oracle, the full phase-space histogram bit-exact (the
  library is built with FMA contraction; no bin edge flips), moments within
  1e-10.  The same run on the mixed path: every moment within 1e-6.
* The near-equator end of that tube, where the quartic of
  RK4DipolePolynomialSolverSub (_8_1_4_RK4DipolePolynomialSolver.f90:30-84)
  is worst conditioned: ions between |q| = 1e-3 and 0.05, FP64 within 1e-12.
"""
import dataclasses

import numpy as np
import pytest

from kaos_b200 import build as kbuild
from kaos_b200 import grids
from kaos_b200.lib import Solver
from kaos_b200.model_input import (KAOS_EAMAG, KAOS_M0, KAOS_M0FILT, KAOS_M1PAR,
                                   KAOS_M1PERP, KAOS_M2, KAOS_M2PAR, KAOS_M2PERP,
                                   KAOS_NQ, KAOS_PREC_MIXED, KB)
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
TRAJ_TOL, MOM_TOL, MIXED_MOM_TOL = 1e-12, 1e-10, 1e-6
MOMENTS_2D = [KAOS_M0, KAOS_M1PAR, KAOS_M1PERP, KAOS_M2, KAOS_M2PAR, KAOS_M2PERP,
              KAOS_NQ, KAOS_EAMAG, KAOS_M0FILT]


@pytest.fixture(scope="module", autouse=True)
def _build():
    kbuild.build()


def rel_norm(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.fixture(scope="module")
def c1_oracle():
    mi, spec, tube, vg = grids.config_c1(n_particles=100_000)
    init = grids.initial_particles(tube, spec, mi, seed=20261203)
    o = Oracle(mi, tube, vg)
    o.load(*init)
    o.step(200)
    return mi, tube, vg, init, o


def test_c1_fp64_full_run(c1_oracle):
    mi, tube, vg, init, o = c1_oracle
    s = Solver(mi, [tube], vg)
    s.set_export(True)
    s.load(0, *init)
    s.step(200)
    assert s.count() == o.count()
    po, ps = o.particles(), s.particles()
    for k in ("rho", "z", "q", "vpar", "vperp1", "vperp2"):
        assert rel_norm(ps[k], po[k]) < TRAJ_TOL, k
    np.testing.assert_array_equal(ps["qind"], po["qind"])
    np.testing.assert_array_equal(s.counts(full=True), o.counts(full=True))
    for m in MOMENTS_2D:
        assert rel_norm(s.moments(m), o.moments(m)) < MOM_TOL, m
    np.testing.assert_array_equal(s.boundary(), o.boundary())


def test_c1_mixed_full_run(c1_oracle):
    mi, tube, vg, init, o = c1_oracle
    mi = dataclasses.replace(mi, precision=KAOS_PREC_MIXED)
    s = Solver(mi, [tube], vg)
    s.load(0, *init)
    s.step(200)
    assert s.count() == o.count()
    for m in MOMENTS_2D:
        err = rel_norm(s.moments(m), o.moments(m))
        assert err < MIXED_MOM_TOL, (m, err)


def test_near_equator_quartic_fp64():
    """Ions between |q| = 1.2e-3 and 0.05.  The trajectories there are ill
    conditioned: a 1e-15 relative change of the initial q alone moves z by
    ~2.5e-12 of its scale after 30 steps.  The tolerance is scaled by that
    measured sensitivity (ten times the oracle's own change under the
    perturbation, at least 1e-12)."""
    mi, spec, tube, vg = grids.config_c1(n_particles=100_000)
    rng = np.random.default_rng(5)
    n = 20000
    q = 10 ** rng.uniform(np.log10(1.2e-3), np.log10(0.05), n)
    sig = np.sqrt(KB * tube.TsG[-1] / mi.ms)
    v = rng.normal(size=(3, n)) * sig
    runs = []
    for eps in (0.0, 1e-15):
        o = Oracle(mi, tube, vg)
        o.load(q * (1.0 + eps), v[0], v[1], v[2])
        o.step(30)
        runs.append(o)
    o, op = runs
    s = Solver(mi, [tube], vg)
    s.load(0, q, v[0], v[1], v[2])
    s.step(30)
    assert s.count() == o.count()
    po, pp, ps = o.particles(), op.particles(), s.particles()
    assert np.min(np.abs(po["q"])) < 2e-3
    for k in ("rho", "z", "q", "vpar"):
        tol = max(TRAJ_TOL, 10.0 * rel_norm(pp[k], po[k]))
        assert rel_norm(ps[k], po[k]) < tol, (k, rel_norm(ps[k], po[k]), tol)
    co = o.counts()
    assert np.abs(s.counts() - co).sum() <= np.abs(op.counts() - co).sum()
