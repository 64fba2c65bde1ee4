"""Branches of the loop that the other parity tests leave at their
defaults, each against the oracle on the same seeded ions:

* the electron-temperature ramp of KineticSolverSub (dNTe per master step
  up to dNTeEND, _8_KineticSolver.f90:69-89), which scales the ambipolar
  field;
* the coherent ICR heating branch (ICRCOHERENCEflag = 1,
  _8_1_1_0_WaveHeating.f90:129-302): |Vperp| kicked by a Gaussian, gyro-angle
  redrawn;
* the unsigned ambipolar field (EAMBSIGNflag = 0,
  _8_1_1_KineticUpdateA.f90:656-658): the field magnitude pointed away from
  the Earth in both hemispheres;
* a finite perpendicular wavelength lambdaPerp (_8_1_1_0_WaveHeating.f90:
  91-97): the diffusion coefficient divided by Sig^3 where Sig = 2 pi
  |Vperp| / (lambdaPerp Omega) >= 1 (lambdaPerp = 5 m: most ions, not all).

FP64 path: states within 1e-12, counts bit-exact, moments within 1e-10;
mixed path (FP32 kick) and KAOS_PREC_MIXED_K64 (FP64 kick): every moment
within 1e-6, and for K64 with heating on Vperp within 1e-9.  Each case also
checks that the branch changes the run (against the default flag).
"""
import dataclasses

import numpy as np
import pytest

from kaos_b200 import build as kbuild
from kaos_b200 import grids
from kaos_b200.lib import Solver
from kaos_b200.model_input import (KAOS_EAMAG, KAOS_M0, KAOS_M1PAR, KAOS_M1PERP1,
                                   KAOS_M1PERP2, KAOS_M2, KAOS_M2PAR, KAOS_M2PERP1,
                                   KAOS_M2PERP2, KAOS_NQ, KAOS_PREC_MIXED,
                                   KAOS_PREC_MIXED_K64)
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
TRAJ_TOL, MOM_TOL, MIXED_MOM_TOL = 1e-12, 1e-10, 1e-6
MOMENTS = [KAOS_M0, KAOS_M1PAR, KAOS_M1PERP1, KAOS_M1PERP2, KAOS_M2, KAOS_M2PAR,
           KAOS_M2PERP1, KAOS_M2PERP2, KAOS_NQ, KAOS_EAMAG]


@pytest.fixture(scope="module", autouse=True)
def _build():
    kbuild.build()


def rel_norm(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def case(name):
    """ModelInput changes of a branch, and the run length."""
    heating = name in ("coherent", "lambda")
    mi, spec, tube, vg = grids.config_small(n_particles=4000, three_d=True,
                                            steps_per_master=5, heating=heating)
    if name == "lambda":
        tube.lambdaPerp = np.full(tube.nq, 5.0)
    if name == "te_ramp":
        mi.dNTe, mi.dNTeEND = 400.0, 5000.0   # K per master step, cap
    elif name == "coherent":
        mi.ICRCOHERENCEflag = 1
    elif name == "eamb_unsigned":
        mi.EAMBSIGNflag = 0
    return mi, spec, tube, vg


def run(mi, tube, vg, init, steps, gpu):
    r = Solver(mi, [tube], vg) if gpu else Oracle(mi, tube, vg)
    if gpu:
        r.load(0, *init)
    else:
        r.load(*init)
    r.step(steps)
    return r


@pytest.mark.parametrize("prec", ["fp64", "mixed", "k64"])
@pytest.mark.parametrize("name", ["te_ramp", "coherent", "eamb_unsigned", "lambda"])
def test_branch_matches_oracle(name, prec):
    mi, spec, tube, vg = case(name)
    init = grids.initial_particles(tube, spec, mi, seed=31)
    steps = 23  # master steps at 5, 10, 15, 20
    o = run(mi, tube, vg, init, steps, gpu=False)
    mg = mi if prec == "fp64" else dataclasses.replace(
        mi, precision=KAOS_PREC_MIXED if prec == "mixed" else KAOS_PREC_MIXED_K64)
    s = run(mg, tube, vg, init, steps, gpu=True)
    assert s.count() == o.count()
    po, ps = o.particles(), s.particles()
    if prec != "fp64":
        for m in MOMENTS:
            err = rel_norm(s.moments(m), o.moments(m))
            assert err < MIXED_MOM_TOL, (name, m, err)
        if prec == "k64" and mi.ICRflag:
            for k in ("vperp1", "vperp2"):
                assert rel_norm(ps[k], po[k]) < 1e-9, (name, k, rel_norm(ps[k], po[k]))
        return
    for k in ("rho", "z", "vpar", "vperp1", "vperp2"):
        assert rel_norm(ps[k], po[k]) < TRAJ_TOL, (name, k)
    np.testing.assert_array_equal(s.counts(), o.counts())
    for m in MOMENTS:
        assert rel_norm(s.moments(m), o.moments(m)) < MOM_TOL, (name, m)
    # the branch is live: the default flag gives a different run
    base = dataclasses.replace(mi, dNTe=0.0, ICRCOHERENCEflag=0, EAMBSIGNflag=1)
    tb = dataclasses.replace(tube, lambdaPerp=np.zeros(tube.nq))
    b = run(base, tb, vg, init, steps, gpu=True)
    pb = b.particles()
    key = "vperp1" if name in ("coherent", "lambda") else "vpar"
    assert rel_norm(pb[key], ps[key]) > 1e-9, name
