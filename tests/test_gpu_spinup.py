"""The spin-up hand-over between runs through the CUDA path
(_8_0_2_DataExport2.f90:706-800 writes, _1_SimParameterization.f90:811-960
reads), against the oracle on the same seeded ions: the eleven
<s>_<f>_<Name>fort.bin files written from a library run equal the oracle's
(integer and table-copied files byte-equal, moment-derived arrays within
1e-10), and the next run -- its ions drawn on the device from the imported
counts and temperature, its first-step field the imported one -- matches
the oracle's next run from the same files (states 1e-12, counts bit-exact,
the first step's EAmag equal to the import)."""
import numpy as np
import pytest

from kaos_b200 import build as kbuild
from kaos_b200 import grids, spinup
from kaos_b200.lib import Solver
from kaos_b200.model_input import KAOS_EAMAG, KAOS_M0, KAOS_M2PAR
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _build():
    kbuild.build()


class _OracleAsSolver:
    def __init__(self, o):
        self.o = o

    def moments(self, k, tube=0):
        return self.o.moments(k)


def rel_norm(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


EXACT = set(spinup.INT_SCALARS) | {"nsnormCLBOutput", "nsnormCUBOutput",
                                    "EAInertialOutputRT"}


def test_spinup_cycle_through_the_library(tmp_path):
    mi, spec, tube, vg = grids.config_small(n_particles=6000, three_d=True, nq=12,
                                            steps_per_master=5)
    init = grids.initial_particles(tube, spec, mi, seed=11)
    o = Oracle(mi, tube, vg)
    o.load(*init)
    o.step(6)  # the master step of n = 5 is the last
    s = Solver(mi, [tube], vg)
    s.load(0, *init)
    s.step(6)
    fo = spinup.write_spinup(str(tmp_path / "oracle"), _OracleAsSolver(o), 0, tube, True)
    fs = spinup.write_spinup(str(tmp_path / "gpu"), s, 0, tube, True)
    assert sorted(fs) == sorted(fo)
    for name in fo:
        dt = np.int64 if name in spinup.INT_SCALARS else np.float64
        a, b = np.fromfile(fo[name], dtype=dt), np.fromfile(fs[name], dtype=dt)
        assert a.shape == b.shape, name
        if name in EXACT:
            np.testing.assert_array_equal(b, a, err_msg=name)
        else:
            assert rel_norm(b, a) < 1e-10, (name, rel_norm(b, a))
    s.close()

    # the next run from the library's files, on the device and on the oracle
    sp = spinup.read_spinup(str(tmp_path / "gpu"), tube.nq, lb_replenish=1, ub_replenish=0)
    t2 = spinup.spun_up_tube(tube, sp)
    counts = spinup.cell_counts(t2, sp)
    assert counts.sum() > 1000
    s2 = Solver(mi, [t2], vg)
    s2.init_particles(0, counts, seed=5)
    s2.set_fields(0, sp.eamag)
    s2.step(1)
    o2 = Oracle(mi, t2, vg)
    o2.init(counts, seed=5)
    o2.set_fields(sp.eamag)
    o2.step(1)
    np.testing.assert_array_equal(s2.moments(KAOS_EAMAG), sp.eamag)
    assert s2.count() == o2.count()
    p2s, p2o = s2.particles(), o2.particles()
    for k in ("rho", "z", "vpar", "vperp1", "vperp2"):
        assert rel_norm(p2s[k], p2o[k]) < 1e-12, k
    np.testing.assert_array_equal(s2.counts(), o2.counts())
    for m in (KAOS_M0, KAOS_M2PAR):
        assert rel_norm(s2.moments(m), o2.moments(m)) < 1e-10, m
    s2.close()
