"""Spin-up hand-over (_8_0_2_DataExport2.f90:706-800 writes,
_1_SimParameterization.f90:811-960 reads): file names and contents, the
import's initial counts and temperature, the imported first-step field.
The CPU oracle stands in for the solver (same .moments surface and the same
initial-ion generator and field import as the library)."""
import os

import numpy as np
import pytest

from kaos_b200 import grids, spinup
from kaos_b200.model_input import (KAOS_EAMAG, KAOS_M0, KAOS_M2PAR,
                                   KAOS_M2PERP1, KAOS_M2PERP2, KB)
from oracle.oracle import Oracle


class _OracleAsSolver:
    def __init__(self, o):
        self.o = o

    def moments(self, k, tube=0):
        return self.o.moments(k)


def _spun(tmp_path, nq=12, steps=6):
    mi, spec, tube, vg = grids.config_small(n_particles=6000, three_d=True, nq=nq,
                                            steps_per_master=5)
    o = Oracle(mi, tube, vg)
    o.load(*grids.initial_particles(tube, spec, mi, seed=11))
    o.step(steps)   # the master step of n = 5 is the last
    files = spinup.write_spinup(str(tmp_path), _OracleAsSolver(o), 0, tube, True)
    return mi, spec, tube, vg, o, files


def test_files_and_contents(tmp_path):
    mi, spec, tube, vg, o, files = _spun(tmp_path)
    names = spinup.FLOAT_ARRAYS + spinup.FLOAT_SCALARS + spinup.INT_SCALARS
    assert sorted(files) == sorted(names)
    for n in names:
        p = files[n]
        assert os.path.basename(p) == f"1_1_{n}fort.bin"
        assert os.path.getsize(p) == 8 * (tube.nq if n in spinup.FLOAT_ARRAYS else 1)
    sp = spinup.read_spinup(str(tmp_path), tube.nq)
    assert (sp.nq_lb, sp.nq_ub) == (1, tube.nq)
    np.testing.assert_array_equal(sp.density, o.moments(KAOS_M0))
    e = o.moments(KAOS_M2PAR) + o.moments(KAOS_M2PERP1) + o.moments(KAOS_M2PERP2)
    np.testing.assert_array_equal(sp.temperature, (2.0 / 3.0) * e / KB)
    np.testing.assert_array_equal(sp.eamag, o.moments(KAOS_EAMAG))
    np.testing.assert_array_equal(sp.ea_pressure, sp.eamag)
    assert not sp.ea_inertial.any()
    assert sp.nsnorm_clb == tube.nsnormCLB and sp.nsnorm_cub == tube.nsnormCUB
    assert (sp.lb_replenish, sp.ub_replenish) == (1, 0)


def test_import_counts_are_the_binned_ions(tmp_path):
    """density = count * nsnormfac / d3x, so the import's initial ions per
    cell are the exporting step's binned ions, exactly."""
    mi, spec, tube, vg, o, files = _spun(tmp_path)
    sp = spinup.read_spinup(str(tmp_path), tube.nq)
    hist = o.counts(full=True).reshape(tube.nq, -1)
    np.testing.assert_array_equal(spinup.cell_counts(tube, sp), hist.sum(axis=1))


def test_next_run_starts_from_the_imported_state(tmp_path):
    mi, spec, tube, vg, o, files = _spun(tmp_path)
    sp = spinup.read_spinup(str(tmp_path), tube.nq, lb_replenish=1, ub_replenish=0)
    t2 = spinup.spun_up_tube(tube, sp)
    counts = spinup.cell_counts(t2, sp)
    o2 = Oracle(mi, t2, vg)
    o2.init(counts, seed=5)
    o2.set_fields(sp.eamag)
    o2.step(1)
    # the first step's field is the imported one
    np.testing.assert_array_equal(o2.moments(KAOS_EAMAG), sp.eamag)
    # the initial ions are drawn at the imported temperature (moments at
    # bin centres add a few per cent of bin-width variance per pass)
    e = o2.moments(KAOS_M2PAR) + o2.moments(KAOS_M2PERP1) + o2.moments(KAOS_M2PERP2)
    T2 = (2.0 / 3.0) * e / KB
    full = counts >= 200
    assert full.sum() >= 4
    rel = np.abs(T2[full] / sp.temperature[full] - 1.0)
    assert np.median(rel) < 0.08


def test_inconsistent_files_are_errors(tmp_path):
    mi, spec, tube, vg, o, files = _spun(tmp_path)
    with pytest.raises(ValueError):
        spinup.read_spinup(str(tmp_path), tube.nq + 1)
    with pytest.raises(ValueError):
        spinup.read_spinup(str(tmp_path), tube.nq, lb_replenish=0)
    with pytest.raises(ValueError):
        spinup.read_spinup(str(tmp_path), tube.nq, ub_replenish=1)
    # a truncated density file
    with open(files["DensityOutputRT"], "r+b") as f:
        f.truncate(8 * (tube.nq - 1))
    with pytest.raises(ValueError):
        spinup.read_spinup(str(tmp_path), tube.nq)


def test_fortran_nint():
    np.testing.assert_array_equal(spinup.nint([0.5, 1.5, 2.5, -0.5, -1.5, 2.49]),
                                  [1, 2, 3, -1, -2, 2])
