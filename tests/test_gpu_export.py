"""DataExport2 files written from the CUDA path (_8_0_2_DataExport2.f90:
29-800, read by KAOS_Data_Plots.py): a run of the library and of the oracle
on the same ions, with heating and charge exchange on, each exported at the
first step and at two later master steps.  Every file the oracle's export
writes is written from the library under the same name and size; the
files of tables, counts and phase-space densities (count * nsnormfac / d3x)
are byte-for-byte equal; the moment and field files agree within 1e-10 (the
library sums the moment integrals in a different order -- from per-axis
marginals -- so their last bits differ, as the reference's own -Ofast build
does from one compiler to the next).
"""
import os

import numpy as np
import pytest

from kaos_b200 import build as kbuild
from kaos_b200 import export, grids
from kaos_b200.lib import Solver
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

MOMENT_FILES = {"M0phRT", "M1Perp1phRT", "M1Perp2phRT", "M1ParphRT", "M0FiltAvrgRT",
                "M1Perp1FiltAvrgRT", "M1Perp2FiltAvrgRT", "M1ParFiltAvrgRT",
                "M2ParFiltAvrgRT", "sigmaIonNeutRT", "nuIonNeutRT", "M2phRT",
                "M2Perp1phRT", "M2Perp2phRT", "M2ParphRT", "EAPressureRT", "EAmagRT",
                "EGmagRT"}


class _OracleAsSolver:
    def __init__(self, o):
        self.o = o

    def moments(self, k, tube=0):
        return self.o.moments(k)


@pytest.mark.parametrize("mixed", [False, True])
def test_export_from_gpu_matches_oracle(tmp_path, mixed):
    kbuild.build()
    mi, spec, tube, vg = grids.config_small(n_particles=3000, three_d=True,
                                            steps_per_master=5, heating=True,
                                            collisions=True)
    if mixed:
        from kaos_b200.model_input import KAOS_PREC_MIXED
        mi.precision = KAOS_PREC_MIXED
    init = grids.initial_particles(tube, spec, mi, seed=12)
    o = Oracle(mi, tube, vg)
    o.load(*init)
    s = Solver(mi, [tube], vg)
    s.set_export(True)
    s.load(0, *init)
    done = 0
    for nn, upto in ((1, 1), (2, 5), (3, 10)):
        o.step(upto - done)
        s.step(upto - done)
        done = upto
        t = (upto - 1) * mi.h
        dg, do = str(tmp_path / f"gpu{nn}"), str(tmp_path / f"orc{nn}")
        fg = export.write_master_step(dg, nn, s, 0, tube, vg, True, t, mi.ndatfac,
                                      hist=s.counts(full=True), mi=mi, ns0=spec.n0)
        fo = export.write_master_step(do, nn, _OracleAsSolver(o), 0, tube, vg, True, t,
                                      mi.ndatfac, hist=o.counts(full=True), mi=mi,
                                      ns0=spec.n0)
        assert sorted(os.listdir(dg)) == sorted(os.listdir(do))
        assert fg.keys() == fo.keys()
        nbytes = 0
        for key in fo:
            a, b = open(fg[key], "rb").read(), open(fo[key], "rb").read()
            assert len(a) == len(b), key
            name = key.split("_", 1)[-1] if key[0].isdigit() else key
            if name in MOMENT_FILES:
                x, y = np.frombuffer(a), np.frombuffer(b)
                scale = max(np.max(np.abs(y)), 1e-300)
                assert np.max(np.abs(x - y)) / scale < 1e-10, (nn, key)
            else:
                assert a == b, (nn, key)
                nbytes += len(a)
        assert nbytes > 0
        # the phase-space densities are not all zero
        n2 = [k for k in fo if k.endswith("_N2PerpphRT")]
        assert n2 and max(np.max(export.read(fo[k])) for k in n2) > 0
