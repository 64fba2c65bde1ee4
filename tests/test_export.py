"""DataExport2 layout: file names, raw stream contents, Fortran order of the
phase-space arrays (_8_0_2_DataExport2.f90:29-800).  The CPU oracle stands in
for the solver (same .moments / .counts surface)."""
import os

import numpy as np
import pytest

from kaos_b200 import export, grids
from kaos_b200.model_input import KAOS_M0, KAOS_M1PAR
from oracle.oracle import Oracle


class _OracleAsSolver:
    def __init__(self, o):
        self.o = o

    def moments(self, k, tube=0):
        return self.o.moments(k)


def test_export_layout_roundtrip(tmp_path):
    mi, spec, tube, vg = grids.config_small(n_particles=1500, three_d=True, nq=12)
    o = Oracle(mi, tube, vg)
    o.load(*grids.initial_particles(tube, spec, mi, seed=4))
    o.step(1)
    hist = o.counts(full=True)
    files = export.write_master_step(str(tmp_path), 1, _OracleAsSolver(o), 0, tube, vg,
                                     True, 0.0, mi.ndatfac, hist=hist, ns0=spec.n0)
    assert export.read(files["ns0GT"])[0] == spec.n0
    assert os.path.basename(files["M0phRT"]) == "1_1_1_M0phRTfort.bin"
    assert os.path.basename(files["3_TeNT"]) == "1_1_1_3_TeNTfort.bin"
    np.testing.assert_array_equal(export.read(files["M0phRT"]), o.moments(KAOS_M0))
    np.testing.assert_array_equal(export.read(files["M1ParphRT"]), o.moments(KAOS_M1PAR))
    assert export.read(files["ndatfacGT"], np.int64)[0] == mi.ndatfac
    # N2PerpphRT(Vperp1, Vperp2, Vpar) in column-major order, density units
    n1, n2, npar = vg.n1, vg.n2, vg.npar
    k = 2
    N = export.read(files[f"{k + 1}_N2PerpphRT"], shape=(n1, n2, npar))
    ref = hist.reshape(tube.nq, n1, n2, npar)[k] * tube.nsnormfac / tube.d3xC[k]
    np.testing.assert_allclose(N, ref, rtol=1e-15)
    assert os.path.getsize(files[f"{k + 1}_d3vCTp"]) == 8 * n1 * n2 * npar


@pytest.mark.parametrize("nq,pt", [(12, 11), (16, 5), (40, 11), (7, 3), (12, 7)])
def test_host_moment_filter_is_the_oracles(nq, pt):
    """MomentFilterSub restated on the host equals the oracle's filter bit
    for bit (same summation order), interior and one-sided ends."""
    from oracle.oracle import moment_filter as orc_filter
    x = np.random.default_rng(nq * 100 + pt).lognormal(size=nq) * 1e9
    np.testing.assert_array_equal(export.moment_filter(x, pt), orc_filter(x, pt))


def test_filtered_moment_files(tmp_path):
    from kaos_b200.model_input import KAOS_M0FILT, KAOS_M1PERP1, KAOS_M2PAR
    mi, spec, tube, vg = grids.config_small(n_particles=1500, three_d=True, nq=12)
    o = Oracle(mi, tube, vg)
    o.load(*grids.initial_particles(tube, spec, mi, seed=4))
    o.step(1)
    files = export.write_master_step(str(tmp_path), 1, _OracleAsSolver(o), 0, tube, vg,
                                     True, 0.0, mi.ndatfac, mi=mi)
    for n in ("M1ParFiltAvrgRT", "M1Perp1FiltAvrgRT", "M1Perp2FiltAvrgRT",
              "M2ParFiltAvrgRT"):
        assert os.path.basename(files[n]) == f"1_1_1_{n}fort.bin"
    np.testing.assert_array_equal(export.read(files["M2ParFiltAvrgRT"]),
                                  export.moment_filter(o.moments(KAOS_M2PAR),
                                                       mi.M2ParMAfilterPt))
    np.testing.assert_array_equal(export.read(files["M1Perp1FiltAvrgRT"]),
                                  export.moment_filter(o.moments(KAOS_M1PERP1),
                                                       mi.M1Perp1MAfilterPt))
    # the library's own filtered M0 is the same filter
    np.testing.assert_array_equal(export.moment_filter(o.moments(KAOS_M0), mi.M0MAfilterPt),
                                  o.moments(KAOS_M0FILT))


def test_sigma_file_with_charge_exchange(tmp_path):
    from kaos_b200.model_input import KAOS_M2PAR
    mi, spec, tube, vg = grids.config_small(n_particles=1500, three_d=True, nq=12,
                                            collisions=True)
    o = Oracle(mi, tube, vg)
    o.load(*grids.initial_particles(tube, spec, mi, seed=4))
    o.step(1)
    files = export.write_master_step(str(tmp_path), 1, _OracleAsSolver(o), 0, tube, vg,
                                     True, 0.0, mi.ndatfac, mi=mi)
    sig = export.read(files["sigmaIonNeutRT"])
    m0 = o.moments(KAOS_M0)
    m2 = export.moment_filter(o.moments(KAOS_M2PAR), mi.M2ParMAfilterPt)
    assert sig.shape == (tube.nq,)
    for q in range(tube.nq):
        if m0[q] == 0.0 or m2[q] == 0.0:
            assert sig[q] == 0.0
        else:
            e = 6.242e18 * 1e-3 * m2[q]    # keV
            assert sig[q] == pytest.approx((4.07 - 0.269 * np.log(e)) ** 2
                                           * (1.0 - np.exp(-415.0 / e)) ** 0.8, rel=1e-14)
    assert np.all(sig[m0 > 0] > 0)
