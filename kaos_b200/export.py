"""Master-step output in the reference's DataExport2 layout.

DataExport2Sub (_8_0_2_DataExport2.f90:29-800) writes one Fortran
`access='stream'` file per quantity per master step, named
`<nn>_<s>_<f>_<Name>fort.bin` (per-cell quantities `<nn>_<s>_<f>_<Qind>_<Name>
fort.bin`), holding the raw little-endian values with no record markers:
real(dp) -> float64, integer(dp) -> int64, multi-dimensional arrays in
Fortran column-major order.  Indices nn, s, f, Qind are 1-based as in the
reference (Qind = NqLB + k with NqLB = 1).  The MATLAB / matplotlib readers
of the reference consume these files.
"""
from __future__ import annotations

import os
from typing import Dict, Optional

import numpy as np

from .model_input import (KAOS_EAMAG, KAOS_EGMAG, KAOS_M0, KAOS_M0FILT,
                          KAOS_M1PAR, KAOS_M1PERP, KAOS_M1PERP1, KAOS_M1PERP2,
                          KAOS_M2, KAOS_M2PAR, KAOS_M2PERP, KAOS_M2PERP1,
                          KAOS_M2PERP2, KAOS_NUPOI)


def _w(path: str, arr, dtype) -> None:
    a = np.asarray(arr, dtype=dtype)
    with open(path, "wb") as f:
        f.write(np.asfortranarray(a).tobytes(order="F"))


def moment_filter(x, pt: int) -> np.ndarray:
    """MomentFilterSub (_8_7_1_MomentFilter.f90:25-147) on the host: the
    mean of the H = nint((pt-1)/2) cells above (with the cell itself) and
    of the H below, averaged; one-sided near the ends.  Sums run in the
    reference's order, so the result is the library's bit for bit."""
    a = [float(v) for v in np.asarray(x, dtype=np.float64)]
    nq = len(a)
    H = int(np.floor((pt - 1) / 2.0 + 0.5))
    lb, ub = 0, nq - 1
    out = np.zeros(nq)

    def run(start, step, count):   # a[start] + a[start+step] + ... in order
        s = a[start]
        for k in range(1, count):
            s += a[start + k * step]
        return s

    for q in range(nq):
        if q <= lb - 1 + H:
            a1 = run(q, 1, H + 1) / (H + 1)
            if q == lb:
                out[q] = a1
            elif q == lb + 1:
                out[q] = (a1 + a[lb]) / 2.0
            else:
                out[q] = (a1 + run(q - 1, -1, q - lb) / (q - lb)) / 2.0
        if lb - 1 + H < q < ub - H:
            out[q] = (run(q, 1, H + 1) / (H + 1) + run(q - 1, -1, H) / H) / 2.0
        if q >= ub - H:
            a2 = run(q, -1, H + 1) / (H + 1)
            if q == ub:
                out[q] = a2
            elif q == ub - 1:
                out[q] = (a[ub] + a2) / 2.0
            else:
                out[q] = (run(q + 1, 1, ub - q) / (ub - q) + a2) / 2.0
    return out


def sigma_ion_neutral(M0, M2par) -> np.ndarray:
    """Lindsay-Stebbings charge-exchange factor per cell,
    (4.07 - 0.269 ln E)^2 (1 - exp(-415/E))^0.8 with E = M2par in keV
    (sigmaIonNeutRT, _8_6_6_1_IonNeutralCollisionFrequencyA.f90:104-127;
    the cross-section is this times 1e-16 cm^2); 0 where M0 or M2par is 0."""
    import math
    out = np.zeros(len(M0))
    for q, (m0, m2) in enumerate(zip(np.asarray(M0, float), np.asarray(M2par, float))):
        if m0 != 0.0 and m2 != 0.0:
            e = (6.242e18) * (1e-3) * float(m2)
            out[q] = (4.07 - 0.269 * math.log(e)) ** 2 * (1.0 - math.exp(-415.0 / e)) ** 0.8
    return out


def file_name(nn: int, s: int, f: int, name: str, qind: Optional[int] = None) -> str:
    if qind is None:
        return f"{nn}_{s}_{f}_{name}fort.bin"
    return f"{nn}_{s}_{f}_{qind}_{name}fort.bin"


def write_master_step(outdir: str, nn: int, solver, tube_index: int, tube,
                      vgrid, three_d: bool, time_s: float, ndatfac: int,
                      s: int = 1, f: int = 1, hist: Optional[np.ndarray] = None,
                      Te: Optional[np.ndarray] = None, mi=None,
                      ns0: Optional[float] = None) -> Dict[str, str]:
    """Write the DataExport2 files of master step `nn` for one tube from a
    `kaos_b200.lib.Solver` (or anything with .moments(which, tube)).
    `hist` is the full count histogram of the step ([nq][...] as returned by
    counts(full=True)); when given, N2PerpphRT (3D) or NphRT (2D) and d3vCTp
    are written per cell, in density units (count * nsnormfac / d3x) as
    IonParticleCountsSub stores them (_8_3_1_IonParticleCounts.f90:440-451).
    With `mi` (the run's ModelInput) and MOMENTFILTERflag = 1, the filtered
    first and parallel second moments the collision model reads
    (_8_6_6_1_IonNeutralCollisionFrequencyA.f90:42-95) are written too
    (M1ParFiltAvrgRT, M1Perp1/2FiltAvrgRT, M2ParFiltAvrgRT,
    _8_0_2_DataExport2.f90:359-410), and with QEXCHANGEflag = 1 the
    charge-exchange factor sigmaIonNeutRT (:416-430).  `ns0`, the run's
    reference ion density at the lower boundary [m^-3], is written as ns0GT
    (:54-58) when given.  Returns {name: path}."""
    os.makedirs(outdir, exist_ok=True)
    out: Dict[str, str] = {}
    nq = tube.nq

    def put(name, arr, dtype=np.float64, qind=None):
        p = os.path.join(outdir, file_name(nn, s, f, name, qind))
        _w(p, arr, dtype)
        out[name if qind is None else f"{qind}_{name}"] = p

    put("TimeT", [time_s])
    put("ndatfacGT", [ndatfac], np.int64)
    if ns0 is not None:
        put("ns0GT", [ns0])
    put("qGCGT", tube.qGC)
    put("pGCGT", np.full(nq, tube.pG))
    put("rGCGT", tube.rGC)
    put("phiGCGT", np.full(nq, tube.phiG))
    put("thetaGCGT", tube.thetaGC)
    put("d3xCGT", tube.d3xC)
    put("TsGT", tube.TsG)
    m = lambda k: solver.moments(k, tube_index)
    put("M0phRT", m(KAOS_M0))
    if three_d:
        put("M1Perp1phRT", m(KAOS_M1PERP1))
        put("M1Perp2phRT", m(KAOS_M1PERP2))
    else:
        put("M1PerpphRT", m(KAOS_M1PERP))
    put("M1ParphRT", m(KAOS_M1PAR))
    put("M0FiltAvrgRT", m(KAOS_M0FILT))
    if mi is not None and mi.MOMENTFILTERflag == 1:
        if three_d:
            put("M1Perp1FiltAvrgRT", moment_filter(m(KAOS_M1PERP1), mi.M1Perp1MAfilterPt))
            put("M1Perp2FiltAvrgRT", moment_filter(m(KAOS_M1PERP2), mi.M1Perp2MAfilterPt))
        put("M1ParFiltAvrgRT", moment_filter(m(KAOS_M1PAR), mi.M1ParMAfilterPt))
        put("M2ParFiltAvrgRT", moment_filter(m(KAOS_M2PAR), mi.M2ParMAfilterPt))
    if mi is not None and mi.QEXCHANGEflag == 1:
        m2 = (moment_filter(m(KAOS_M2PAR), mi.M2ParMAfilterPt)
              if mi.MOMENTFILTERflag == 1 else m(KAOS_M2PAR))
        put("sigmaIonNeutRT", sigma_ion_neutral(m(KAOS_M0), m2))
    put("nuIonNeutRT", m(KAOS_NUPOI))
    put("M2phRT", m(KAOS_M2))
    if three_d:
        put("M2Perp1phRT", m(KAOS_M2PERP1))
        put("M2Perp2phRT", m(KAOS_M2PERP2))
    else:
        put("M2PerpphRT", m(KAOS_M2PERP))
    put("M2ParphRT", m(KAOS_M2PAR))
    ea = m(KAOS_EAMAG)
    put("EAInertialRT", np.zeros(nq))  # EAINERTIALflag = 0
    put("EAPressureRT", ea)
    put("EAmagRT", ea)
    put("EGmagRT", m(KAOS_EGMAG))
    put("EPmagRT", np.zeros(nq))       # EPARflag = 0
    put("PhiParRT", np.zeros(nq))
    put("NqLBT", [1], np.int64)
    put("NqUBT", [nq], np.int64)
    Te = tube.TeG if Te is None else Te
    e1, epar = np.asarray(vgrid.e1), np.asarray(vgrid.epar)
    d1, dp = np.abs(np.diff(e1)), np.abs(np.diff(epar))
    if three_d:
        e2 = np.asarray(vgrid.e2)
        d2 = np.abs(np.diff(e2))
        d3v = d1[:, None, None] * d2[None, :, None] * dp[None, None, :]
    else:
        c1 = 0.5 * (e1[:-1] + e1[1:])
        d3v = np.abs(c1)[:, None] * d1[:, None] * dp[None, :] * (2.0 * np.pi)
    d3v = np.where(d3v == 0.0, 1e-9, d3v)
    for k in range(nq):
        q = k + 1
        put("TeNT", [Te[k]], qind=q)
        if hist is not None:
            h = np.asarray(hist).reshape(nq, *d3v.shape)[k]
            dens = h * (tube.nsnormfac / tube.d3xC[k])
            put("N2PerpphRT" if three_d else "NphRT", dens, qind=q)
            put("d3vCTp", d3v, qind=q)
    return out


def read(path: str, dtype=np.float64, shape=None) -> np.ndarray:
    """Read one stream file back (Fortran order when a shape is given)."""
    a = np.fromfile(path, dtype=dtype)
    return a if shape is None else a.reshape(shape, order="F")
