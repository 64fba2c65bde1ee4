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


def file_name(nn: int, s: int, f: int, name: str, qind: Optional[int] = None) -> str:
    if qind is None:
        return f"{nn}_{s}_{f}_{name}fort.bin"
    return f"{nn}_{s}_{f}_{qind}_{name}fort.bin"


def write_master_step(outdir: str, nn: int, solver, tube_index: int, tube,
                      vgrid, three_d: bool, time_s: float, ndatfac: int,
                      s: int = 1, f: int = 1, hist: Optional[np.ndarray] = None,
                      Te: Optional[np.ndarray] = None) -> Dict[str, str]:
    """Write the DataExport2 files of master step `nn` for one tube from a
    `kaos_b200.lib.Solver` (or anything with .moments(which, tube)).
    `hist` is the full count histogram of the step ([nq][...] as returned by
    counts(full=True)); when given, N2PerpphRT (3D) or NphRT (2D) and d3vCTp
    are written per cell, in density units (count * nsnormfac / d3x) as
    IonParticleCountsSub stores them (_8_3_1_IonParticleCounts.f90:440-451).
    Returns {name: path}."""
    os.makedirs(outdir, exist_ok=True)
    out: Dict[str, str] = {}
    nq = tube.nq

    def put(name, arr, dtype=np.float64, qind=None):
        p = os.path.join(outdir, file_name(nn, s, f, name, qind))
        _w(p, arr, dtype)
        out[name if qind is None else f"{qind}_{name}"] = p

    put("TimeT", [time_s])
    put("ndatfacGT", [ndatfac], np.int64)
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
