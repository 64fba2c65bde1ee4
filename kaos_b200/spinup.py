"""Spin-up hand-over: the state one run leaves for the next.

A run with SPINUPflag = 1 writes, per species s and flux tube f, into the
density data directory at its master steps (DataExport2Sub,
_8_0_2_DataExport2.f90:706-800), eleven Fortran stream files
`<s>_<f>_<Name>fort.bin`:

  NqLBT, NqUBT                     integer(dp): the tube's cell range
  DensityOutputRT                  M0 of the step (_8_6_6_SecondParIonMoment
                                   .f90:666)
  TemperatureOutputRT              (2/3)(M2par + M2perp1 + M2perp2)/kB
                                   (_8_6_6_SecondParIonMoment.f90:667-670)
  EAInertialOutputRT, EAPressureOutputRT, EAmagOutputRT
                                   the ambipolar field's parts
                                   (_8_7_AmbipolarEfield.f90:1410-1420)
  nsnormCLBOutput, nsnormCUBOutput real(dp): boundary injection counts
  LBREPLENISHflagTOutput, UBREPLENISHflagTOutput   integer(dp)

A run with SPINUPflag = 0 reads them back (SimParameterizationSub,
_1_SimParameterization.f90:811-960): the density sets the initial ions per
cell, nint(density / nsnormfac * d3x) (_2_1_DensityProfileA1.f90:53-55),
the temperature their Maxwellian (_6_VelocityDistribution.f90:70-73), the
ambipolar field the first step's field (_8_7_AmbipolarEfield.f90:1375-1402),
and the boundary counts the injection.  Here the import gives a Tube with
the imported temperature and injection counts, the initial counts for
`Solver.init_particles`, and the field for `Solver.set_fields`.

Values are raw little-endian float64 / int64 with no record markers, as
Fortran writes `access='stream'` files.  On the 2D velocity grid (one
perpendicular axis) the perpendicular energy is the one 2D moment
M2perp, which holds both perpendicular directions.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Dict

import numpy as np

from .model_input import (KAOS_EAMAG, KAOS_M0, KAOS_M2PAR, KAOS_M2PERP,
                          KAOS_M2PERP1, KAOS_M2PERP2, KB, Tube)

FLOAT_ARRAYS = ("DensityOutputRT", "TemperatureOutputRT", "EAInertialOutputRT",
                "EAPressureOutputRT", "EAmagOutputRT")
FLOAT_SCALARS = ("nsnormCLBOutput", "nsnormCUBOutput")
INT_SCALARS = ("NqLBT", "NqUBT", "LBREPLENISHflagTOutput", "UBREPLENISHflagTOutput")


def file_name(s: int, f: int, name: str) -> str:
    return f"{s}_{f}_{name}fort.bin"


@dataclasses.dataclass
class SpinUp:
    """One tube's imported spin-up state (cells 0-based)."""
    nq_lb: int
    nq_ub: int
    density: np.ndarray
    temperature: np.ndarray
    ea_inertial: np.ndarray
    ea_pressure: np.ndarray
    eamag: np.ndarray
    nsnorm_clb: float
    nsnorm_cub: float
    lb_replenish: int
    ub_replenish: int


def write_spinup(datadir: str, solver, tube_index: int, tube: Tube, three_d: bool,
                 s: int = 1, f: int = 1, lb_replenish: int = 1,
                 ub_replenish: int = 0) -> Dict[str, str]:
    """Write the spin-up files of one tube from the latest master step of
    `solver` (a `kaos_b200.lib.Solver`, or anything with
    .moments(which, tube)).  Returns {name: path}."""
    os.makedirs(datadir, exist_ok=True)
    m = lambda k: np.asarray(solver.moments(k, tube_index), dtype=np.float64)
    nq = tube.nq
    if three_d:
        e = m(KAOS_M2PAR) + m(KAOS_M2PERP1) + m(KAOS_M2PERP2)
    else:
        e = m(KAOS_M2PAR) + m(KAOS_M2PERP)
    ea = m(KAOS_EAMAG)
    values = {
        "NqLBT": np.array([1], np.int64),
        "NqUBT": np.array([nq], np.int64),
        "DensityOutputRT": m(KAOS_M0),
        "TemperatureOutputRT": (2.0 / 3.0) * e / KB,
        "EAInertialOutputRT": np.zeros(nq),   # EAINERTIALflag = 0
        "EAPressureOutputRT": ea,             # EAmag = EAInertial + EAPressure
        "EAmagOutputRT": ea,
        "nsnormCLBOutput": np.array([tube.nsnormCLB], np.float64),
        "nsnormCUBOutput": np.array([tube.nsnormCUB], np.float64),
        "LBREPLENISHflagTOutput": np.array([lb_replenish], np.int64),
        "UBREPLENISHflagTOutput": np.array([ub_replenish], np.int64),
    }
    out = {}
    for name, a in values.items():
        p = os.path.join(datadir, file_name(s, f, name))
        with open(p, "wb") as fh:
            fh.write(np.ascontiguousarray(a).tobytes())
        out[name] = p
    return out


def read_spinup(datadir: str, nq: int, s: int = 1, f: int = 1,
                lb_replenish: int = None, ub_replenish: int = None) -> SpinUp:
    """Read one tube's spin-up files.  The cell range must give `nq` cells
    and, when given, the replenish flags must match this run's (the
    reference reports both as errors, _1_SimParameterization.f90:950-961)."""
    def rd(name, dtype, n=None):
        p = os.path.join(datadir, file_name(s, f, name))
        a = np.fromfile(p, dtype=dtype)
        if n is not None and a.size != n:
            raise ValueError(f"{p}: {a.size} values, expected {n}")
        return a

    lb, ub = int(rd("NqLBT", np.int64, 1)[0]), int(rd("NqUBT", np.int64, 1)[0])
    if ub - lb + 1 != nq:
        raise ValueError(f"spin-up cell range {lb}..{ub} does not give {nq} cells")
    sp = SpinUp(
        nq_lb=lb, nq_ub=ub,
        density=rd("DensityOutputRT", np.float64, nq),
        temperature=rd("TemperatureOutputRT", np.float64, nq),
        ea_inertial=rd("EAInertialOutputRT", np.float64, nq),
        ea_pressure=rd("EAPressureOutputRT", np.float64, nq),
        eamag=rd("EAmagOutputRT", np.float64, nq),
        nsnorm_clb=float(rd("nsnormCLBOutput", np.float64, 1)[0]),
        nsnorm_cub=float(rd("nsnormCUBOutput", np.float64, 1)[0]),
        lb_replenish=int(rd("LBREPLENISHflagTOutput", np.int64, 1)[0]),
        ub_replenish=int(rd("UBREPLENISHflagTOutput", np.int64, 1)[0]))
    if lb_replenish is not None and sp.lb_replenish != lb_replenish:
        raise ValueError("inconsistent LBREPLENISHflag in the spin-up files")
    if ub_replenish is not None and sp.ub_replenish != ub_replenish:
        raise ValueError("inconsistent UBREPLENISHflag in the spin-up files")
    return sp


def nint(x) -> np.ndarray:
    """Fortran NINT: nearest integer, halves away from zero."""
    x = np.asarray(x, dtype=np.float64)
    return (np.sign(x) * np.floor(np.abs(x) + 0.5)).astype(np.int64)


def cell_counts(tube: Tube, sp: SpinUp) -> np.ndarray:
    """Initial ions per cell from the imported density,
    nint((density / nsnormfac) * d3x) (_2_1_DensityProfileA1.f90:53-55)."""
    return nint((sp.density / tube.nsnormfac) * np.asarray(tube.d3xC))


def spun_up_tube(tube: Tube, sp: SpinUp) -> Tube:
    """`tube` with the imported ion temperature (the initial Maxwellian's,
    _6_VelocityDistribution.f90:70-73) and boundary injection counts."""
    if sp.density.size != tube.nq:
        raise ValueError("spin-up state is for another cell count")
    return dataclasses.replace(tube, TsG=np.array(sp.temperature, dtype=np.float64),
                               nsnormCLB=sp.nsnorm_clb, nsnormCUB=sp.nsnorm_cub)
