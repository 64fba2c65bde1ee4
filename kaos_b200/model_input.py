"""Run parameters of the kinetic particle loop, mirroring KAOS's
``_ModelInput.f90`` / ``FluxTubeT`` flag fields, and the ctypes mirrors of
the C-ABI structs declared in ``include/kaos_gpu.h``.

Names keep the reference spelling (``ICRflag``, ``EAMBSIGNflag``, ...) so a
KAOS user finds the same switches.  Defaults are the reference defaults
(_ModelInput.f90:54-158) except where noted.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional

import numpy as np

# ---- physical constants, _ModelInput.f90:35-43 and :173-174 ----------------
PI = 4.0 * np.arctan(1.0)
KB = 138e-25          # Boltzmann constant
EPSILON0 = 8.854e-12
MDIP = 8.06e15        # Earth magnetic moment "m" [T m^3]
GG = 667e-13          # gravitational constant
ME = 598e22           # Earth mass
RE = 638e4            # Earth radius [m]
MO = 16.0 * 1.66054e-27   # O+ mass [kg]
QO = 1.602e-19            # O+ charge [C]
MH = 1.0 * 1.66054e-27    # H+ / H mass [kg]

KAOS_PREC_FP64 = 0
KAOS_PREC_MIXED = 1
KAOS_PREC_MIXED_K64 = 2  # mixed push, heating kick in FP64

(KAOS_M0, KAOS_M1PERP1, KAOS_M1PERP2, KAOS_M1PAR, KAOS_M2, KAOS_M2PERP1,
 KAOS_M2PERP2, KAOS_M2PAR, KAOS_M1PERP, KAOS_M2PERP, KAOS_NQ, KAOS_EAMAG,
 KAOS_EGMAG, KAOS_M0FILT, KAOS_NUPOI) = range(15)
# ENA statistics (ENAParticleCounts, ZerothENAMoment .. SecondPHIENAMoment)
(KAOS_ENA_NQ, KAOS_ENA_M0, KAOS_ENA_M1P, KAOS_ENA_M1Q, KAOS_ENA_M1PHI,
 KAOS_ENA_M2, KAOS_ENA_M2P, KAOS_ENA_M2Q, KAOS_ENA_M2PHI) = range(15, 24)
KAOS_NMOMENTS = 24
MOMENT_NAMES = ["M0", "M1Perp1", "M1Perp2", "M1Par", "M2", "M2Perp1",
                "M2Perp2", "M2Par", "M1Perp", "M2Perp", "Nq", "EAmag",
                "EGmag", "M0Filt", "nuPoi"]

_DP = C.POINTER(C.c_double)


class KaosParams(C.Structure):
    """ctypes mirror of ``kaos_params_c``."""
    _fields_ = [
        ("ms", C.c_double), ("qs", C.c_double), ("h", C.c_double),
        ("mNeut", C.c_double), ("TNeut", C.c_double), ("dNTe", C.c_double),
        ("dNTeEND", C.c_double), ("seed", C.c_uint64),
        ("ndatfac", C.c_int32), ("precision", C.c_int32),
        ("ION2VPERPflag", C.c_int32), ("ICRflag", C.c_int32),
        ("ICRCOHERENCEflag", C.c_int32), ("MIRRORflag", C.c_int32),
        ("GRAVflag", C.c_int32), ("EAMBflag", C.c_int32),
        ("EAMBSIGNflag", C.c_int32), ("EAMBSELFCONSISTflag", C.c_int32),
        ("EAPRESSUREflag", C.c_int32), ("MOMENTFILTERflag", C.c_int32),
        ("QEXCHANGEflag", C.c_int32), ("LBCONDITIONflag", C.c_int32),
        ("UBCONDITIONflag", C.c_int32), ("STATICINJECTIONflag", C.c_int32),
        ("PHASEENERGYPARIONMOMENTCENTERflag", C.c_int32),
        ("PHASEENERGYPERPIONMOMENTCENTERflag", C.c_int32),
        ("M0MAfilterPt", C.c_int32), ("M1ParMAfilterPt", C.c_int32),
        ("M1Perp1MAfilterPt", C.c_int32), ("M1Perp2MAfilterPt", C.c_int32),
        ("M2ParMAfilterPt", C.c_int32), ("FLUXINJECTIONflag", C.c_int32),
        ("reserved", C.c_int32 * 3),
    ]


class KaosTube(C.Structure):
    """ctypes mirror of ``kaos_tube_c``."""
    _fields_ = [
        ("nq", C.c_int32), ("capacity", C.c_int32), ("pG", C.c_double),
        ("phiG", C.c_double), ("nsnormfac", C.c_double),
        ("nsnormCLB", C.c_double), ("nsnormCUB", C.c_double),
        ("sumdsICR", C.c_double),
        ("qGL", _DP), ("qGH", _DP), ("qGC", _DP), ("hqC", _DP), ("dqC", _DP),
        ("d3xC", _DP), ("rGC", _DP), ("thetaGC", _DP), ("ellGC", _DP),
        ("TeG", _DP), ("TsG", _DP), ("nsnormCNeut", _DP),
        ("lambdaPerp", _DP), ("EtaLH", _DP), ("XiPerp1", _DP),
        ("XiPerp2", _DP), ("S0", _DP), ("OmegaG0", _DP), ("ChiPerp1", _DP),
        ("ChiPerp2", _DP), ("ms", C.c_double), ("qs", C.c_double),
    ]


class KaosInit(C.Structure):
    """ctypes mirror of ``kaos_init_c``."""
    _fields_ = [("counts", C.POINTER(C.c_int64)), ("tail_fraction", C.c_double),
                ("kappa", C.c_double), ("tail_T", C.c_double), ("seed", C.c_uint64)]


class KaosVGrid(C.Structure):
    """ctypes mirror of ``kaos_vgrid_c``."""
    _fields_ = [("n1", C.c_int32), ("n2", C.c_int32), ("npar", C.c_int32),
                ("e1", _DP), ("e2", _DP), ("epar", _DP)]


@dataclasses.dataclass
class ModelInput:
    """Parameter surface of _ModelInput.f90 used by the per-step loop."""
    ms: float = MO
    qs: float = QO
    h: float = 0.01
    mNeut: float = MO
    TNeut: float = 848.0
    dNTe: float = 0.0
    dNTeEND: float = 3e10
    seed: int = 20261203
    ndatfac: int = 50
    precision: int = KAOS_PREC_FP64
    ION2VPERPflag: int = 1
    ICRflag: int = 0
    ICRCOHERENCEflag: int = 0
    MIRRORflag: int = 1
    GRAVflag: int = 1
    EAMBflag: int = 1
    EAMBSIGNflag: int = 1
    EAMBSELFCONSISTflag: int = 1
    EAPRESSUREflag: int = 1
    MOMENTFILTERflag: int = 1
    QEXCHANGEflag: int = 0
    LBCONDITIONflag: int = 1
    UBCONDITIONflag: int = 0
    STATICINJECTIONflag: int = 0
    PHASEENERGYPARIONMOMENTCENTERflag: int = 1
    PHASEENERGYPERPIONMOMENTCENTERflag: int = 0
    M0MAfilterPt: int = 11
    M1ParMAfilterPt: int = 11
    M1Perp1MAfilterPt: int = 11
    M1Perp2MAfilterPt: int = 11
    M2ParMAfilterPt: int = 11
    FLUXINJECTIONflag: int = 0    # extension: flux-weighted V|| at injection

    def to_c(self) -> KaosParams:
        p = KaosParams()
        for f in dataclasses.fields(self):
            setattr(p, f.name, getattr(self, f.name))
        return p


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return _DP()
    return a.ctypes.data_as(_DP)


@dataclasses.dataclass
class Tube:
    """Per-cell grid tables of one flux tube (FluxTubeT, 0-based cells)."""
    nq: int
    pG: float
    phiG: float
    nsnormfac: float
    nsnormCLB: float
    nsnormCUB: float
    qGL: np.ndarray
    qGH: np.ndarray
    qGC: np.ndarray
    hqC: np.ndarray
    dqC: np.ndarray
    d3xC: np.ndarray
    rGC: np.ndarray
    thetaGC: np.ndarray
    ellGC: np.ndarray
    TeG: np.ndarray
    TsG: np.ndarray
    nsnormCNeut: np.ndarray
    lambdaPerp: np.ndarray
    EtaLH: np.ndarray
    XiPerp1: np.ndarray
    XiPerp2: np.ndarray
    S0: np.ndarray
    OmegaG0: np.ndarray
    ChiPerp1: np.ndarray
    ChiPerp2: np.ndarray
    sumdsICR: float = 1.0
    capacity: int = 0
    ms: float = 0.0   # species of this entry; 0 = ModelInput.ms / qs
    qs: float = 0.0

    def to_c(self) -> KaosTube:
        t = KaosTube()
        t.nq = self.nq
        t.capacity = self.capacity
        for k in ("pG", "phiG", "nsnormfac", "nsnormCLB", "nsnormCUB",
                  "sumdsICR", "ms", "qs"):
            setattr(t, k, float(getattr(self, k)))
        for k in ("qGL", "qGH", "qGC", "hqC", "dqC", "d3xC", "rGC",
                  "thetaGC", "ellGC", "TeG", "TsG", "nsnormCNeut",
                  "lambdaPerp", "EtaLH", "XiPerp1", "XiPerp2", "S0",
                  "OmegaG0", "ChiPerp1", "ChiPerp2"):
            a = np.ascontiguousarray(getattr(self, k), dtype=np.float64)
            setattr(self, k, a)
            setattr(t, k, _ptr(a))
        return t


@dataclasses.dataclass
class VGrid:
    """Separable velocity grid: edges per axis (n+1 values each)."""
    e1: np.ndarray
    epar: np.ndarray
    e2: Optional[np.ndarray] = None

    @property
    def n1(self):
        return len(self.e1) - 1

    @property
    def n2(self):
        return 0 if self.e2 is None else len(self.e2) - 1

    @property
    def npar(self):
        return len(self.epar) - 1

    def nbins(self, three_d: bool) -> int:
        return self.n1 * self.n2 * self.npar if three_d else self.n1 * self.npar

    def to_c(self) -> KaosVGrid:
        g = KaosVGrid()
        self.e1 = np.ascontiguousarray(self.e1, dtype=np.float64)
        self.epar = np.ascontiguousarray(self.epar, dtype=np.float64)
        if self.e2 is not None:
            self.e2 = np.ascontiguousarray(self.e2, dtype=np.float64)
        g.n1, g.n2, g.npar = self.n1, self.n2, self.npar
        g.e1, g.e2, g.epar = _ptr(self.e1), _ptr(self.e2), _ptr(self.epar)
        return g
