"""ctypes front of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg;
never by the product path.  Mirrors the call surface of include/kaos_gpu.h
for one tube so parity tests read the same for both sides.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        vp = C.c_void_p
        L.orc_create.restype = vp
        L.orc_create.argtypes = [vp, vp, vp]
        L.orc_load.argtypes = [vp] + [vp] * 4 + [C.c_int64]
        L.orc_set_fields.argtypes = [vp, vp]
        L.orc_set_literal.argtypes = [vp, C.c_int]
        L.orc_set_ena_grid.argtypes = [vp, vp]
        L.orc_update_tube.argtypes = [vp, vp]
        L.orc_convect_now.argtypes = [vp]
        L.orc_init.argtypes = [vp, vp, C.c_double, C.c_double, C.c_double, C.c_uint64]
        L.orc_step.argtypes = [vp, C.c_int64]
        L.orc_count.restype = C.c_int64
        L.orc_count.argtypes = [vp, vp]
        L.orc_get_moments.argtypes = [vp, C.c_int, vp]
        L.orc_get_counts.argtypes = [vp, vp, C.c_int64]
        L.orc_get_particles.argtypes = [vp] + [vp] * 7
        L.orc_get_enas.argtypes = [vp] + [vp] * 6
        L.orc_get_boundary.argtypes = [vp, vp]
        L.orc_quartic.argtypes = [C.c_double, C.c_double, C.c_double, vp]
        L.orc_filter.argtypes = [vp, vp, C.c_int, C.c_int]
        L.orc_destroy.argtypes = [vp]
        L.orc_ambipolar.argtypes = [vp, vp, vp]
        L.orc_force.argtypes = [vp, C.c_double, C.c_double, C.c_double,
                                C.c_double, C.c_double, C.c_double, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


class Oracle:
    """One tube on the CPU oracle."""

    def __init__(self, mi, tube, vg):
        self._mi, self._tube, self._vg = mi.to_c(), tube.to_c(), vg.to_c()
        self._keep = (tube, vg)
        self.nq = tube.nq
        self.three_d = mi.ION2VPERPflag == 1
        self.nbins = vg.nbins(self.three_d)
        self.h = lib().orc_create(C.addressof(self._mi), C.addressof(self._tube),
                                  C.addressof(self._vg))
        if not self.h:
            raise ValueError("oracle: moving-average windows must be odd, >= 3 and "
                             "at most the tube's cell count")

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_destroy(self.h)
            self.h = None

    def load(self, q, vpar, v1, v2):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (q, vpar, v1, v2)]
        lib().orc_load(self.h, *[_p(a) for a in arrs], len(arrs[0]))

    def init(self, counts, tail_fraction=0.0, kappa=3.0, tail_T=0.0, seed=20261203):
        """The initial-ion generator of kaos_init_particles, then load."""
        c = np.ascontiguousarray(counts, dtype=np.int64)
        lib().orc_init(self.h, _p(c), float(tail_fraction), float(kappa),
                       float(tail_T), int(seed))

    def set_fields(self, EA):
        self._EA = None if EA is None else np.ascontiguousarray(EA, dtype=np.float64)
        lib().orc_set_fields(self.h, _p(self._EA))

    def set_literal(self, on):
        lib().orc_set_literal(self.h, int(on))

    def update_tube(self, t):
        """Move the tube to Tube `t`'s tables at the next master step."""
        tc = t.to_c()
        if lib().orc_update_tube(self.h, C.addressof(tc)):
            raise ValueError("oracle: the moved tube must keep its cell count")

    def convect_now(self):
        """Test hook: apply a pending tube move immediately."""
        lib().orc_convect_now(self.h)

    def set_ena_grid(self, vg):
        """ENA velocity grid: Vp edges = vg.e1, Vphi = vg.e2, Vq = vg.epar."""
        self._evg = vg.to_c()
        self._ekeep = vg
        lib().orc_set_ena_grid(self.h, C.addressof(self._evg))

    def step(self, n):
        lib().orc_step(self.h, int(n))

    def count(self):
        ne = C.c_int64()
        ni = lib().orc_count(self.h, C.byref(ne))
        return ni, ne.value

    def moments(self, which):
        out = np.zeros(self.nq)
        lib().orc_get_moments(self.h, which, _p(out))
        return out

    def counts(self, full=False):
        n = self.nq * self.nbins if full else self.nq
        out = np.zeros(n, dtype=np.int64)
        lib().orc_get_counts(self.h, _p(out), n)
        return out

    def particles(self):
        ni, _ = self.count()
        q, vp, v1, v2, rho, z = (np.zeros(ni) for _ in range(6))
        qi = np.zeros(ni, dtype=np.int32)
        lib().orc_get_particles(self.h, _p(q), _p(vp), _p(v1), _p(v2), _p(qi),
                                _p(rho), _p(z))
        return dict(q=q, vpar=vp, vperp1=v1, vperp2=v2, qind=qi, rho=rho, z=z)

    def enas(self):
        _, ne = self.count()
        a = [np.zeros(ne) for _ in range(6)]
        lib().orc_get_enas(self.h, *[_p(x) for x in a])
        return dict(zip(("x", "y", "z", "vx", "vy", "vz"), a))

    def ambipolar(self, M0):
        M0 = np.ascontiguousarray(M0, dtype=np.float64)
        out = np.zeros(self.nq)
        lib().orc_ambipolar(self.h, _p(M0), _p(out))
        return out

    def force(self, x, y, z, vperp, aea, ag):
        out = np.zeros(4)
        lib().orc_force(self.h, x, y, z, vperp, aea, ag, _p(out))
        return out

    def boundary(self):
        v = np.zeros(4, dtype=np.int64)
        lib().orc_get_boundary(self.h, _p(v))
        return v


def quartic(q, p, phi=np.pi / 2):
    out = np.zeros(6)
    lib().orc_quartic(float(q), float(p), float(phi), _p(out))
    return out


def moment_filter(x, pt=11):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    lib().orc_filter(_p(x), _p(out), len(x), pt)
    return out
