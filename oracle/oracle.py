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
_LIB_OPS = os.path.join(_HERE, "_build", "liboracle_ops.so")
_lib = None
_lib_ops = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        _lib = _open(_LIB)
    return _lib


def lib_ops():
    """The op-counting build (oracle/op_count.cpp): same entry points and
    results, plus orc_ops_reset / orc_ops_get."""
    global _lib_ops
    if _lib_ops is None:
        L = _open(_LIB_OPS)
        L.orc_ops_reset.argtypes = []
        L.orc_ops_get.argtypes = [C.c_void_p]
        _lib_ops = L
    return _lib_ops


def _open(path):
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
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
    L.orc_get_boundary_ena.argtypes = [vp, vp]
    L.orc_quartic.argtypes = [C.c_double, C.c_double, C.c_double, vp]
    u32 = C.c_uint32
    L.orc_philox.argtypes = [u32, u32, u32, u32, C.c_uint64, vp]
    L.orc_filter.argtypes = [vp, vp, C.c_int, C.c_int]
    L.orc_destroy.argtypes = [vp]
    L.orc_ambipolar.argtypes = [vp, vp, vp]
    L.orc_force.argtypes = [vp, C.c_double, C.c_double, C.c_double,
                            C.c_double, C.c_double, C.c_double, vp]
    return L


def _p(a):
    return None if a is None else a.ctypes.data


class Oracle:
    """One tube on the CPU oracle."""

    def __init__(self, mi, tube, vg, counted=False):
        """counted: run on the op-counting build (same results)."""
        self._L = lib_ops() if counted else lib()
        self._mi, self._tube, self._vg = mi.to_c(), tube.to_c(), vg.to_c()
        self._keep = (tube, vg)
        self.nq = tube.nq
        self.three_d = mi.ION2VPERPflag == 1
        self.nbins = vg.nbins(self.three_d)
        self.h = self._L.orc_create(C.addressof(self._mi), C.addressof(self._tube),
                                    C.addressof(self._vg))
        if not self.h:
            raise ValueError("oracle: moving-average windows must be odd, >= 3 and "
                             "at most the tube's cell count")

    def __del__(self):
        if getattr(self, "h", None):
            self._L.orc_destroy(self.h)
            self.h = None

    def load(self, q, vpar, v1, v2):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (q, vpar, v1, v2)]
        self._L.orc_load(self.h, *[_p(a) for a in arrs], len(arrs[0]))

    def init(self, counts, tail_fraction=0.0, kappa=3.0, tail_T=0.0, seed=20261203):
        """The initial-ion generator of kaos_init_particles, then load."""
        c = np.ascontiguousarray(counts, dtype=np.int64)
        self._L.orc_init(self.h, _p(c), float(tail_fraction), float(kappa),
                       float(tail_T), int(seed))

    def set_fields(self, EA):
        self._EA = None if EA is None else np.ascontiguousarray(EA, dtype=np.float64)
        self._L.orc_set_fields(self.h, _p(self._EA))

    def set_literal(self, on):
        self._L.orc_set_literal(self.h, int(on))

    def update_tube(self, t):
        """Move the tube to Tube `t`'s tables at the next master step."""
        tc = t.to_c()
        if self._L.orc_update_tube(self.h, C.addressof(tc)):
            raise ValueError("oracle: the moved tube must keep its cell count")

    def convect_now(self):
        """Test hook: apply a pending tube move immediately."""
        self._L.orc_convect_now(self.h)

    def set_ena_grid(self, vg):
        """ENA velocity grid: Vp edges = vg.e1, Vphi = vg.e2, Vq = vg.epar."""
        self._evg = vg.to_c()
        self._ekeep = vg
        self._L.orc_set_ena_grid(self.h, C.addressof(self._evg))

    def step(self, n):
        self._L.orc_step(self.h, int(n))

    def count(self):
        ne = C.c_int64()
        ni = self._L.orc_count(self.h, C.byref(ne))
        return ni, ne.value

    def moments(self, which):
        out = np.zeros(self.nq)
        self._L.orc_get_moments(self.h, which, _p(out))
        return out

    def counts(self, full=False):
        n = self.nq * self.nbins if full else self.nq
        out = np.zeros(n, dtype=np.int64)
        self._L.orc_get_counts(self.h, _p(out), n)
        return out

    def particles(self):
        ni, _ = self.count()
        q, vp, v1, v2, rho, z = (np.zeros(ni) for _ in range(6))
        qi = np.zeros(ni, dtype=np.int32)
        self._L.orc_get_particles(self.h, _p(q), _p(vp), _p(v1), _p(v2), _p(qi),
                                _p(rho), _p(z))
        return dict(q=q, vpar=vp, vperp1=v1, vperp2=v2, qind=qi, rho=rho, z=z)

    def enas(self):
        _, ne = self.count()
        a = [np.zeros(ne) for _ in range(6)]
        self._L.orc_get_enas(self.h, *[_p(x) for x in a])
        return dict(zip(("x", "y", "z", "vx", "vy", "vz"), a))

    def ambipolar(self, M0):
        M0 = np.ascontiguousarray(M0, dtype=np.float64)
        out = np.zeros(self.nq)
        self._L.orc_ambipolar(self.h, _p(M0), _p(out))
        return out

    def force(self, x, y, z, vperp, aea, ag):
        out = np.zeros(4)
        self._L.orc_force(self.h, x, y, z, vperp, aea, ag, _p(out))
        return out

    def boundary(self):
        v = np.zeros(4, dtype=np.int64)
        self._L.orc_get_boundary(self.h, _p(v))
        return v

    def boundary_ena(self):
        """Escaped LB/UB ENA counts of the latest master step."""
        v = np.zeros(2, dtype=np.int64)
        self._L.orc_get_boundary_ena(self.h, _p(v))
        return v


OPS_PHASES = ("push_ion", "push_ena", "charge_exchange", "master")
OPS_CLASSES = ("add", "mul", "div", "sqrt", "transcendental")
# Weights of F_alg (FP64 flop-equivalents), fixed: add/mul 1, div/sqrt 4,
# each transcendental call 20.
OPS_WEIGHTS = (1, 1, 4, 4, 20)


def ops_reset():
    lib_ops().orc_ops_reset()


def ops_get():
    """{phase: {class: count}} accumulated by oracles built with
    counted=True since the last ops_reset()."""
    a = np.zeros(len(OPS_PHASES) * len(OPS_CLASSES), dtype=np.int64)
    lib_ops().orc_ops_get(_p(a))
    a = a.reshape(len(OPS_PHASES), len(OPS_CLASSES))
    return {ph: dict(zip(OPS_CLASSES, map(int, a[i])))
            for i, ph in enumerate(OPS_PHASES)}


def ops_weighted(counts):
    """Weighted sum of one phase's {class: count}."""
    return sum(w * counts[c] for c, w in zip(OPS_CLASSES, OPS_WEIGHTS))


def philox(counter, key):
    """Philox4x32-10 words of a 4-word counter and a 64-bit key (low word
    first), from the shared generator header."""
    out = np.zeros(4, dtype=np.uint32)
    lib().orc_philox(*[int(c) for c in counter], int(key), out.ctypes.data)
    return out


def quartic(q, p, phi=np.pi / 2):
    out = np.zeros(6)
    lib().orc_quartic(float(q), float(p), float(phi), _p(out))
    return out


def moment_filter(x, pt=11):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    lib().orc_filter(_p(x), _p(out), len(x), pt)
    return out
