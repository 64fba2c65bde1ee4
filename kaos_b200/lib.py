"""ctypes binding of libkaos_gpu.so (the C-ABI in include/kaos_gpu.h) and a
small Python front (`Solver`) that drives one handle the way KAOS's
KineticSolverSub drives its tubes.

The product path is the CUDA library; there is no CPU fallback: loading
fails loudly when libkaos_gpu.so is missing or no GPU is present.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

from .model_input import (KaosParams, KaosTube, KaosVGrid, ModelInput, Tube,
                          VGrid, KAOS_NMOMENTS)

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libkaos_gpu.so")

# every symbol declared in include/kaos_gpu.h
EXPORTS = [
    "kaos_create", "kaos_load_particles", "kaos_set_fields", "kaos_step",
    "kaos_get_step", "kaos_get_count", "kaos_get_moments", "kaos_get_counts",
    "kaos_set_export", "kaos_get_particles", "kaos_get_positions",
    "kaos_get_enas", "kaos_get_boundary", "kaos_get_boundary_ena", "kaos_get_timing",
    "kaos_set_graph",
    "kaos_set_launch", "kaos_last_error", "kaos_get_status", "kaos_destroy",
    "kaos_version", "kaos_get_push_timing", "kaos_moments_noalloc",
    "kaos_get_launch", "kaos_set_ena_grid", "kaos_init_particles",
    "kaos_set_reduce", "kaos_set_rank", "kaos_set_id_base", "kaos_update_tube",
    "kaos_get_moments_all", "kaos_sample_rng",
]

# kaos_sample_rng kinds and values per draw
SAMPLE_PHILOX, SAMPLE_GAUSS32, SAMPLE_GAUSS64, SAMPLE_POISSON, SAMPLE_GAUSS64T = 0, 1, 2, 3, 4
_SAMPLE_WIDTH = {0: 4, 1: 2, 2: 2, 3: 1, 4: 2}

# int fn(void *ctx, uint32_t *buf, int64_t count, void *stream)
REDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p)

_lib = None


class KaosError(RuntimeError):
    pass


def load(path: str = LIBPATH):
    """Load the library (no compute, works without a GPU)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise KaosError(f"{path} missing: build it with `python -m kaos_b200.build`")
    L = C.CDLL(path)
    vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
    L.kaos_create.argtypes = [vp, vp, i32, vp, C.POINTER(vp)]
    L.kaos_load_particles.argtypes = [vp, i32, vp, vp, vp, vp, i64]
    L.kaos_set_fields.argtypes = [vp, i32, vp, i32]
    L.kaos_step.argtypes = [vp, i64]
    L.kaos_get_step.argtypes = [vp, C.POINTER(i64)]
    L.kaos_get_count.argtypes = [vp, i32, C.POINTER(i64), C.POINTER(i64)]
    L.kaos_get_moments.argtypes = [vp, i32, i32, vp, i32]
    L.kaos_get_moments_all.argtypes = [vp, i32, vp, i32]
    L.kaos_get_counts.argtypes = [vp, i32, vp, i64]
    L.kaos_set_export.argtypes = [vp, i32]
    L.kaos_get_particles.argtypes = [vp, i32, vp, vp, vp, vp, vp, i64]
    L.kaos_get_positions.argtypes = [vp, i32, vp, vp, i64]
    L.kaos_get_enas.argtypes = [vp, i32] + [vp] * 6 + [i64]
    L.kaos_get_boundary.argtypes = [vp, i32] + [C.POINTER(i64)] * 4
    L.kaos_get_boundary_ena.argtypes = [vp, i32] + [C.POINTER(i64)] * 2
    L.kaos_get_timing.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(i64)]
    L.kaos_get_push_timing.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(i64)]
    L.kaos_moments_noalloc.argtypes = [vp, vp, i32, vp, vp, C.c_double, vp, vp,
                                        vp, vp, i64, vp, vp, vp]
    L.kaos_sample_rng.argtypes = [i32, C.c_uint64, C.c_uint64, C.c_uint32,
                                  C.c_uint32, C.c_double, i64, vp]
    L.kaos_set_graph.argtypes = [vp, i32]
    L.kaos_set_launch.argtypes = [vp, i32, i32]
    L.kaos_get_launch.argtypes = [vp, C.POINTER(i32), C.POINTER(i32)]
    L.kaos_set_ena_grid.argtypes = [vp, vp]
    L.kaos_init_particles.argtypes = [vp, i32, vp]
    L.kaos_set_reduce.argtypes = [vp, REDUCE_FN, vp]
    L.kaos_set_rank.argtypes = [vp, i32, i32]
    L.kaos_set_id_base.argtypes = [vp, i32, C.c_uint64]
    L.kaos_update_tube.argtypes = [vp, i32, vp]
    L.kaos_last_error.argtypes = [vp]
    L.kaos_last_error.restype = C.c_char_p
    L.kaos_get_status.argtypes = [vp, C.POINTER(C.c_uint32)]
    L.kaos_destroy.argtypes = [vp]
    L.kaos_version.restype = C.c_char_p
    _lib = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data


def sample_rng(kind, n, seed=1, id0=0, step=0, c3=0, lam=0.0):
    """Draws of the device random-number generators (kaos_sample_rng):
    array [n, width] (width 4 Philox words, 2 Gaussians, 1 Poisson count)."""
    w = _SAMPLE_WIDTH[kind]
    out = np.zeros((n, w))
    rc = load().kaos_sample_rng(int(kind), int(seed), int(id0), int(step), int(c3),
                                float(lam), int(n), _p(out))
    if rc != 0:
        raise KaosError(f"kaos_sample_rng failed (status {rc})")
    return out


class Solver:
    """One libkaos_gpu handle over one or more tubes."""

    def __init__(self, mi: ModelInput, tubes: Sequence[Tube], vg: VGrid):
        L = load()
        self.mi = mi
        self._p = mi.to_c()
        self._tubes = list(tubes)
        arr = (KaosTube * len(tubes))()
        for k, t in enumerate(tubes):
            arr[k] = t.to_c()
        self._tarr = arr
        self._vg = vg
        self._vgc = vg.to_c()
        self.three_d = mi.ION2VPERPflag == 1
        self.nbins = vg.nbins(self.three_d)
        h = C.c_void_p()
        rc = L.kaos_create(C.addressof(self._p), C.addressof(arr), len(tubes),
                           C.addressof(self._vgc), C.byref(h))
        self.h = h.value
        self._check(rc)

    def _check(self, rc):
        if rc != 0:
            msg = load().kaos_last_error(self.h).decode() if self.h else ""
            raise KaosError(f"kaos call failed (status {rc}): {msg}")

    def close(self):
        if getattr(self, "h", None):
            load().kaos_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- calls -----------------------------------------------------------
    def load(self, tube, q, vpar, v1, v2):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (q, vpar, v1, v2)]
        self._check(load().kaos_load_particles(self.h, tube, *[_p(a) for a in arrs],
                                               len(arrs[0])))

    def set_fields(self, tube, EA):
        a = None if EA is None else np.ascontiguousarray(EA, dtype=np.float64)
        self._check(load().kaos_set_fields(self.h, tube, _p(a),
                                           0 if a is None else len(a)))

    def set_export(self, on):
        self._check(load().kaos_set_export(self.h, int(on)))

    def step(self, n):
        self._check(load().kaos_step(self.h, int(n)))

    def count(self, tube=0):
        a, b = C.c_int64(), C.c_int64()
        self._check(load().kaos_get_count(self.h, tube, C.byref(a), C.byref(b)))
        return a.value, b.value

    def moments(self, which, tube=0):
        out = np.zeros(self._tubes[tube].nq)
        self._check(load().kaos_get_moments(self.h, tube, which, _p(out), len(out)))
        return out

    def moments_all(self, tube=0, out=None):
        """All KAOS_NMOMENTS selectors at once: array [KAOS_NMOMENTS, nq]
        (into `out` when given, e.g. pinned host memory)."""
        nq = self._tubes[tube].nq
        if out is None:
            out = np.zeros((KAOS_NMOMENTS, nq))
        elif out.shape != (KAOS_NMOMENTS, nq) or out.dtype != np.float64 or \
                not out.flags.c_contiguous:
            raise ValueError(f"out: C-contiguous float64 array of shape ({KAOS_NMOMENTS}, {nq})")
        self._check(load().kaos_get_moments_all(self.h, tube, _p(out), nq))
        return out

    def counts(self, tube=0, full=False):
        nq = self._tubes[tube].nq
        n = nq * self.nbins if full else nq
        out = np.zeros(n, dtype=np.int64)
        self._check(load().kaos_get_counts(self.h, tube, _p(out), n))
        return out

    def state(self, tube=0, out=None):
        """The ions' field-line state: q, V||, Vperp1, Vperp2, Qindk1.  With
        `out` (arrays q, vpar, vperp1, vperp2 float64 and qind int32 of at
        least the ion count, e.g. in pinned host memory) the state is
        written into views of those arrays."""
        ni, _ = self.count(tube)
        if out is None:
            q, vp, v1, v2 = (np.zeros(ni) for _ in range(4))
            qi = np.zeros(ni, dtype=np.int32)
        else:
            q, vp, v1, v2 = (out[k][:ni] for k in ("q", "vpar", "vperp1", "vperp2"))
            qi = out["qind"][:ni]
            if not (all(a.dtype == np.float64 and a.flags.c_contiguous and len(a) == ni
                        for a in (q, vp, v1, v2)) and qi.dtype == np.int32 and len(qi) == ni):
                raise ValueError("out: float64 q/vpar/vperp1/vperp2 and int32 qind "
                                 f"arrays of at least {ni} elements")
        self._check(load().kaos_get_particles(self.h, tube, _p(q), _p(vp), _p(v1),
                                              _p(v2), _p(qi), ni))
        return dict(q=q, vpar=vp, vperp1=v1, vperp2=v2, qind=qi)

    def particles(self, tube=0):
        ni, _ = self.count(tube)
        q, vp, v1, v2 = (np.zeros(ni) for _ in range(4))
        qi = np.zeros(ni, dtype=np.int32)
        self._check(load().kaos_get_particles(self.h, tube, _p(q), _p(vp), _p(v1),
                                              _p(v2), _p(qi), ni))
        rho, z = np.zeros(ni), np.zeros(ni)
        self._check(load().kaos_get_positions(self.h, tube, _p(rho), _p(z), ni))
        return dict(q=q, vpar=vp, vperp1=v1, vperp2=v2, qind=qi, rho=rho, z=z)

    def enas(self, tube=0):
        _, ne = self.count(tube)
        a = [np.zeros(ne) for _ in range(6)]
        self._check(load().kaos_get_enas(self.h, tube, *[_p(x) for x in a], ne))
        return dict(zip(("x", "y", "z", "vx", "vy", "vz"), a))

    def boundary(self, tube=0):
        v = [C.c_int64() for _ in range(4)]
        self._check(load().kaos_get_boundary(self.h, tube, *[C.byref(x) for x in v]))
        return np.array([x.value for x in v])

    def boundary_ena(self, tube=0):
        """Escaped LB/UB ENA counts of the latest master step."""
        v = [C.c_int64() for _ in range(2)]
        self._check(load().kaos_get_boundary_ena(self.h, tube, *[C.byref(x) for x in v]))
        return np.array([x.value for x in v])

    def timing(self):
        ms, nl = C.c_double(), C.c_int64()
        self._check(load().kaos_get_timing(self.h, C.byref(ms), C.byref(nl)))
        return ms.value, nl.value

    def push_timing(self):
        ms, nl = C.c_double(), C.c_int64()
        self._check(load().kaos_get_push_timing(self.h, C.byref(ms), C.byref(nl)))
        return ms.value, nl.value

    def set_graph(self, on):
        self._check(load().kaos_set_graph(self.h, int(on)))

    def set_reduce(self, fn):
        """Cross-rank sum of the binning accumulators of a split tube:
        fn(buf_ptr, count, stream_ptr) -> 0 sums `count` uint32 counters at
        device address buf_ptr over the ranks in place; None removes it."""
        if fn is None:
            self._reduce = None
            self._check(load().kaos_set_reduce(self.h, REDUCE_FN(), None))
            return
        self._reduce = REDUCE_FN(lambda ctx, buf, count, stream: int(fn(buf, count, stream)))
        self._check(load().kaos_set_reduce(self.h, self._reduce, None))

    def update_tube(self, tube, t):
        """Move tube `tube` to the tables of Tube `t` (new L-shell, same q
        grid) at the next master step (ConvectionSub)."""
        tc = t.to_c()
        self._check(load().kaos_update_tube(self.h, int(tube), C.addressof(tc)))
        self._tubes[tube] = t

    def set_rank(self, rank, nranks):
        self._check(load().kaos_set_rank(self.h, int(rank), int(nranks)))

    def set_id_base(self, tube, base):
        self._check(load().kaos_set_id_base(self.h, int(tube), int(base)))

    def init_particles(self, tube, counts, tail_fraction=0.0, kappa=3.0,
                       tail_T=0.0, seed=20261203):
        """Generate the initial ions of one tube on the device (counts per
        cell; Maxwellian at TsG, optional kappa tail)."""
        from .model_input import KaosInit
        c = np.ascontiguousarray(counts, dtype=np.int64)
        ini = KaosInit()
        ini.counts = c.ctypes.data_as(C.POINTER(C.c_int64))
        ini.tail_fraction, ini.kappa, ini.tail_T, ini.seed = (
            float(tail_fraction), float(kappa), float(tail_T), int(seed))
        self._check(load().kaos_init_particles(self.h, int(tube), C.addressof(ini)))

    def set_ena_grid(self, vg):
        """ENA velocity grid: Vp edges = vg.e1, Vphi = vg.e2, Vq = vg.epar."""
        self._evg = vg.to_c()
        self._ekeep = vg
        self._check(load().kaos_set_ena_grid(self.h, C.addressof(self._evg)))

    def set_launch(self, chunk, mode):
        """chunk ions per work item (1024/2048/4096); mode bit 0: 0 = block
        per item, 1 = persistent grid; bits 1-2 (mixed): register budget
        0 = 64, 1 = 80, 2 = 72 (128-thread blocks); chunk 0 re-arms the
        autotuner."""
        self._check(load().kaos_set_launch(self.h, int(chunk), int(mode)))

    def launch(self):
        c, m = C.c_int32(), C.c_int32()
        self._check(load().kaos_get_launch(self.h, C.byref(c), C.byref(m)))
        return c.value, m.value
