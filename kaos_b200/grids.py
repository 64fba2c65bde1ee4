"""Flux-tube and velocity grids, initial particles and the synthetic
workloads.

The per-cell geometry follows ConfigGridGeneratorSub
(_0_ConfigGridGenerator.f90:299-310 uniform q edges, :514-545 metric factors
and cell volumes, :664-666 master-step cadence).  The velocity grid is
separable per axis with centres at (lo+hi)/2 and volumes as in
VelGridGeneratorSub (_0_0_VelGridGenerator.f90:338-467); geometric spacing
(an extension over the reference's uniform grids) is what the benchmark
configurations ask for.  All inputs are seeded synthetic data.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .model_input import (KB, MH, MO, PI, RE, GG, ME, ModelInput, Tube, VGrid,
                          KAOS_PREC_FP64, KAOS_PREC_MIXED)


def dipole_q_to_rtheta(q, p):
    """(q, p) -> (r, theta) on a dipole line: positive root u = r/RE of
    q^2 u^4 + u/p - 1 = 0 (closed form of the depressed resolvent cubic,
    then Newton polish), theta from sin^2 = u/p with the hemisphere of q."""
    q = np.asarray(q, dtype=np.float64)
    p = np.broadcast_to(np.asarray(p, dtype=np.float64), q.shape)
    Cp = 1.0 / (p * q * q)
    eps = 4.0 / (3.0 * q * q)
    t = (Cp * Cp / 2.0) / eps ** 1.5
    sigma = 2.0 * np.sqrt(eps) * np.sinh(np.arcsinh(t) / 3.0)
    mu = np.sqrt(sigma)
    u = (-mu + np.sqrt(-sigma + 2.0 * Cp / mu)) / 2.0
    for _ in range(3):
        f = q * q * u ** 4 + u / p - 1.0
        fp = 4.0 * q * q * u ** 3 + 1.0 / p
        u = u - f / fp
    th3 = np.arcsin(np.sqrt(u / p))
    th = np.where(q <= 0.0, PI - th3, th3)
    return u * RE, th


def q_of_altitude(alt_m, L):
    """q of the point at altitude alt_m on the dipole line p = L."""
    r = RE + alt_m
    s2 = r / (RE * L)
    ct = np.sqrt(1.0 - s2)
    return RE * RE * ct / (r * r)


@dataclasses.dataclass
class TubeSpec:
    L: float = 4.0
    nq: int = 128
    alt_lb: float = 1000e3        # lower-boundary altitude [m]
    q_ub: float = 1e-3            # upper boundary |q| (cap near the equator)
    phi: float = PI / 2.0         # phiLshellIC
    n0: float = 1e10              # base ion density at the LB altitude [m^-3]
    H: float = 300e3              # density scale height [m]
    Ti: float = 0.3 * 1.602e-19 / KB   # 0.3 eV in K
    n_particles: int = 100_000
    neut_n0: float = 0.0          # neutral density at LB altitude [m^-3]
    neut_H: float = 60e3          # neutral scale height [m]
    sigma_scale: float = 1e-20    # Lindsay-Stebbings unit 1e-16 cm^2 in m^2
    heat_rate_eV_s: float = 0.0   # ICR heating rate at the base cell [eV/s]
    chi: float = 1.7              # ICR spectral index
    capacity_factor: float = 1.3
    ms: float = 0.0               # species mass [kg]; 0 = ModelInput.ms
    qs: float = 0.0               # species charge [C]; 0 = ModelInput.qs



def make_tube(spec: TubeSpec, mi: ModelInput, q_edges=None) -> Tube:
    """Build the per-cell tables of one tube (NMH: q decreases upward);
    q_edges (nq + 1 values) keeps a given q grid, as a convected tube does
    (its q boundaries qGA/qGB are held, _8_11_Convection.f90:64-66)."""
    L, nq = spec.L, spec.nq
    if q_edges is not None:
        qe = np.array(q_edges, dtype=np.float64)
    else:
        qa = q_of_altitude(spec.alt_lb, L)
        qb = spec.q_ub
        # uniform q edges, _0_ConfigGridGenerator.f90:299-310
        k = np.arange(nq + 1, dtype=np.float64)
        qe = qa - k * (abs(qb - qa) / nq)
        qe[-1] = qb
    qGL, qGH = qe[:-1].copy(), qe[1:].copy()
    qGC = (qGL + qGH) / 2.0
    r, th = dipole_q_to_rtheta(qGC, L)
    ell = 1.0 + 3.0 * np.cos(th) ** 2
    # metric factors and volumes, _0_ConfigGridGenerator.f90:514-545
    hq = np.abs(r ** 3 / (RE ** 2 * np.sqrt(ell)))
    hp = np.abs(RE * np.sin(th) ** 3 / np.sqrt(ell))
    hphi = np.abs(r * np.sin(th))
    dq = np.abs(qGH - qGL)
    d3x = hq * hp * hphi * dq * 1e-3 * (PI / 180.0)
    d3x[d3x == 0.0] = 1e-9
    alt = r - RE
    n_c = spec.n0 * np.exp(-(alt - spec.alt_lb) / spec.H)
    nsnormfac = float(np.sum(n_c * d3x) / spec.n_particles)
    Ti = np.full(nq, spec.Ti)
    Te = np.full(nq, spec.Ti)          # Te = Ti (config 1)
    neut = spec.neut_n0 * np.exp(-(alt - spec.alt_lb) / spec.neut_H)
    # ICR tables: S0 chosen so that the mean heating rate of the base cell's
    # Maxwellian ions is heat_rate_eV_s under the reference's stochastic
    # kick (_8_1_1_0_WaveHeating.f90:83-150): per step and component
    # dV_i = (h/tau) sqrt(2 D_i tau) G_i, so <d(m v^2/2)/dt> =
    # m (D1 + D2) h <1/tau>, with D_i = q^2/(2 m^2) xi_i eta S0
    # (Omega/Omega0)^-chi_i (sigma = 1, Omega = Omega0 at the base) and
    # 1/tau = (Omega/2 pi) sqrt(|V|||/(Omega sum ds)); for V|| ~ N(0, s^2),
    # <|V|||^(1/2)> = s^(1/2) 2^(1/4) Gamma(3/4) / sqrt(pi).
    ms = spec.ms if spec.ms > 0 else mi.ms
    qs = spec.qs if spec.qs != 0 else mi.qs
    Bc = 8.06e15 * np.sqrt(ell) / r ** 3
    Om = qs * Bc / ms
    Om0 = np.full(nq, Om[0])
    xi, eta = 0.5, 0.125
    arc = float(np.sum(hq * dq))
    S0val = 0.0
    if spec.heat_rate_eV_s > 0:
        rate_J = spec.heat_rate_eV_s * 1.602e-19
        sig = np.sqrt(KB * spec.Ti / ms)
        e_sqrt_v = np.sqrt(sig) * 2.0 ** 0.25 * math.gamma(0.75) / np.sqrt(PI)
        inv_tau = (Om[0] / (2.0 * PI)) * np.sqrt(1.0 / (Om[0] * arc)) * e_sqrt_v
        S0val = rate_J / (ms * 2.0 * (qs ** 2 / (2 * ms ** 2)) * xi * eta * mi.h * inv_tau)
    t = Tube(nq=nq, pG=L, phiG=spec.phi, nsnormfac=nsnormfac,
             nsnormCLB=0.0, nsnormCUB=0.0, qGL=qGL, qGH=qGH, qGC=qGC,
             hqC=hq, dqC=dq, d3xC=d3x, rGC=r, thetaGC=th, ellGC=ell,
             TeG=Te, TsG=Ti,
             nsnormCNeut=neut * spec.sigma_scale,
             lambdaPerp=np.zeros(nq), EtaLH=np.full(nq, eta),
             XiPerp1=np.full(nq, xi), XiPerp2=np.full(nq, xi),
             S0=np.full(nq, S0val), OmegaG0=Om0,
             ChiPerp1=np.full(nq, spec.chi), ChiPerp2=np.full(nq, spec.chi),
             sumdsICR=arc, ms=spec.ms, qs=spec.qs)
    counts = np.rint(n_c * d3x / nsnormfac).astype(np.int64)
    # LB injection: the LB-cell macro-particle count per master step
    # (_0_1_1_ConfigGridGeneratorB.f90:189), scaled by the ratio of the
    # master-step cadence to the LB-cell transit time (Q0ndatfac,
    # _0_ConfigGridGenerator.f90:664-666) when the cadence is shorter.
    q0ndatfac = hq[0] * dq[0] * np.sqrt(ms / (KB * Ti[0])) / mi.h
    frac = min(1.0, mi.ndatfac / q0ndatfac)
    t.nsnormCLB = float(np.rint(counts[0] * frac))
    t.capacity = int(spec.n_particles * spec.capacity_factor) + 1024
    t._counts = counts  # type: ignore[attr-defined]
    return t


def geometric_edges(n: int, vmax: float, ratio: float = 1.06, symmetric=True):
    """Edges of a geometric grid: symmetric about 0 with n cells over
    [-vmax, vmax] (n even), or n cells over [0, vmax]."""
    if symmetric:
        half = n // 2
        w = ratio ** np.arange(half)
        w = w / w.sum() * vmax
        pos = np.concatenate([[0.0], np.cumsum(w)])
        e = np.concatenate([-pos[::-1], pos[1:]])
        if n % 2:
            raise ValueError("symmetric geometric grid needs an even n")
        e[0], e[-1] = -vmax, vmax
        return e
    w = ratio ** np.arange(n)
    w = w / w.sum() * vmax
    e = np.concatenate([[0.0], np.cumsum(w)])
    e[-1] = vmax
    return e


def make_vgrid(three_d: bool, n1: int, n2: int, npar: int, vmax: float) -> VGrid:
    if three_d:
        return VGrid(e1=geometric_edges(n1, vmax), e2=geometric_edges(n2, vmax),
                     epar=geometric_edges(npar, vmax))
    return VGrid(e1=geometric_edges(n1, vmax, symmetric=False), e2=None,
                 epar=geometric_edges(npar, vmax))


def initial_particles(tube: Tube, spec: TubeSpec, mi: ModelInput, seed: int,
                      at_centre: bool = False):
    """Maxwellian ions, per-cell counts nint(n d3x / nsnormfac)
    (_2_1_DensityProfileA1.f90); positions uniform in q within each cell
    (at_centre=True puts them at the cell centre as DensityProfileB does)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = tube._counts  # type: ignore[attr-defined]
    n = int(counts.sum())
    cell = np.repeat(np.arange(tube.nq), counts)
    if at_centre:
        q = tube.qGC[cell].copy()
    else:
        f = rng.uniform(0.02, 0.98, size=n)
        q = tube.qGL[cell] + f * (tube.qGH[cell] - tube.qGL[cell])
    sig = np.sqrt(KB * tube.TsG[cell] / (tube.ms if tube.ms > 0 else mi.ms))
    v = rng.normal(size=(3, n)) * sig
    return q, v[0].copy(), v[1].copy(), v[2].copy()


# ---- the named workloads -------------------------------------------------
def config_small(n_particles=4000, three_d=True, nq=32, steps_per_master=5,
                 heating=False, collisions=False, seed=7):
    """A small tube for parity tests (seconds on the oracle)."""
    mi = ModelInput(h=0.01, ndatfac=steps_per_master,
                    ION2VPERPflag=1 if three_d else 0,
                    ICRflag=1 if heating else 0,
                    QEXCHANGEflag=1 if collisions else 0)
    spec = TubeSpec(L=4.0, nq=nq, n_particles=n_particles,
                    q_ub=0.15, H=600e3,
                    heat_rate_eV_s=5.0 if heating else 0.0,
                    neut_n0=3e18 if collisions else 0.0, neut_H=300e3)
    tube = make_tube(spec, mi)
    vg = (make_vgrid(True, 16, 16, 24, 8e3) if three_d
          else make_vgrid(False, 16, 0, 24, 8e3))
    return mi, spec, tube, vg


def config_c1(n_particles=100_000):
    """Plain FP64 method, small: L=4, 1000 km -> equator (|q| >= 1e-3),
    128 cells, 2D grid vpar 64 x vperp 32 geometric, |v|max 30 km/s,
    n0 1e10 m^-3, H 300 km, T 0.3 eV, gravity + mirror + ambipolar,
    dt 0.01 s, 200 steps."""
    mi = ModelInput(h=0.01, ndatfac=20, ION2VPERPflag=0)
    spec = TubeSpec(L=4.0, nq=128, n_particles=n_particles, q_ub=1e-3)
    tube = make_tube(spec, mi)
    vg = make_vgrid(False, 32, 0, 64, 30e3)
    return mi, spec, tube, vg


def config_c2(n_particles=10_000_000, heating=True, collisions=True,
              precision=KAOS_PREC_FP64, ndatfac=50):
    """Precision A/B: L=4, 256 cells, 3D grid 48x48x64, 1e7 O+, heating
    (chi 1.7, 1e-3 eV/s at the base), O neutrals n0 1e14 m^-3 H 60 km,
    dt 0.005 s, 500 steps."""
    mi = ModelInput(h=0.005, ndatfac=ndatfac, ION2VPERPflag=1,
                    ICRflag=1 if heating else 0,
                    QEXCHANGEflag=1 if collisions else 0,
                    precision=precision)
    spec = TubeSpec(L=4.0, nq=256, n_particles=n_particles, q_ub=1e-3,
                    heat_rate_eV_s=1e-3 if heating else 0.0, chi=1.7,
                    neut_n0=1e14 if collisions else 0.0, neut_H=60e3)
    tube = make_tube(spec, mi)
    vg = make_vgrid(True, 48, 48, 64, 30e3)
    return mi, spec, tube, vg


def moved_tube(spec: TubeSpec, mi: ModelInput, tube: Tube, L_new: float) -> Tube:
    """The tables of `tube` regenerated on a new L-shell for ConvectionSub:
    same q grid and macro-particle weight, geometry of the new field line."""
    import dataclasses
    sp = dataclasses.replace(spec, L=L_new)
    t = make_tube(sp, mi, q_edges=np.concatenate([tube.qGL, tube.qGH[-1:]]))
    t.nsnormfac = tube.nsnormfac
    t.nsnormCLB, t.nsnormCUB = tube.nsnormCLB, tube.nsnormCUB
    t.capacity = tube.capacity
    return t


# kappa tail of the large single-tube workload
C3_TAIL = dict(tail_fraction=0.1, kappa=3.0, tail_T=5.0 * 1.602e-19 / KB)


def config_c3(n_particles=100_000_000, precision=KAOS_PREC_MIXED, ndatfac=50):
    """Large single tube: L=6, 512 cells from 800 km to the equator
    (|q| >= 1e-3), 3D grid 64x64x96, 1e8 O+ (90 % 0.3 eV Maxwellian core +
    10 % kappa = 3, 5 eV tail: C3_TAIL with kaos_init_particles), heating
    (chi 1.7, 1e-3 eV/s at the base) and O neutrals (1e14 m^-3, H 60 km) on,
    LB injection with V|| drawn from the Maxwellian flux into the tube
    (FLUXINJECTIONflag), UB outflow removal, dt 0.005 s."""
    mi = ModelInput(h=0.005, ndatfac=ndatfac, ION2VPERPflag=1, ICRflag=1,
                    QEXCHANGEflag=1, FLUXINJECTIONflag=1, precision=precision)
    spec = TubeSpec(L=6.0, nq=512, alt_lb=800e3, n_particles=n_particles,
                    q_ub=1e-3, heat_rate_eV_s=1e-3, chi=1.7, neut_n0=1e14,
                    neut_H=60e3)
    tube = make_tube(spec, mi)
    vg = make_vgrid(True, 64, 64, 96, 40e3)
    return mi, spec, tube, vg


def config_c4(ntubes=256, precision=KAOS_PREC_MIXED, ndatfac=50, seed=4):
    """Batched uneven tubes in one launch: ntubes flux tubes with L uniform
    in [2, 8], cells per tube uniform in {64..512}, ions per tube
    log-uniform in [1e4, 1e6] (about 5e7 for 256 tubes), base density
    log-uniform in [1e9, 1e11] m^-3, T uniform in [0.1, 1] eV, a shared
    3D grid 48x48x64, heating on with a per-tube base rate log-uniform in
    [1e-4, 1e-2] eV/s; dt 0.005 s.  The tube parameters are drawn from a
    seeded generator; initial ions come from kaos_init_particles with each
    tube's per-cell counts (tube._counts)."""
    rng = np.random.default_rng(seed)
    mi = ModelInput(h=0.005, ndatfac=ndatfac, ION2VPERPflag=1, ICRflag=1,
                    precision=precision)
    specs, tubes = [], []
    for _ in range(ntubes):
        sp = TubeSpec(L=float(rng.uniform(2.0, 8.0)),
                      nq=int(rng.integers(64, 513)),
                      n_particles=int(round(10 ** rng.uniform(4.0, 6.0))),
                      q_ub=1e-3, n0=float(10 ** rng.uniform(9.0, 11.0)),
                      Ti=float(rng.uniform(0.1, 1.0)) * 1.602e-19 / KB,
                      heat_rate_eV_s=float(10 ** rng.uniform(-4.0, -2.0)),
                      chi=1.7)
        specs.append(sp)
        tubes.append(make_tube(sp, mi))
    vg = make_vgrid(True, 48, 48, 64, 30e3)
    return mi, specs, tubes, vg


def config_c5(ntubes=64, n_ions=20_000_000, precision=KAOS_PREC_MIXED,
              ndatfac=50, seed=5, neut_n0=1e16):
    """Two species plus neutral products, batched: ntubes flux tubes with L
    uniform in [3, 7], 256 cells each, H+ and O+ at a 1:4 density ratio as
    two entries per tube (2e7 ions in all), charge exchange with a neutral
    H exosphere (scale height 1000 km) producing ENAs, ENA moments on a
    48x48x64 grid (the returned evg), dt 0.005 s.  The collision model's
    Poisson mean is per cell and step (n_n sigma v h, not times the cell's
    ions), so at the configuration's 1e11 m^-3 base density it is ~1e-7 and
    no ENA would form within a run; neut_n0 (default 1e16 m^-3) sets it.
    Entries alternate O+, H+ per tube.  The E x B drift of 0.5 km/s moves
    each tube by CONV_C5_DL in L per master step (grids.moved_tube and
    kaos_update_tube)."""
    rng = np.random.default_rng(seed)
    mi = ModelInput(h=0.005, ndatfac=ndatfac, ION2VPERPflag=1, QEXCHANGEflag=1,
                    precision=precision)
    mi.mNeut = MH
    per_tube = n_ions / ntubes
    specs, tubes = [], []
    for _ in range(ntubes):
        L = float(rng.uniform(3.0, 7.0))
        for ms, frac, n0 in ((MO, 0.8, 1e10), (MH, 0.2, 2.5e9)):
            sp = TubeSpec(L=L, nq=256, n_particles=int(round(per_tube * frac)),
                          q_ub=1e-3, n0=n0, neut_n0=neut_n0, neut_H=1000e3,
                          ms=ms, qs=1.602e-19)
            specs.append(sp)
            tubes.append(make_tube(sp, mi))
    vg = make_vgrid(True, 48, 48, 64, 30e3)
    evg = make_vgrid(True, 48, 48, 64, 30e3)
    return mi, specs, tubes, vg, evg


def conv_c5_dl(ndatfac, h=0.005, v=500.0):
    """L-shell change of a tube per master interval of ndatfac steps under
    an E x B drift v [m/s] at the equator (dL = v ndatfac h / RE)."""
    return v * ndatfac * h / RE


# the change per master interval of 50 steps of 5 ms at 0.5 km/s
CONV_C5_DL = conv_c5_dl(50)


def config_escaping(neut_n0=0.0):
    """A short hot tube (L=3, 24 cells up to |q| = 0.5, 5 eV O+, dt 1 s,
    master step every 2 steps) that loses ~40 ions per master step through
    both boundaries, with 30 injected at the lower one: the removal and
    injection test case.  neut_n0 > 0 adds charge exchange with neutrals of
    that base density (scale height 300 km), whose ENAs leave through both
    boundaries too."""
    mi = ModelInput(h=1.0, ndatfac=2, ION2VPERPflag=1,
                    QEXCHANGEflag=1 if neut_n0 > 0 else 0)
    vg = make_vgrid(True, 16, 16, 24, 3e4)
    spec = TubeSpec(L=3.0, nq=24, n_particles=2500, q_ub=0.5, H=400e3,
                    Ti=5.0 * 1.602e-19 / KB, neut_n0=neut_n0, neut_H=300e3)
    tube = make_tube(spec, mi)
    tube.nsnormCLB = 30.0
    return mi, spec, tube, vg
