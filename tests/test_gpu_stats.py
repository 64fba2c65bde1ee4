"""Statistical validation of the stochastic terms on the GPU.

The reference draws from gfortran's unseeded random_number
(GaussianRNGSub _3_1_GaussianRNG.f90:27-37, PoissonRNGSub
_3_2_PoissonRNG.f90:27-42, used by WaveHeatingSub
_8_1_1_0_WaveHeating.f90:141-150 and IonNeutralCollisionFrequencyASub
_8_6_6_1_...:275-301), which cannot be reproduced, so the stochastic terms
are checked by their distributions:

* the device Philox4x32-10 against the published known-answer vectors;
* the FP32 Gaussian pair of the mixed push's heating kick and the FP64 pair
  of the FP64 push (kaos_sample_rng evaluates the same device functions):
  mean, variance, tail fractions, independence of the pair, a KS test
  against the normal law, and agreement of the two precisions;
* the collision-count Poisson draw: mean and a chi-square test of its
  distribution for several means;
* a seed ensemble: 20 oracle runs and 20 mixed-precision GPU runs of a
  heated tube with charge exchange, from the same initial ions with
  different random streams -- every moment of every cell agrees between
  the ensembles (difference of means within 3 sigma), and one further GPU
  run lies within 3 sigma of the oracle ensemble;
* two-sample KS tests on the V|| and Vperp marginals of the distribution
  function, pooled and per cell (cells with >= 80 ions), between a GPU
  run and an oracle run with
  different streams (and a heated against an unheated run, which must
  fail: the test has power).
"""
import dataclasses
import math

import numpy as np
import pytest
from scipy import stats

from kaos_b200 import build as kbuild
from kaos_b200 import grids
from kaos_b200 import lib as klib
from kaos_b200.lib import Solver
from kaos_b200.model_input import (KAOS_EAMAG, KAOS_M0, KAOS_M1PAR, KAOS_M1PERP1,
                                   KAOS_M1PERP2, KAOS_M2, KAOS_M2PAR, KAOS_M2PERP1,
                                   KAOS_M2PERP2, KAOS_NQ, KAOS_PREC_MIXED)
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

MOMENTS = [KAOS_M0, KAOS_M1PAR, KAOS_M1PERP1, KAOS_M1PERP2, KAOS_M2, KAOS_M2PAR,
           KAOS_M2PERP1, KAOS_M2PERP2, KAOS_NQ, KAOS_EAMAG]
ENSEMBLE = 20
STEPS = 25  # master steps at 5, 10, 15, 20, 25


@pytest.fixture(scope="module", autouse=True)
def _build():
    kbuild.build()


# ---- generators ------------------------------------------------------------
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff, 0xffffffff),
     (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_device_philox_known_answers(ctr, key, want):
    w = klib.sample_rng(klib.SAMPLE_PHILOX, 1, seed=key[0] | (key[1] << 32),
                        id0=ctr[0] | (ctr[1] << 32), step=ctr[2], c3=ctr[3])
    assert [int(x) for x in w[0]] == list(want)


@pytest.fixture(scope="module")
def gauss():
    n = 4_000_000
    g32 = klib.sample_rng(klib.SAMPLE_GAUSS32, n, seed=20261203, id0=1 << 20, step=77)
    g64 = klib.sample_rng(klib.SAMPLE_GAUSS64, n, seed=20261203, id0=1 << 20, step=77)
    return g32, g64


def test_table_reduced_gaussian_pair_equals_fp64_pair(gauss):
    """The Gaussian pair of the KAOS_PREC_MIXED_K64 kick (table-reduced FP64
    logarithm and sine/cosine, kaos_f64.cuh) against the FP64 push's pair
    from the same Philox words: equal to a few units of 2^-52."""
    n = len(gauss[1])
    g64t = klib.sample_rng(klib.SAMPLE_GAUSS64T, n, seed=20261203, id0=1 << 20, step=77)
    assert np.max(np.abs(g64t - gauss[1])) < 1e-14


@pytest.mark.parametrize("which", [0, 1])
def test_gaussian_moments_tails_ks(gauss, which):
    g = gauss[which]
    x = g.ravel()
    n = len(x)
    assert abs(x.mean()) < 5.0 / math.sqrt(n)
    assert abs(x.var() - 1.0) < 5.0 * math.sqrt(2.0 / n)
    for t in (2.0, 3.0, 4.0):
        p = math.erfc(t / math.sqrt(2.0))
        k = np.count_nonzero(np.abs(x) > t)
        assert abs(k - n * p) < 5.0 * math.sqrt(n * p * (1 - p)) + 2, (t, k, n * p)
    # the two members of a pair are independent
    r = np.corrcoef(g[:, 0], g[:, 1])[0, 1]
    assert abs(r) < 5.0 / math.sqrt(len(g))
    assert stats.kstest(x, "norm").pvalue > 1e-4
    if which == 0:
        # 23-bit uniforms: |G| <= sqrt(-2 ln 2^-24) = 5.77 (tail truncated at
        # a probability of 8e-9)
        assert np.max(np.abs(x)) <= 5.78


def test_gaussian_fp32_tracks_fp64(gauss):
    """Same Philox words, 23-bit uniforms and hardware functions against
    53-bit uniforms and FP64 functions: the pairs agree closely except for
    the rare draws whose first uniform lies within 2^-23 of 1."""
    d = np.abs(gauss[0] - gauss[1])
    assert np.median(d) < 1e-6
    assert np.quantile(d, 0.999) < 1e-5


@pytest.mark.parametrize("lam", [0.05, 0.7, 3.0, 12.0])
def test_poisson_draw(lam):
    n = 200_000
    k = klib.sample_rng(klib.SAMPLE_POISSON, n, seed=99, id0=0, step=5, lam=lam)[:, 0]
    assert np.all(k == np.round(k)) and k.min() >= 0
    assert abs(k.mean() - lam) < 5.0 * math.sqrt(lam / n)
    kmax = int(lam + 6 * math.sqrt(lam) + 3)
    obs = np.bincount(k.astype(np.int64), minlength=kmax + 1)
    exp = stats.poisson.pmf(np.arange(len(obs)), lam) * n
    exp[-1] += stats.poisson.sf(len(obs) - 1, lam) * n
    # lump the bins whose expectation is below 5 into their neighbours
    o2, e2, acc_o, acc_e = [], [], 0.0, 0.0
    for a, b in zip(obs, exp):
        acc_o += a
        acc_e += b
        if acc_e >= 5.0:
            o2.append(acc_o)
            e2.append(acc_e)
            acc_o = acc_e = 0.0
    if acc_e > 0:
        o2[-1] += acc_o
        e2[-1] += acc_e
    o2, e2 = np.array(o2), np.array(e2)
    if len(o2) > 1:
        chi2 = float(np.sum((o2 - e2) ** 2 / e2))
        assert stats.chi2.sf(chi2, len(o2) - 1) > 1e-4, (lam, chi2)


# ---- seed ensembles ------------------------------------------------------------
def heated_tube(seed, mixed=False, heating=True):
    mi, spec, tube, vg = grids.config_small(n_particles=4000, three_d=True,
                                            steps_per_master=5, heating=heating,
                                            collisions=True)
    mi = dataclasses.replace(mi, seed=seed)
    if mixed:
        mi = dataclasses.replace(mi, precision=KAOS_PREC_MIXED)
    init = grids.initial_particles(tube, spec, mi, seed=3)
    return mi, tube, vg, init


def run_oracle(seed, heating=True):
    mi, tube, vg, init = heated_tube(seed, heating=heating)
    o = Oracle(mi, tube, vg)
    o.load(*init)
    o.step(STEPS)
    return o


def run_gpu(seed):
    mi, tube, vg, init = heated_tube(seed, mixed=True)
    s = Solver(mi, [tube], vg)
    s.load(0, *init)
    s.step(STEPS)
    return s


def moments(r):
    return np.stack([r.moments(m) for m in MOMENTS])


@pytest.fixture(scope="module")
def ensembles():
    mo = np.stack([moments(run_oracle(1 + k)) for k in range(ENSEMBLE)])
    mg = np.stack([moments(run_gpu(1001 + k)) for k in range(ENSEMBLE)])
    return mo, mg


def _worst(z, live, mu_a, mu_b, sd_a, sd_b, k=5):
    """The k largest deviations: (z, moment, cell, mean a, mean b, sd a, sd b)."""
    idx = np.argwhere(live)
    order = np.argsort(z)[::-1][:k]
    return [(round(float(z[o]), 2), MOMENTS[idx[o][0]], int(idx[o][1]),
             float(mu_a[tuple(idx[o])]), float(mu_b[tuple(idx[o])]),
             float(sd_a[tuple(idx[o])]), float(sd_b[tuple(idx[o])])) for o in order]


def test_ensemble_means_agree(ensembles):
    mo, mg = ensembles
    K = ENSEMBLE
    mu_o, mu_g = mo.mean(0), mg.mean(0)
    sd_o, sd_g = mo.std(0, ddof=1), mg.std(0, ddof=1)
    # standard error of the difference of means, with a floor of 1e-9 of the
    # moment's scale (entries whose spread is rounding noise)
    scale = np.max(np.abs(mu_o), axis=1, keepdims=True)
    se = np.sqrt((sd_o ** 2 + sd_g ** 2) / K + (1e-9 * scale) ** 2)
    live = (sd_o > 0) | (sd_g > 0)
    # entries without spread are deterministic: equal on both sides
    assert np.all(np.abs(mu_g - mu_o)[~live] <= 1e-6 * np.broadcast_to(scale, mu_o.shape)[~live])
    z = np.abs(mu_g - mu_o)[live] / se[live]
    assert live.sum() > 100
    worst = _worst(z, live, mu_o, mu_g, sd_o, sd_g)
    assert np.mean(z > 3.0) <= 0.02, worst
    assert z.max() < 5.0, worst


def test_single_gpu_run_within_3_sigma(ensembles):
    mo, _ = ensembles
    K = ENSEMBLE
    mu, sd = mo.mean(0), mo.std(0, ddof=1)
    m = moments(run_gpu(777))
    live = sd > 0
    scale = np.max(np.abs(mu), axis=1, keepdims=True)
    se = np.sqrt(sd ** 2 * (1.0 + 1.0 / K) + (1e-9 * scale) ** 2)
    z = np.abs(m - mu)[live] / se[live]
    worst = _worst(z, live, mu, m, sd, sd)
    assert np.mean(z > 3.0) <= 0.03, worst
    assert z.max() < 6.0, worst


def ks_samples(r):
    p = r.particles()
    return p["qind"], p["vpar"], p["vperp1"], p["vperp2"]


def test_distribution_function_ks():
    g = ks_samples(run_gpu(4242))
    o = ks_samples(run_oracle(4343))
    cold = ks_samples(run_oracle(4343, heating=False))
    # pooled marginals: same law; a heated run against an unheated one differs
    for a in (1, 2, 3):
        assert stats.ks_2samp(g[a], o[a]).pvalue > 1e-3, a
    assert stats.ks_2samp(g[2], cold[2]).pvalue < 1e-6
    # per cell: V||, Vperp1, Vperp2 of every cell holding >= 80 ions
    pv = []
    for c in np.unique(o[0]):
        if c < 0:
            continue
        mg, mo_ = g[0] == c, o[0] == c
        if mg.sum() < 80 or mo_.sum() < 80:
            continue
        for a in (1, 2, 3):
            pv.append(stats.ks_2samp(g[a][mg], o[a][mo_]).pvalue)
    pv = np.array(pv)
    assert len(pv) >= 30
    assert np.mean(pv < 0.01) <= 0.05, np.sort(pv)[:10]
    assert pv.min() > 1e-5
