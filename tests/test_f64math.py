"""The table-reduced FP64 functions of kaos_b200/csrc/kaos_f64.cuh (the
heating kick of precision mode KAOS_PREC_MIXED_K64) against the C library's
long double functions, over the input ranges the kick uses, within two
units of 2^-52: logarithms absolute (relative beyond 1 in magnitude, and
next to 1), the exponential relative, sine and cosine absolute.  Their host
build (the same source; only the FP32 seed that picks the table point
differs on the device, which cannot change the result beyond rounding).
The device build is compared with the FP64 push's own Gaussian pair in
tests/test_gpu_stats.py."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER_DIR = os.path.join(ROOT, "kaos_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <cstdint>
#include <cmath>
#include "kaos_f64.cuh"
using namespace kaos;

static uint64_t st = 0x9E3779B97F4A7C15ull;
static double urand() {  // splitmix64 -> (0, 1)
  uint64_t z = (st += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return ((double)(z >> 11) + 0.5) * 0x1.0p-53;
}
static double rel(long double a, long double b) {
  long double d = fabsl(a - b), s = fabsl(b);
  return (double)(s > 0 ? d / s : d);
}
// error of a logarithm: absolute below 1 in magnitude, relative above (an
// absolute error in the logarithm is a relative error of what it scales)
static double lerr(long double a, long double b) {
  long double d = fabsl(a - b), s = fabsl(b);
  return (double)(s > 1 ? d / s : d);
}

int main() {
  double p2[KF_N + 1], cs[2 * (KF_N + 1)];
  const long double twopi = 6.283185307179586476925286766559L;
  for (int i = 0; i <= KF_N; ++i) {
    p2[i] = (double)exp2l((long double)i / KF_N);
    cs[2 * i] = (double)cosl(twopi * i / KF_N);
    cs[2 * i + 1] = (double)sinl(twopi * i / KF_N);
  }
  const int N = 2000000;
  double e_ln = 0, e_ln1 = 0, e_log2 = 0, e_exp2 = 0, e_sc = 0;
  for (int k = 0; k < N; ++k) {
    // ln of a 53-bit uniform (the Box-Muller radius), log-spread too
    double u = urand();
    e_ln = fmax(e_ln, lerr(kf_ln(p2, u), logl((long double)u)));
    double v = exp2(-53.0 * urand());
    e_ln = fmax(e_ln, lerr(kf_ln(p2, v), logl((long double)v)));
    // arguments next to 1 (table point 0): relative accuracy of the small
    // logarithm
    double w = 1.0 - (double)(k % 4096 + 1) * 0x1.0p-53;
    double w2 = 1.0 + (double)(k % 4096 + 1) * 0x1.0p-52;
    e_ln1 = fmax(e_ln1, rel(kf_ln(p2, w), logl((long double)w)));
    e_ln1 = fmax(e_ln1, rel(kf_ln(p2, w2), logl((long double)w2)));
    // log2 over many octaves (Om/Om0, y Sig^-6)
    double x = exp2(200.0 * (urand() - 0.5));
    e_log2 = fmax(e_log2, lerr(kf_log2(p2, x), log2l((long double)x)));
    // exp2 of the kick exponent's range
    double E = 120.0 * (urand() - 0.5);
    e_exp2 = fmax(e_exp2, rel(kf_exp2(p2, E), exp2l((long double)E)));
    // sin, cos of 2 pi u: absolute error
    double s, c, a = urand();
    kf_sincos2pi(cs, a, s, c);
    e_sc = fmax(e_sc, (double)fabsl(s - sinl(twopi * a)));
    e_sc = fmax(e_sc, (double)fabsl(c - cosl(twopi * a)));
  }
  double s, c;  // the end points of the table
  kf_sincos2pi(cs, 0.0, s, c);
  e_sc = fmax(e_sc, fmax(fabs(s), fabs(c - 1.0)));
  kf_sincos2pi(cs, 1.0, s, c);
  e_sc = fmax(e_sc, fmax(fabs(s - (double)sinl(twopi)), fabs(c - 1.0)));
  printf("%.3e %.3e %.3e %.3e %.3e\n", e_ln, e_ln1, e_log2, e_exp2, e_sc);
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_table_reduced_functions_accuracy(tmp_path):
    src = tmp_path / "f64math_check.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "f64math_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", HEADER_DIR, str(src), "-o", str(exe),
                    "-lm"], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    e_ln, e_ln1, e_log2, e_exp2, e_sc = (float(t) for t in out.split())
    eps = 2.0 ** -52  # one unit in the last place at 1
    assert e_ln < 2 * eps, e_ln        # ln of uniforms (absolute below 1)
    assert e_ln1 < 2 * eps, e_ln1      # ln next to 1, relative
    assert e_log2 < 2 * eps, e_log2    # log2 (absolute below 1)
    assert e_exp2 < 2 * eps, e_exp2    # exp2, relative
    assert e_sc < 2 * eps, e_sc        # sin, cos of 2 pi u, absolute


def test_log_form_kick_equals_the_reference_form():
    """The log form of the FP64 kick (heat64t: K G 2^E, E = -c log2(Om/Om0) +
    log2(y Sig^-6)/4, y = Om |V||| / sum ds, applied while y <= (2 pi/h)^2)
    equals heat()'s form K x^-c sqrt(Om s) Sig^-3/2 G, x = Om/Om0,
    s = sqrt(|V||| / (Om sum ds)), applied while h Om s <= 2 pi (the
    reference's (h/tau) sqrt(2 D tau) G, _8_1_1_0_WaveHeating.f90:141-150,
    with D's Sig^-3 factor), over random arguments of the kick's ranges."""
    import numpy as np
    rng = np.random.default_rng(3)
    n = 20000
    Om = 10.0 ** rng.uniform(0.5, 3.0, n)
    Om0 = 10.0 ** rng.uniform(1.5, 2.5, n)
    vabs = 10.0 ** rng.uniform(-2.0, 4.5, n)
    sumds = 10.0 ** rng.uniform(5.0, 7.5, n)
    c = rng.uniform(0.2, 1.2, n)
    sig = np.where(rng.uniform(size=n) < 0.5, 1.0, 10.0 ** rng.uniform(0.0, 2.0, n))
    h = 0.005
    s = np.sqrt(vabs / (Om * sumds))
    ref = (Om / Om0) ** (-c) * np.sqrt(Om * s) * sig ** -1.5
    on_ref = h * Om * s <= 2.0 * np.pi
    y = Om * vabs / sumds
    E = -c * np.log2(Om / Om0) + 0.25 * np.log2(y * sig ** -6.0)
    on_log = y <= (2.0 * np.pi / h) ** 2
    # the branch agrees except within rounding of its threshold
    edge = np.abs(h * Om * s / (2.0 * np.pi) - 1.0) < 1e-12
    assert np.array_equal(on_ref[~edge], on_log[~edge])
    np.testing.assert_allclose(2.0 ** E, ref, rtol=1e-12)
