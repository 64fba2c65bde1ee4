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
