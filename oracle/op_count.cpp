/*
 * op_count.cpp -- op-counting build of the CPU oracle.  TEST AND
 * MEASUREMENT INFRASTRUCTURE ONLY: it compiles kaos_oracle.c unchanged as
 * C++ with every `double` replaced by `opd`, a double that counts the
 * arithmetic done on it, so that the oracle's own code gives the FP64
 * flop-equivalents of one particle-step of the reference formulation
 * (F_alg).  It computes the same values as the plain oracle (every
 * operation is the same single IEEE operation in the same order, no
 * contraction); tests check that bit for bit.
 *
 * Weights (fixed; the counts are reported per class, the weighted sum is
 * F_alg):
 *   add, sub, mul = 1;  div, sqrt = 4;  each transcendental call = 20
 *   (acos asin atan atan2 cos sin exp log pow, complex acos and cos).
 *   fabs, negation, comparisons, conversions: 0.
 * Complex operations of the quartic's resolvent cubic
 * (_8_1_4_RK4DipolePolynomialSolver.f90:30-84) count as the real
 * operations a compiler emits for them: complex +- real 1 add;
 * complex * real 2 mul; complex / real 2 div; real / complex 4 mul, 1 add,
 * 2 div; complex * complex 4 mul, 2 add; complex +- complex 2 add.
 * Operations on compile-time constants (pi, R_E, the dipole moment) fold
 * away as in the reference, where they are Fortran parameters
 * (_ModelInput.f90:35-43); the cell and field searches, whose orientation
 * products stand for the reference's two branches of plain comparisons
 * (_8_1_1_KineticUpdateA.f90:221-273), are not counted.
 *
 * Counts are kept per phase of a step: ion push, ENA push, charge
 * exchange, master-step work (fields, removal, injection, counts,
 * moments).
 */
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <type_traits>

#include "../include/kaos_philox.h"

namespace {

enum { OP_ADD, OP_MUL, OP_DIV, OP_SQRT, OP_TRANS, OP_N };
enum { NPHASE = 4 };
int64_t g_ops[NPHASE][OP_N];
int g_phase = 0;
int g_search = 0;

inline void cnt(int k, int64_t n = 1) {
  if (!g_search)
    g_ops[g_phase][k] += n;
}

} // namespace

struct opd {
  double v;
  opd() = default;
  constexpr opd(double x) : v(x) {}
  template <class T, class = typename std::enable_if<std::is_arithmetic<T>::value>::type>
  explicit constexpr operator T() const {
    return static_cast<T>(v);
  }
};
static_assert(sizeof(opd) == sizeof(double), "layout of the C structs");
static_assert(std::is_trivially_copyable<opd>::value, "memcpy of arrays");

inline opd operator+(opd a, opd b) { cnt(OP_ADD); return opd(a.v + b.v); }
inline opd operator-(opd a, opd b) { cnt(OP_ADD); return opd(a.v - b.v); }
inline opd operator*(opd a, opd b) { cnt(OP_MUL); return opd(a.v * b.v); }
inline opd operator/(opd a, opd b) { cnt(OP_DIV); return opd(a.v / b.v); }
inline opd operator-(opd a) { return opd(-a.v); }
inline opd operator+(opd a) { return a; }
inline opd &operator+=(opd &a, opd b) { return a = a + b; }
inline opd &operator-=(opd &a, opd b) { return a = a - b; }
inline opd &operator*=(opd &a, opd b) { return a = a * b; }
inline opd &operator/=(opd &a, opd b) { return a = a / b; }
inline bool operator<(opd a, opd b) { return a.v < b.v; }
inline bool operator<=(opd a, opd b) { return a.v <= b.v; }
inline bool operator>(opd a, opd b) { return a.v > b.v; }
inline bool operator>=(opd a, opd b) { return a.v >= b.v; }
inline bool operator==(opd a, opd b) { return a.v == b.v; }
inline bool operator!=(opd a, opd b) { return a.v != b.v; }

inline opd sqrt(opd a) { cnt(OP_SQRT); return opd(std::sqrt(a.v)); }
inline opd fabs(opd a) { return opd(std::fabs(a.v)); }
#define ORC_T1(fn)                                                             \
  inline opd fn(opd a) {                                                       \
    cnt(OP_TRANS);                                                             \
    return opd(std::fn(a.v));                                                  \
  }
ORC_T1(acos)
ORC_T1(asin)
ORC_T1(atan)
ORC_T1(cos)
ORC_T1(sin)
ORC_T1(exp)
ORC_T1(log)
#undef ORC_T1
inline opd atan2(opd a, opd b) { cnt(OP_TRANS); return opd(std::atan2(a.v, b.v)); }
inline opd pow(opd a, opd b) { cnt(OP_TRANS); return opd(std::pow(a.v, b.v)); }
inline long lround(opd a) { return std::lround(a.v); }
inline long long llround(opd a) { return std::llround(a.v); }
inline opd floor(opd a) { return opd(std::floor(a.v)); }
inline int isfinite(opd a) { return std::isfinite(a.v); }
inline int isnan(opd a) { return std::isnan(a.v); }

/* complex values through std::complex<double>, whose operators and
 * acos/cos are the C99 ones (same results as the plain build) */
struct orc_cplx {
  std::complex<double> z;
};
inline orc_cplx operator*(orc_cplx a, opd b) { cnt(OP_MUL, 2); return {a.z * b.v}; }
inline orc_cplx operator*(opd a, orc_cplx b) { cnt(OP_MUL, 2); return {a.v * b.z}; }
inline orc_cplx operator*(orc_cplx a, orc_cplx b) {
  cnt(OP_MUL, 4);
  cnt(OP_ADD, 2);
  return {a.z * b.z};
}
inline orc_cplx operator/(orc_cplx a, opd b) { cnt(OP_DIV, 2); return {a.z / b.v}; }
inline orc_cplx operator/(opd a, orc_cplx b) {
  cnt(OP_MUL, 4);
  cnt(OP_ADD, 1);
  cnt(OP_DIV, 2);
  return {a.v / b.z};
}
inline orc_cplx operator+(orc_cplx a, opd b) { cnt(OP_ADD); return {a.z + b.v}; }
inline orc_cplx operator-(orc_cplx a, opd b) { cnt(OP_ADD); return {a.z - b.v}; }
inline orc_cplx orc_cacos(orc_cplx a) { cnt(OP_TRANS); return {std::acos(a.z)}; }
inline orc_cplx orc_ccos(orc_cplx a) { cnt(OP_TRANS); return {std::cos(a.z)}; }
inline opd orc_creal(orc_cplx a) { return opd(a.z.real()); }
static inline orc_cplx orc_i() { return {std::complex<double>(0.0, 1.0)}; }
#define ORC_I orc_i()

/* uniforms: the random-number generator is not arithmetic of the
 * formulation (the reference calls random_number) */
static inline opd orc_u01_counted(uint32_t hi, uint32_t lo) { return opd(kaos_u01(hi, lo)); }
#define kaos_u01 orc_u01_counted

#define ORC_OPS_COUNTED 1
#define ORC_PHASE(ph) (g_phase = (ph))
#define ORC_SEARCH_BEGIN() (++g_search)
#define ORC_SEARCH_END() (--g_search)

#define double opd
extern "C" {
#include "kaos_oracle.c"
}
#undef double

extern "C" {

/* Zero the counters. */
void orc_ops_reset(void) {
  memset(g_ops, 0, sizeof g_ops);
  g_search = 0;
}

/* out[NPHASE * 5]: per phase (ion push, ENA push, charge exchange, master)
 * the counts of add, mul, div, sqrt and transcendental calls. */
void orc_ops_get(int64_t *out) { memcpy(out, g_ops, sizeof g_ops); }

}
