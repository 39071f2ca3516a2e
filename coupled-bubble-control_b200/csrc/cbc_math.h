// cbc_math.h -- FP64 elementary functions shared by the CUDA kernels and the
// CPU oracle.
//
// Why not libm / CUDA's libdevice: the integrator is compared against its CPU
// oracle bit for bit.  That only works if both sides evaluate sin, cos, exp and
// log with the same operations in the same order.  These routines use only
// IEEE-754 add, mul, fma, division and exact bit manipulation, so gcc (with
// -ffp-contract=off) and nvcc (with -fmad=false) produce identical results.
//
// Methods (all published, coefficients are the exact Taylor coefficients
// rounded to double, computed with mpmath; no vendor constants are used):
//   * sin/cos: Cody & Waite additive argument reduction by pi/2 with a
//     three-part split of pi/2 applied through fma (W. J. Cody, W. Waite,
//     "Software Manual for the Elementary Functions", 1980, ch. 8), followed by
//     Taylor polynomials on |r| <= pi/4 (sin to r^19, cos to r^18; truncation
//     < 1e-19 relative).  Valid for |x| < 2^20 (accuracy degrades gracefully
//     beyond); the integrator's phase arguments stay below 2e5.
//   * exp: reduction x = n ln2 + r, |r| <= ln2/2, two-part ln2 through fma,
//     Taylor polynomial to r^13 (truncation < 1e-17), scaling by 2^n built from
//     the exponent bits (Cody & Waite ch. 6).
//   * log: x = 2^e m, m in [sqrt(2)/2, sqrt(2)), log m = 2 atanh(f),
//     f = (m-1)/(m+1), odd series to f^23 (Cody & Waite ch. 5).
//   * pow(x, y) for x > 0 as exp(y log x).
// Accuracy against glibc (checked by tests/test_cbc_math.py): sin/cos/exp/log
// within 2 ulp; pow within ~1e-15 relative for |y log x| < 50.
#pragma once

#include <stdint.h>
#include <math.h>
#if !defined(__CUDACC__)
#include <string.h>
#endif

#if defined(__CUDACC__)
#define CBC_HD __host__ __device__ __forceinline__
#else
#define CBC_HD static inline
#endif

// Coefficient tables.  On the device they live in constant memory, so FP64
// fma instructions take them as constant-bank operands instead of
// rematerialising every 64-bit immediate in registers; the host (and the CPU
// oracle) reads the identical constexpr values.
#if defined(__CUDACC__)
#define CBCM_TABLE(name, ...)                                  \
  static constexpr double name##_h[] = {__VA_ARGS__};          \
  static __constant__ const double name##_d[] = {__VA_ARGS__};
#else
#define CBCM_TABLE(name, ...) static constexpr double name##_h[] = {__VA_ARGS__};
#endif
#if defined(__CUDA_ARCH__)
#define CBCM_K(name, i) (name##_d[i])
#else
#define CBCM_K(name, i) (name##_h[i])
#endif

namespace cbcm {

CBC_HD double bits_to_double(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double d;
  memcpy(&d, &u, sizeof(d));
  return d;
#endif
}

CBC_HD uint64_t double_to_bits(double d) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(d);
#else
  uint64_t u;
  memcpy(&u, &d, sizeof(u));
  return u;
#endif
}

CBC_HD double fma_(double a, double b, double c) { return fma(a, b, c); }
CBC_HD double rint_(double a) { return rint(a); }
CBC_HD double fabs_(double a) { return fabs(a); }
CBC_HD bool isfinite_(double a) {
  // exponent field all ones <=> inf or nan
  return ((double_to_bits(a) >> 52) & 0x7ff) != 0x7ff;
}

// pi/2 = PIO2_1 + PIO2_2 + PIO2_3 (each the nearest double of the remainder)
static constexpr double PIO2_1 = 0x1.921fb54442d18p+0;
static constexpr double PIO2_2 = 0x1.1a62633145c07p-54;
static constexpr double PIO2_3 = -0x1.f1976b7ed8fbcp-110;
static constexpr double TWO_OVER_PI = 0x1.45f306dc9c883p-1;

// sin(r) = r + r z (S3 + z (S5 + ...)),  z = r^2,  S_n = (-1)^((n-1)/2) / n!
static constexpr double S3 = -0x1.5555555555555p-3;
static constexpr double S5 = 0x1.1111111111111p-7;
static constexpr double S7 = -0x1.a01a01a01a01ap-13;
static constexpr double S9 = 0x1.71de3a556c734p-19;
static constexpr double S11 = -0x1.ae64567f544e4p-26;
static constexpr double S13 = 0x1.6124613a86d09p-33;
static constexpr double S15 = -0x1.ae7f3e733b81fp-41;
static constexpr double S17 = 0x1.952c77030ad4ap-49;
static constexpr double S19 = -0x1.2f49b46814157p-57;
// cos(r) = 1 + z (C2 + z (C4 + ...)),  C_n = (-1)^(n/2) / n!
static constexpr double C2 = -0x1.0000000000000p-1;
static constexpr double C4 = 0x1.5555555555555p-5;
static constexpr double C6 = -0x1.6c16c16c16c17p-10;
static constexpr double C8 = 0x1.a01a01a01a01ap-16;
static constexpr double C10 = -0x1.27e4fb7789f5cp-22;
static constexpr double C12 = 0x1.1eed8eff8d898p-29;
static constexpr double C14 = -0x1.93974a8c07c9dp-37;
static constexpr double C16 = 0x1.ae7f3e733b81fp-45;
static constexpr double C18 = -0x1.6827863b97d97p-53;

CBCM_TABLE(SC_RED, PIO2_1, PIO2_2, PIO2_3, TWO_OVER_PI)
CBCM_TABLE(SIN_P, S3, S5, S7, S9, S11, S13, S15, S17, S19)
CBCM_TABLE(COS_P, C2, C4, C6, C8, C10, C12, C14, C16, C18)

// sin and cos of x together.  NaN/inf input gives NaN outputs.
// Branch-free: the main path runs on a sanitised argument and the special
// case is selected at the end (lets the compiler interleave independent calls).
CBC_HD void sincos(double x_in, double* s, double* c) {
  const bool fin = isfinite_(x_in);
  const double x = fin ? x_in : 0.0;
  double kd = rint_(x * CBCM_K(SC_RED, 3));
  double r = fma_(-kd, CBCM_K(SC_RED, 0), x);
  r = fma_(-kd, CBCM_K(SC_RED, 1), r);
  r = fma_(-kd, CBCM_K(SC_RED, 2), r);
  double z = r * r;
  // Horner from the highest coefficient down (S19 ... S3, C18 ... C2)
  double ps = fma_(CBCM_K(SIN_P, 8), z, CBCM_K(SIN_P, 7));
#pragma unroll
  for (int i = 6; i >= 0; --i) ps = fma_(ps, z, CBCM_K(SIN_P, i));
  double sr = fma_(r * z, ps, r);
  double pc = fma_(CBCM_K(COS_P, 8), z, CBCM_K(COS_P, 7));
#pragma unroll
  for (int i = 6; i >= 0; --i) pc = fma_(pc, z, CBCM_K(COS_P, i));
  double cr = fma_(z, pc, 1.0);
  // quadrant q = k mod 4 from the low two bits of k (two's complement keeps
  // k mod 4 in the low bits for negative k).
  //   q=0: ( s,  c)   q=1: ( c, -s)   q=2: (-s, -c)   q=3: (-c,  s)
  long long ki = (long long)kd;
  int q = (int)(ki & 3);
  double a = (q & 1) ? cr : sr;
  double b = (q & 1) ? sr : cr;
  const double nan_ = x_in - x_in;  // NaN for +-inf and NaN
  *s = fin ? ((q & 2) ? -a : a) : nan_;
  *c = fin ? (((q + 1) & 2) ? -b : b) : nan_;
}

static constexpr double LOG2E = 0x1.71547652b82fep+0;
static constexpr double LN2_HI = 0x1.62e42fefa39efp-1;
static constexpr double LN2_LO = 0x1.abc9e3b39803fp-56;
static constexpr double E2 = 0x1.0000000000000p-1;
static constexpr double E3 = 0x1.5555555555555p-3;
static constexpr double E4 = 0x1.5555555555555p-5;
static constexpr double E5 = 0x1.1111111111111p-7;
static constexpr double E6 = 0x1.6c16c16c16c17p-10;
static constexpr double E7 = 0x1.a01a01a01a01ap-13;
static constexpr double E8 = 0x1.a01a01a01a01ap-16;
static constexpr double E9 = 0x1.71de3a556c734p-19;
static constexpr double E10 = 0x1.27e4fb7789f5cp-22;
static constexpr double E11 = 0x1.ae64567f544e4p-26;
static constexpr double E12 = 0x1.1eed8eff8d898p-29;
static constexpr double E13 = 0x1.6124613a86d09p-33;

CBCM_TABLE(EXP_RED, LOG2E, LN2_HI, LN2_LO)
CBCM_TABLE(EXP_P, E2, E3, E4, E5, E6, E7, E8, E9, E10, E11, E12, E13)

// 2^n for integer n in [-1022, 1023] (exact)
CBC_HD double pow2i(int n) { return bits_to_double((uint64_t)(n + 1023) << 52); }

// Branch-free (special cases selected at the end); the scaling by 2^n is
// split in two factors so that results in the subnormal range round once
// (the second factor is exactly 1 when |n| <= 1000).
CBC_HD double exp(double x_in) {
  const bool big = !(x_in < 709.8);  // also NaN and +inf
  const bool tiny = x_in < -745.2;
  const double x = (big || tiny) ? 0.0 : x_in;
  double nd = rint_(x * CBCM_K(EXP_RED, 0));
  double r = fma_(-nd, CBCM_K(EXP_RED, 1), x);
  r = fma_(-nd, CBCM_K(EXP_RED, 2), r);
  // Horner E13 ... E2, then 1, 1
  double p = fma_(CBCM_K(EXP_P, 11), r, CBCM_K(EXP_P, 10));
#pragma unroll
  for (int i = 9; i >= 0; --i) p = fma_(p, r, CBCM_K(EXP_P, i));
  p = fma_(p, r, 1.0);
  p = fma_(p, r, 1.0);
  const int n = (int)nd;
  const int n1 = n > 1000 ? 1000 : (n < -1000 ? -1000 : n);
  const double res = (p * pow2i(n1)) * pow2i(n - n1);
  const double ovf = (x_in != x_in) ? x_in : bits_to_double(0x7ff0000000000000ULL);
  return big ? ovf : (tiny ? 0.0 : res);
}

static constexpr double SQRT1_2 = 0x1.6a09e667f3bcdp-1;
static constexpr double L3 = 0x1.5555555555555p-2;
static constexpr double L5 = 0x1.999999999999ap-3;
static constexpr double L7 = 0x1.2492492492492p-3;
static constexpr double L9 = 0x1.c71c71c71c71cp-4;
static constexpr double L11 = 0x1.745d1745d1746p-4;
static constexpr double L13 = 0x1.3b13b13b13b14p-4;
static constexpr double L15 = 0x1.1111111111111p-4;
static constexpr double L17 = 0x1.e1e1e1e1e1e1ep-5;
static constexpr double L19 = 0x1.af286bca1af28p-5;
static constexpr double L21 = 0x1.8618618618618p-5;
static constexpr double L23 = 0x1.642c8590b2164p-5;

CBCM_TABLE(LOG_P, L3, L5, L7, L9, L11, L13, L15, L17, L19, L21, L23)
CBCM_TABLE(LOG_C, LN2_HI, LN2_LO)

// Branch-free (special cases selected at the end).
CBC_HD double log(double x_in) {
  const bool pos = x_in > 0.0;  // false for +-0, negatives and NaN
  const bool main_path = pos && isfinite_(x_in);
  double x = main_path ? x_in : 1.0;
  const bool sub = x < 0x1p-1022;  // subnormal: scale into the normal range (exact)
  x = sub ? x * 0x1p54 : x;
  const int eadj = sub ? -54 : 0;
  uint64_t u = double_to_bits(x);
  int e = (int)((u >> 52) & 0x7ff) - 1023;
  // m in [1, 2)
  double m = bits_to_double((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
  const bool hi = m > 2.0 * SQRT1_2;
  m = hi ? m * 0.5 : m;
  e += hi ? 1 : 0;
  e += eadj;
  double f = (m - 1.0) / (m + 1.0);
  double s = f * f;
  // Horner L23 ... L3
  double p = fma_(CBCM_K(LOG_P, 10), s, CBCM_K(LOG_P, 9));
#pragma unroll
  for (int i = 8; i >= 0; --i) p = fma_(p, s, CBCM_K(LOG_P, i));
  double f2 = f + f;
  double logm = fma_(f2 * s, p, f2);
  double ed = (double)e;
  const double res = fma_(ed, CBCM_K(LOG_C, 0), fma_(ed, CBCM_K(LOG_C, 1), logm));
  // x == 0: -inf; x < 0 or NaN: NaN; +inf: +inf
  const double special = (x_in == 0.0) ? -bits_to_double(0x7ff0000000000000ULL)
                                       : (pos ? x_in : bits_to_double(0x7ff8000000000000ULL));
  return main_path ? res : special;
}

// x^y for x > 0 (x <= 0 gives NaN, matching the physical meaning of a
// collapsed radius).
CBC_HD double pow_pos(double x, double y) { return cbcm::exp(y * cbcm::log(x)); }

}  // namespace cbcm
