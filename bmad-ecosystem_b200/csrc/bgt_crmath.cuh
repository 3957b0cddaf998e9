// bgt_crmath.cuh -- correctly rounded FP64 sin, cos, sinh, cosh, exp, asin, atan2 for the
// tracker's device code (and, compiled for the host, for testing).
//
// Why: the exact sector-bend map (track_a_bend.f90:163-209) cancels
// O(L^2 g) ~ 5e-2 terms to produce O(1e-3) coordinates, so a one-ulp change
// in sin/asin/atan2 moves the orbit by ~1e-13 relative per bend.  The
// reference evaluates these with the platform libm (glibc), which is
// correctly rounded in nearly every case on the arguments used here; a
// correctly rounded device implementation therefore reproduces the
// reference's values, where the CUDA math library (a few ulp) does not.
//
// Method (Ziv's strategy: fast path + rounding test + accurate path):
//   fast path   the leading Taylor terms in double-double, the tail in
//               double; error bound e; if both v - e and v + e round to the
//               same double, that double is the correctly rounded result.
//   slow path   full double-double Taylor evaluation after Cody-Waite
//               argument reduction (sin/cos), argument halving (atan) or
//               the half-angle identity (asin), on the argument itself for
//               sinh/cosh/exp (|x| <= 2): error ~2^-100, then round.
// Arguments beyond the documented ranges (|x| >= 2^19 for sin/cos,
// non-finite values, extreme atan2 exponents) use the CUDA / C library
// function.
#pragma once
#include <math.h>

#include "bgt_crmath_tables.h"

#ifdef __CUDACC__
#define BGT_HD __host__ __device__ __forceinline__
// accurate paths run rarely: kept out of line so the hot loop stays small
#define BGT_HD_NOINLINE static __host__ __device__ __noinline__
#else
#define BGT_HD static inline
#define BGT_HD_NOINLINE static __attribute__((noinline))
#endif

namespace bgt {
namespace cr {

struct dd {
  double hi, lo;
};

BGT_HD dd two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}
BGT_HD dd fast_two_sum(double a, double b) {  // |a| >= |b|
  double s = a + b;
  return {s, b - (s - a)};
}
BGT_HD dd two_prod(double a, double b) {
  double p = a * b;
  return {p, fma(a, b, -p)};
}
BGT_HD dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}
BGT_HD dd dd_add_d(dd a, double b) {
  dd s = two_sum(a.hi, b);
  s.lo += a.lo;
  return fast_two_sum(s.hi, s.lo);
}
BGT_HD dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo = fma(a.hi, b.lo, fma(a.lo, b.hi, p.lo));
  return fast_two_sum(p.hi, p.lo);
}
BGT_HD dd dd_mul_d(dd a, double b) {
  dd p = two_prod(a.hi, b);
  p.lo = fma(a.lo, b, p.lo);
  return fast_two_sum(p.hi, p.lo);
}
BGT_HD dd dd_c(const double c[2]) { return {c[0], c[1]}; }
BGT_HD dd dd_neg(dd a) { return {-a.hi, -a.lo}; }
BGT_HD dd dd_div(dd a, dd b) {
  double q1 = a.hi / b.hi;
  dd r = dd_add(a, dd_neg(dd_mul_d(b, q1)));
  double q2 = r.hi / b.hi;
  r = dd_add(r, dd_neg(dd_mul_d(b, q2)));
  double q3 = r.hi / b.hi;
  return dd_add_d(fast_two_sum(q1, q2), q3);
}
BGT_HD dd dd_sqrt(dd a) {
  if (a.hi <= 0) return {sqrt(a.hi), 0.0};
  double s = sqrt(a.hi);
  dd sq = two_prod(s, s);
  double r = (((a.hi - sq.hi) - sq.lo) + a.lo) / (2 * s);
  return fast_two_sum(s, r);
}

// Round v to double if every value within +/- err of v rounds the same way.
BGT_HD bool round_test(dd v, double err, double* out) {
  double a = v.hi + (v.lo - err);
  double b = v.hi + (v.lo + err);
  if (a == b) {
    *out = a;
    return true;
  }
  return false;
}

// ---- light fast paths for small arguments, 2^-27 <= |x| <= 2^-4 ----
//
// Every particle-dependent argument in a bend step (phi_1 = asin(px/pt),
// angle + phi_1, the atan2 ratio, the exit angle) and the per-step focusing
// phase of a quadrupole is a few 1e-2 or smaller, where one plain-double
// polynomial already lands within a few thousandths of an ulp.  u = 2^-53.
//
// Odd series  f(x) = x + x y P(y),  y = fl(x^2),
//             P(y) = C[1] + C[2] y + ... + C[K] y^(K-1)  (Horner, plain double).
//   |x y P| <= |x| y / 3 <= 1.3e-3 |x|.  Relative error of the computed
//   correction c: y (u), x*y (u), P (2u + O(u y): the C[1] rounding and the
//   final add dominate), the product (u) -> < 6.1u < 8u = 2^-50.  The
//   omitted terms are < 2^-70 |x| for the K used (sin/sinh K=5: < y^6/13!;
//   asin K=8: < 0.0098 y^9; atan K=8: < y^9/19), and 2^-69 |x| also covers
//   the roundings inside round_test.  hi + lo = x + c exactly (|x| >= |c|).
// Even series f(x) = 1 + C[1] y + y^2 Q(y), C[1] = -1/2 (cos) or 1/2 (cosh)
//   is a power of two, so C[1] (yh + yl) with yh + yl = x^2 (two_prod) is
//   exact; t = yh^2 Q(yh) carries < 6u relative error; the two roundings
//   in the low word are < |t| 2^-53 + 2^-105; omitted terms < y^6/12! < 2^-77.
//
// Below 2^-27, |x|^3/6 (asin, sinh: x^3/6; atan: x^3/3) is below half an ulp
// of x and x^2/2 below half an ulp of 1, so the correctly rounded value is
// x (odd) or 1 (even); that also keeps every product here normal.
//
// The polynomials are evaluated by Estrin's scheme with fused multiply-adds
// (independent pairs first, then powers y^2, y^4): the same terms with a
// dependency chain of depth ~log2(K) instead of K.  Its rounding error is of
// the Horner bound's order: every partial sum is the leading coefficient plus
// terms smaller by y <= 2^-8, so P still carries < 2u + O(u y) relative
// error, within the 8u of the bounds above.

// C[f] + C[f+1] y + ... + C[K] y^(K-f) by Estrin's scheme (fused multiply-adds)
template <int F, int K>
BGT_HD double poly_estrin(double y, const double (*C)[2]) {
  constexpr int N = K - F + 1;  // number of coefficients: 4, 5 or 8
  static_assert(N == 4 || N == 5 || N == 8, "poly_estrin: 4, 5 or 8 coefficients");
  const double y2 = y * y;
  const double b0 = fma(C[F + 1][0], y, C[F][0]);
  const double b1 = fma(C[F + 3][0], y, C[F + 2][0]);
  if constexpr (N == 4) {
    return fma(b1, y2, b0);
  } else {
    const double y4 = y2 * y2;
    const double c0 = fma(b1, y2, b0);
    if constexpr (N == 5) {
      return fma(C[K][0], y4, c0);
    } else {
      const double b2 = fma(C[F + 5][0], y, C[F + 4][0]);
      const double b3 = fma(C[F + 7][0], y, C[F + 6][0]);
      return fma(fma(b3, y2, b2), y4, c0);
    }
  }
}

template <int K>
BGT_HD bool odd_series_light(double x, const double (*C)[2], double* out) {
  double y = x * x;
  double p = poly_estrin<1, K>(y, C);
  double c = (x * y) * p;
  dd s = fast_two_sum(x, c);
  double err = fabs(c) * 0x1p-50 + fabs(x) * 0x1p-69;
  return round_test(s, err, out);
}

template <int K>
BGT_HD bool even_series_light(double x, const double (*C)[2], double* out) {
  dd y = two_prod(x, x);
  double q = poly_estrin<2, K>(y.hi, C);
  double t = (y.hi * y.hi) * q;
  dd s = fast_two_sum(1.0, y.hi * C[1][0]);
  s.lo = s.lo + (y.lo * C[1][0] + t);
  double err = fabs(t) * 0x1p-49 + 0x1p-100;
  return round_test(s, err, out);
}

// ---- double-double Taylor kernels on a reduced double-double argument ----

// sin(r), |r| <= pi/4 + tiny
BGT_HD dd dd_sin_kernel(dd r) {
  dd r2 = dd_mul(r, r);
  // Horner over k = 16 .. 1 in double-double, then * r
  dd acc = dd_c(SIN_C[16]);
  for (int k = 15; k >= 1; k--) acc = dd_add(dd_mul(acc, r2), dd_c(SIN_C[k]));
  acc = dd_mul(acc, r2);  // sum_{k>=1} c_k r^(2k)
  return dd_add(r, dd_mul(acc, r));
}
// cos(r), |r| <= pi/4 + tiny
BGT_HD dd dd_cos_kernel(dd r) {
  dd r2 = dd_mul(r, r);
  dd acc = dd_c(COS_C[16]);
  for (int k = 15; k >= 1; k--) acc = dd_add(dd_mul(acc, r2), dd_c(COS_C[k]));
  acc = dd_mul(acc, r2);
  return dd_add_d(acc, 1.0);
}

// Cody-Waite reduction x = k*pi/2 + r, |k| < 2^19; r as double-double.
BGT_HD dd reduce_pio2(double x, int* quadrant) {
  double k = rint(x * BGT_CR_TWO_OVER_PI);
  // x - k*p1 is exact (k*p1 exact, Sterbenz); k*p2 exact (33-bit factors)
  double t = x - k * BGT_CR_PIO2_CW1;
  dd r = two_sum(t, -(k * BGT_CR_PIO2_CW2));
  r = dd_add(r, dd_neg(two_prod(k, BGT_CR_PIO2_CW3)));
  long long ki = (long long)k;
  *quadrant = (int)(ki & 3);
  return r;
}

BGT_HD_NOINLINE void dd_sincos_any(double x, dd* s, dd* c) {
  int q = 0;
  dd r = (fabs(x) <= 0.78539816339744828) ? dd{x, 0.0} : reduce_pio2(x, &q);
  dd sr = dd_sin_kernel(r), cr = dd_cos_kernel(r);
  switch (q) {
    case 0: *s = sr; *c = cr; break;
    case 1: *s = cr; *c = dd_neg(sr); break;
    case 2: *s = dd_neg(sr); *c = dd_neg(cr); break;
    default: *s = dd_neg(cr); *c = sr; break;
  }
}

// ---- sin / cos ----

BGT_HD double sin_fast_or_nan(double x) {
  // |x| <= pi/4: x + T3 + T5 (double-double) + x^7 P(x^2) (double)
  dd x2 = two_prod(x, x);
  dd x3 = dd_mul_d(x2, x);
  dd x5 = dd_mul(x3, x2);
  dd t3 = dd_mul(x3, dd_c(SIN_C[1]));
  dd t5 = dd_mul(x5, dd_c(SIN_C[2]));
  double y = x2.hi;
  double p = SIN_C[8][0];
  for (int k = 7; k >= 3; k--) p = p * y + SIN_C[k][0];
  double tail = x5.hi * y * p;
  dd acc = dd_add_d(t5, tail);
  acc = dd_add(t3, acc);
  acc = dd_add_d(acc, x);
  // tail evaluation error (relative 2^-49), double-double terms (2^-96 |x|),
  // truncation after x^17 (< x^19/19! <= 1e-17 |x| y^9)
  double err = fabs(tail) * 0x1p-49 + fabs(x) * 0x1p-96 + fabs(x) * (y * y * y) * (y * y * y) * (y * y * y) * 1e-17;
  double out;
  if (round_test(acc, err, &out)) return out;
  return NAN;
}

BGT_HD double cos_fast_or_nan(double x) {
  dd x2 = two_prod(x, x);
  dd x4 = dd_mul(x2, x2);
  dd t2 = {x2.hi * COS_C[1][0], x2.lo * COS_C[1][0]};  // * (-1/2), exact
  dd t4 = dd_mul(x4, dd_c(COS_C[2]));
  double y = x2.hi;
  double p = COS_C[9][0];
  for (int k = 8; k >= 3; k--) p = p * y + COS_C[k][0];
  double tail = x4.hi * y * p;
  dd acc = dd_add_d(t4, tail);
  acc = dd_add(t2, acc);
  acc = dd_add_d(acc, 1.0);
  double err = fabs(tail) * 0x1p-49 + 0x1p-100 + (y * y * y) * (y * y * y) * (y * y * y) * y * 1e-18;
  double out;
  if (round_test(acc, err, &out)) return out;
  return NAN;
}

BGT_HD double sin(double x) {
  if (!(fabs(x) < 524288.0)) return ::sin(x);  // non-finite or huge: library value
  if (x == 0) return x;
  if (fabs(x) <= 0x1p-4) {
    if (fabs(x) < 0x1p-27) return x;
    double f;
    if (odd_series_light<5>(x, SIN_C, &f)) return f;
  }
  if (fabs(x) <= 0.78539816339744828) {
    double f = sin_fast_or_nan(x);
    if (f == f) return f;
  }
  dd s, c;
  dd_sincos_any(x, &s, &c);
  return s.hi + s.lo;
}

BGT_HD double cos(double x) {
  if (!(fabs(x) < 524288.0)) return ::cos(x);
  if (fabs(x) <= 0x1p-4) {
    if (fabs(x) < 0x1p-27) return 1.0;
    double f;
    if (even_series_light<5>(x, COS_C, &f)) return f;
  }
  if (fabs(x) <= 0.78539816339744828) {
    double f = cos_fast_or_nan(x);
    if (f == f) return f;
  }
  dd s, c;
  dd_sincos_any(x, &s, &c);
  return c.hi + c.lo;
}

BGT_HD void sincos(double x, double* s, double* c) {
  *s = cr::sin(x);
  *c = cr::cos(x);
}

// ---- tan (|x| < 2^19; larger or non-finite arguments use the library) ----
// Below 2^-27, x^3/3 is below half an ulp of x, so the correctly rounded
// value is x.  Elsewhere sin / cos of the double-double reduced argument,
// divided in double-double: the relative error stays far below the 2^-53
// rounding step except within a few 1e-20 of the poles, which no tracking
// argument reaches.  Used by the exact (PTC) bend edge only.
BGT_HD_NOINLINE double tan(double x) {
  if (!(fabs(x) < 524288.0)) return ::tan(x);
  if (fabs(x) < 0x1p-27) return x;
  dd s, c;
  dd_sincos_any(x, &s, &c);
  dd t = dd_div(s, c);
  return t.hi + t.lo;
}

// ---- sinh / cosh (|x| <= 2; larger arguments use the library) ----

BGT_HD_NOINLINE dd dd_sinh_kernel(double x) {
  dd x2 = two_prod(x, x);
  dd acc = dd_c(SINH_C[16]);
  for (int k = 15; k >= 1; k--) acc = dd_add(dd_mul(acc, x2), dd_c(SINH_C[k]));
  acc = dd_mul(acc, x2);
  return dd_add_d(dd_mul_d(acc, x), x);
}
BGT_HD_NOINLINE dd dd_cosh_kernel(double x) {
  dd x2 = two_prod(x, x);
  dd acc = dd_c(COSH_C[16]);
  for (int k = 15; k >= 1; k--) acc = dd_add(dd_mul(acc, x2), dd_c(COSH_C[k]));
  acc = dd_mul(acc, x2);
  return dd_add_d(acc, 1.0);
}

BGT_HD double sinh(double x) {
  double a = fabs(x);
  if (!(a <= 2.0)) return ::sinh(x);
  if (x == 0) return x;
  if (a <= 0x1p-4) {
    if (a < 0x1p-27) return x;
    double f;
    if (odd_series_light<5>(x, SINH_C, &f)) return f;
  }
  if (a <= 0.78539816339744828) {
    dd x2 = two_prod(x, x);
    dd x3 = dd_mul_d(x2, x);
    dd x5 = dd_mul(x3, x2);
    dd t3 = dd_mul(x3, dd_c(SINH_C[1]));
    dd t5 = dd_mul(x5, dd_c(SINH_C[2]));
    double y = x2.hi;
    double p = SINH_C[8][0];
    for (int k = 7; k >= 3; k--) p = p * y + SINH_C[k][0];
    double tail = x5.hi * y * p;
    dd acc = dd_add_d(t5, tail);
    acc = dd_add(t3, acc);
    acc = dd_add_d(acc, x);
    double err = fabs(tail) * 0x1p-49 + a * 0x1p-96 + a * (y * y * y) * (y * y * y) * (y * y * y) * 1e-17;
    double out;
    if (round_test(acc, err, &out)) return out;
  }
  dd r = dd_sinh_kernel(x);
  return r.hi + r.lo;
}

BGT_HD double cosh(double x) {
  double a = fabs(x);
  if (!(a <= 2.0)) return ::cosh(x);
  if (a <= 0x1p-4) {
    if (a < 0x1p-27) return 1.0;
    double f;
    if (even_series_light<5>(x, COSH_C, &f)) return f;
  }
  if (a <= 0.78539816339744828) {
    dd x2 = two_prod(x, x);
    dd x4 = dd_mul(x2, x2);
    dd t2 = {x2.hi * COSH_C[1][0], x2.lo * COSH_C[1][0]};  // * (1/2), exact
    dd t4 = dd_mul(x4, dd_c(COSH_C[2]));
    double y = x2.hi;
    double p = COSH_C[9][0];
    for (int k = 8; k >= 3; k--) p = p * y + COSH_C[k][0];
    double tail = x4.hi * y * p;
    dd acc = dd_add_d(t4, tail);
    acc = dd_add(t2, acc);
    acc = dd_add_d(acc, 1.0);
    double err = fabs(tail) * 0x1p-49 + 0x1p-100 + (y * y * y) * (y * y * y) * (y * y * y) * y * 1e-18;
    double out;
    if (round_test(acc, err, &out)) return out;
  }
  dd r = dd_cosh_kernel(x);
  return r.hi + r.lo;
}

// ---- exp (|x| <= 2; larger arguments use the library) ----
//
// Light path, 2^-54 <= |x| <= 2^-4: e^x = (1 + x) + x^2 P(x) with
// P(x) = 1/2 + x/6 + ... + x^13/15! in plain double (Horner); 1 + x is exact
// as a double-double (two_sum), |x^2 P| <= 0.52 x^2 <= 2^-8.9.  Relative
// error of c = x^2 P: the square (u), P (< 1.2u: its leading 1/2 is exact
// and the next term is below x/6), the product (u) -> < 4u < 2^-50; the
// omitted terms are < x^16/16! < 2^-108; the add into 1 + x < 2^-105.
// Below 2^-54 the correctly rounded value is 1.  Accurate path: the Taylor
// series to x^40/40! in double-double (Horner), error < 2^-99 relative.

BGT_HD_NOINLINE dd dd_exp_kernel(double x) {
  dd acc = dd_c(EXP_C[40]);
  for (int k = 39; k >= 0; k--) acc = dd_add(dd_mul_d(acc, x), dd_c(EXP_C[k]));
  return acc;
}

BGT_HD double exp(double x) {
  double a = fabs(x);
  if (!(a <= 2.0)) return ::exp(x);
  if (a < 0x1p-54) return 1.0;
  if (a <= 0x1p-4) {
    double p = EXP_C[15][0];
    for (int k = 14; k >= 2; k--) p = p * x + EXP_C[k][0];
    double c = (x * x) * p;
    dd acc = dd_add_d(two_sum(1.0, x), c);
    double out;
    if (round_test(acc, fabs(c) * 0x1p-50 + 0x1p-104, &out)) return out;
  }
  dd r = dd_exp_kernel(x);
  return r.hi + r.lo;
}

// ---- asin ----

// asin(r) for a double-double r with |r| <= 1/2, full double-double series.
BGT_HD_NOINLINE dd dd_asin_kernel(dd r) {
  dd r2 = dd_mul(r, r);
  dd acc = dd_c(ASIN_C[39]);
  for (int k = 38; k >= 1; k--) acc = dd_add(dd_mul(acc, r2), dd_c(ASIN_C[k]));
  acc = dd_mul(acc, r2);
  return dd_add(r, dd_mul(acc, r));
}

// |u| <= 1/8: u + T3 + T5 (double-double) + u^7 P(u^2) (double), or NaN
// when the rounding test fails
BGT_HD double asin_mid_or_nan(double u) {
  const double a = fabs(u);
  dd u2 = two_prod(u, u);
  dd u3 = dd_mul_d(u2, u);
  dd u5 = dd_mul(u3, u2);
  dd t3 = dd_mul(u3, dd_c(ASIN_C[1]));
  dd t5 = dd_mul(u5, dd_c(ASIN_C[2]));
  double y = u2.hi;
  double p = ASIN_C[12][0];
  for (int k = 11; k >= 3; k--) p = p * y + ASIN_C[k][0];
  double tail = u5.hi * y * p;
  dd acc = dd_add_d(t5, tail);
  acc = dd_add(t3, acc);
  acc = dd_add_d(acc, u);
  // truncation after u^25: < 0.02 u y^12 / (1 - y)
  double y4 = y * y * y * y;
  double err = fabs(tail) * 0x1p-49 + a * 0x1p-96 + a * y4 * y4 * y4 * 0.03;
  double out;
  if (round_test(acc, err, &out)) return out;
  return NAN;
}

BGT_HD double asin(double u) {
  double a = fabs(u);
  if (!(a <= 1.0)) return ::asin(u);  // |u| > 1 or NaN
  if (u == 0) return u;
  if (a <= 0x1p-4) {
    if (a < 0x1p-27) return u;
    double f;
    if (odd_series_light<8>(u, ASIN_C, &f)) return f;
  }
  if (a <= 0.125) {
    double f = asin_mid_or_nan(u);
    if (f == f) return f;
  }
  dd r;
  if (a <= 0.5) {
    r = dd_asin_kernel({a, 0.0});
  } else {
    // asin(a) = pi/2 - 2 asin(sqrt((1 - a) / 2)), (1 - a)/2 exact for a >= 1/2
    double z = (1.0 - a) * 0.5;
    dd s = dd_sqrt({z, 0.0});
    dd as = dd_asin_kernel(s);
    r = dd_add(dd{BGT_CR_PIO2_HI, BGT_CR_PIO2_LO}, dd_neg(dd_mul_d(as, 2.0)));
  }
  double v = r.hi + r.lo;
  return u < 0 ? -v : v;
}

// ---- atan2 ----

// atan(q) for a double-double q with |q| <= 1, via two argument halvings
// atan(q) = 2 atan(q / (1 + sqrt(1 + q^2))) and the series.
BGT_HD_NOINLINE dd dd_atan_kernel(dd q) {
  int halvings = 0;
  while (fabs(q.hi) > 0.1 && halvings < 4) {
    dd den = dd_add_d(dd_sqrt(dd_add_d(dd_mul(q, q), 1.0)), 1.0);
    q = dd_div(q, den);
    halvings++;
  }
  dd q2 = dd_mul(q, q);
  dd acc = dd_c(ATAN_C[39]);
  for (int k = 38; k >= 1; k--) acc = dd_add(dd_mul(acc, q2), dd_c(ATAN_C[k]));
  acc = dd_mul(acc, q2);
  dd r = dd_add(q, dd_mul(acc, q));
  for (int h = 0; h < halvings; h++) r = dd_mul_d(r, 2.0);
  return r;
}

// atan(qh + ql), |qh| <= 1/8, ql the low word of the quotient: qh + T3 + T5
// (double-double) + qh^7 P(qh^2) (double) + ql / (1 + qh^2), or NaN when
// the rounding test fails
BGT_HD double atan_mid_or_nan(double qh, double ql) {
  dd q2 = two_prod(qh, qh);
  dd q3 = dd_mul_d(q2, qh);
  dd q5 = dd_mul(q3, q2);
  dd t3 = dd_mul(q3, dd_c(ATAN_C[1]));
  dd t5 = dd_mul(q5, dd_c(ATAN_C[2]));
  double yy = q2.hi;
  double p = ATAN_C[11][0];
  for (int k = 10; k >= 3; k--) p = p * yy + ATAN_C[k][0];
  double tail = q5.hi * yy * p;
  double corr = ql / (1.0 + yy);  // d atan = dq / (1 + q^2)
  dd acc = dd_add_d(t5, tail);
  acc = dd_add(t3, acc);
  acc = dd_add_d(acc, corr);
  acc = dd_add_d(acc, qh);
  double y4 = yy * yy * yy * yy;
  double err = fabs(tail) * 0x1p-49 + fabs(corr) * 0x1p-49 + fabs(qh) * 0x1p-96 +
               fabs(qh) * y4 * y4 * y4 * 0.05;
  double out;
  if (round_test(acc, err, &out)) return out;
  return NAN;
}

BGT_HD double atan2(double y, double x) {
  if (!(fabs(x) < 1e300 && fabs(y) < 1e300) || x == 0 || y == 0) return ::atan2(y, x);
  double ax = fabs(x), ay = fabs(y);
  if (ay > ax * 0x1p60 || ay < ax * 0x1p-60) return ::atan2(y, x);
  if (ax < 0x1p-900) {  // same quotient, reciprocal and remainders kept normal
    x *= 0x1p900;
    y *= 0x1p900;
  }
  // q = y / x as double-double from one reciprocal rx = RN(1 / x): a Newton
  // step from y rx lands qh within one ulp of y / x (a faithful quotient),
  // so the remainder y - x qh is exact, and ql = (y - x qh) rx carries a
  // relative error below 2u + u^2.
  const double rx = 1.0 / x;
  const double q0 = y * rx;
  const double qh = fma(fma(-q0, x, y), rx, q0);
  const double ql = fma(-qh, x, y) * rx;
  if (x > 0 && fabs(qh) <= 0x1p-4) {
    // atan(qh + ql) = atan(qh) + ql - ql qh^2 / (1 + qh^2) + O(ql^2): the
    // odd-series bound for atan(qh) (K = 8) plus the rounding of c + ql,
    // the error of ql (< 2u + u^2 < 2^-51) and the dropped ql qh^2 term
    // (< 2 |ql| yy).
    double yy = qh * qh;
    double p = poly_estrin<1, 8>(yy, ATAN_C);
    double c = (qh * yy) * p;
    double t = c + ql;
    dd s = fast_two_sum(qh, t);
    double err = fabs(c) * 0x1p-50 + fabs(t) * 0x1p-52 + fabs(ql) * (2 * yy + 0x1p-51) + fabs(qh) * 0x1p-69;
    double out;
    if (round_test(s, err, &out)) return out;
  }
  if (x > 0 && fabs(qh) <= 0.125) {
    double f = atan_mid_or_nan(qh, ql);
    if (f == f) return f;
  }
  dd q = {qh, ql};
  dd a;
  if (fabs(qh) <= 1.0) {
    a = dd_atan_kernel(q);
  } else {
    dd inv = dd_div({1.0, 0.0}, q);
    dd b = dd_atan_kernel(inv);
    dd hp = dd{BGT_CR_PIO2_HI, BGT_CR_PIO2_LO};
    a = qh > 0 ? dd_add(hp, dd_neg(b)) : dd_add(dd_neg(hp), dd_neg(b));
  }
  if (x < 0) a = (y >= 0) ? dd_add(a, dd{BGT_CR_PI_HI, BGT_CR_PI_LO}) : dd_add(a, dd_neg(dd{BGT_CR_PI_HI, BGT_CR_PI_LO}));
  return a.hi + a.lo;
}

// atan(x) = atan2(x, 1): the quotient x / 1 is exact, so the correctly
// rounded atan2 is the correctly rounded atan.
BGT_HD double atan(double x) { return cr::atan2(x, 1.0); }

}  // namespace cr
}  // namespace bgt
