// ddmath.h -- sine and cosine of a double, rounded to nearest, from double-double arithmetic.
//
// The refinement of the rotation search (f-src/mod_struct_calcmat.f90:778-1012) evaluates
// sin and cos at angles k * div, div = (pi/180) * 0.1^jj, and its argmin at deep levels is
// decided by the last bits of those values.  The reference takes them from the platform's
// libm (gfortran: glibc), whose results are the correctly rounded ones for practically all
// arguments.  This header computes the correctly rounded value itself so that host and device
// builds agree bit for bit with each other and with such a libm:
//   * argument reduction by Cody and Waite: r = x - k pi/2 with pi/2 held as three doubles
//     (about 160 bits) and the subtraction carried out in double-double;
//   * sin r and cos r for |r| <= pi/4 from their Taylor series, nested (Horner) form, in
//     double-double arithmetic (Dekker's and Knuth's error-free sum and product, the product
//     through one fused multiply-add), truncated where the next term is below 2^-110;
//   * the double-double result rounded once to double.
// The result is the double nearest to the exact value unless that value lies within about
// 2^-100 (relative) of a midpoint between two doubles.  Meant for |x| up to a few hundred;
// the rotation search uses |x| < 4.
//
// Every operation is written out: compile with floating-point contraction off (nvcc
// --fmad=false, g++ -ffp-contract=off) so the error-free transformations stay exact.
#pragma once

#if defined(__CUDACC__)
#define DTC_HD __host__ __device__ __forceinline__
#else
#include <cmath>
#define DTC_HD inline
#endif

namespace dtc {
namespace dd {

struct DD {
  double hi, lo;
};

DTC_HD DD two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  const double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}

DTC_HD DD quick_two_sum(double a, double b) {  // |a| >= |b|
  const double s = a + b;
  return {s, b - (s - a)};
}

DTC_HD DD two_prod(double a, double b) {
  const double p = a * b;
  return {p, fma(a, b, -p)};
}

DTC_HD DD add(DD a, DD b) {
  DD s = two_sum(a.hi, b.hi);
  const DD t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}

DTC_HD DD neg(DD a) { return {-a.hi, -a.lo}; }

DTC_HD DD mul(DD a, DD b) {
  DD p = two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return quick_two_sum(p.hi, p.lo);
}

DTC_HD DD mul_d(DD a, double b) {
  DD p = two_prod(a.hi, b);
  p.lo += a.lo * b;
  return quick_two_sum(p.hi, p.lo);
}

// a / b for a double b (two correction steps of the long division)
DTC_HD DD div_d(DD a, double b) {
  const double q1 = a.hi / b;
  DD p = two_prod(q1, b);
  DD r = two_sum(a.hi, -p.hi);
  r.lo = r.lo + a.lo - p.lo;
  const double q2 = (r.hi + r.lo) / b;
  p = two_prod(q2, b);
  DD r2 = two_sum(r.hi, -p.hi);
  r2.lo = r2.lo + r.lo - p.lo;
  const double q3 = (r2.hi + r2.lo) / b;
  DD q = quick_two_sum(q1, q2);
  return add(q, DD{q3, 0.0});
}

// pi/2 = kPio2a + kPio2b + kPio2c (each the nearest double to what remains)
constexpr double kPio2a = 1.5707963267948966;
constexpr double kPio2b = 6.123233995736766e-17;
constexpr double kPio2c = -1.4973849048591698e-33;

// sin r and cos r for a double-double |r| <= pi/4 + eps
DTC_HD void sincos_reduced(DD r, DD& s, DD& c) {
  const DD r2 = mul(r, r);
  // sin r = r (1 - r^2/(2*3) (1 - r^2/(4*5) (1 - ... (1 - r^2/(28*29)))))
  DD ps{1.0, 0.0}, pc{1.0, 0.0};
  for (int n = 14; n >= 1; --n) {
    ps = add(DD{1.0, 0.0}, neg(div_d(mul(ps, r2), (double)((2 * n) * (2 * n + 1)))));
    // cos r = 1 - r^2/(1*2) (1 - r^2/(3*4) (1 - ... (1 - r^2/(27*28))))
    pc = add(DD{1.0, 0.0}, neg(div_d(mul(pc, r2), (double)((2 * n - 1) * (2 * n)))));
  }
  s = mul(r, ps);
  c = pc;
}

// Correctly rounded sin(x) and cos(x) (see the header comment for the one exception).
DTC_HD void sincos_cr(double x, double* sn, double* cs) {
  const double kq = x * 0.63661977236758138;  // 2/pi, only to pick the quadrant
  const double k = (kq >= 0.0) ? (double)(long long)(kq + 0.5) : -(double)(long long)(-kq + 0.5);
  // r = x - k*pi/2 in double-double; k*kPio2a is exact to two doubles through two_prod
  DD r = two_sum(x, 0.0);
  r = add(r, neg(two_prod(k, kPio2a)));
  r = add(r, neg(two_prod(k, kPio2b)));
  r = add(r, neg(two_prod(k, kPio2c)));
  DD s, c;
  sincos_reduced(r, s, c);
  const long long q = ((long long)k) & 3;
  DD so, co;
  if (q == 0) { so = s; co = c; }
  else if (q == 1) { so = c; co = neg(s); }
  else if (q == 2) { so = neg(s); co = neg(c); }
  else { so = neg(c); co = s; }
  *sn = so.hi + so.lo;
  *cs = co.hi + co.lo;
}

}  // namespace dd
}  // namespace dtc

#undef DTC_HD
