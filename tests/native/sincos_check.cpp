// Checks dtc::dd::sincos_cr (m-dtc-direct-tensor-computation_b200/csrc/ddmath.h) against the
// nearest double of quad-precision sin/cos (libquadmath), on the angles the rotation search
// evaluates: k degrees (k = 0..180) and the refinement windows i * div, div = (pi/180) 0.1^jj
// (f-src/mod_struct_calcmat.f90:778-1012), for windows spread over [0, 180] degrees at every
// level jj = 1..16.  Prints "n mismatches_vs_quad libm_vs_quad"; exit code 1 on any mismatch.
#include <quadmath.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <random>

#include "ddmath.h"

int main() {
  const double pi = std::acos(-1.0), pid = pi / 180.0;
  long n = 0, bad = 0, libm_bad = 0;
  auto check = [&](double x) {
    double s, c;
    dtc::dd::sincos_cr(x, &s, &c);
    const double sq = (double)sinq((__float128)x), cq = (double)cosq((__float128)x);
    ++n;
    if (s != sq || c != cq) {
      if (++bad <= 5) std::printf("x=%.17g sin %.17g vs %.17g cos %.17g vs %.17g\n", x, s, sq, c, cq);
    }
    if (std::sin(x) != sq || std::cos(x) != cq) ++libm_bad;
  };
  for (int k = 0; k <= 180; ++k) check((double)k * pid);
  std::mt19937_64 g(12345);
  double div = pid;
  for (int jj = 1; jj <= 16; ++jj) {
    div = div * 0.1;
    const double unit = std::pow(10.0, jj - 1);   // window centres in units of 10^-(jj-1) degree
    for (int w = 0; w < 1500; ++w) {
      long long a = w < 12 ? w : (long long)((double)(g() % 1810000) * 1e-4 * unit);
      for (long long t = (a - 1) * 10; t <= (a + 1) * 10; ++t) check((double)t * div);
    }
  }
  std::printf("%ld %ld %ld\n", n, bad, libm_bad);
  return bad ? 1 : 0;
}
