// Host build of the correctly rounded helpers of dgswem_b200/csrc/cr_math.cuh
// beside references: pow_third (the strict kernels' Manning depth factor)
// with the quadruple-precision pow rounded to double (libquadmath; the
// correctly rounded DEPTH**(1.D0/3.D0) up to 2^-112) and the C library's
// double pow; div3 with the IEEE division x / 3.  Built and called by
// tests/test_cr_math.py (test infrastructure).
#include <quadmath.h>

#include <cmath>
#include <cstring>

#include "cr_math.cuh"

// ours: pow_third as the kernels call it (series = 0) or with the series
// for ln(x) on every call (series = 1, the rare path alone)
extern "C" void cr_pow_third_eval(const double* xs, long n, int series, double* ours, double* quad, double* libm) {
  for (long i = 0; i < n; ++i) {
    const double x = xs[i];
    ours[i] = series ? dgswem::pow_third<false>(x) : dgswem::pow_third(x);
    quad[i] = (double)powq((__float128)x, (__float128)(1.0 / 3.0));
    libm[i] = std::pow(x, 1.0 / 3.0);
  }
}

// count of x in xs[0..n) whose div3(x) and x / 3.0 differ in any bit
// (signed zeros included)
extern "C" long cr_div3_mismatches(const double* xs, long n) {
  long bad = 0;
  for (long i = 0; i < n; ++i) {
    const double a = dgswem::div3(xs[i]), b = xs[i] / 3.0;
    if (std::memcmp(&a, &b, sizeof a) != 0) ++bad;
  }
  return bad;
}
