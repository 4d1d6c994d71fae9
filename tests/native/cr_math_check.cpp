// Host build of dgswem::pow_third (dgswem_b200/csrc/cr_math.cuh, the strict
// kernels' Manning depth factor) beside two references: the quadruple-
// precision pow rounded to double (libquadmath; the correctly rounded
// DEPTH**(1.D0/3.D0) up to 2^-112) and the C library's double pow.  Built
// and called by tests/test_cr_math.py (test infrastructure).
#include <quadmath.h>

#include <cmath>

#include "cr_math.cuh"

extern "C" void cr_pow_third_eval(const double* xs, long n, double* ours, double* quad, double* libm) {
  for (long i = 0; i < n; ++i) {
    const double x = xs[i];
    ours[i] = dgswem::pow_third(x);
    quad[i] = (double)powq((__float128)x, (__float128)(1.0 / 3.0));
    libm[i] = std::pow(x, 1.0 / 3.0);
  }
}
