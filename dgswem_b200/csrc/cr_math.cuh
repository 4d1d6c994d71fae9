// cr_math.cuh -- the correctly rounded value of DEPTH**(1.D0/3.D0), the
// Manning depth factor of rhs_dg_hydro.F, computed with IEEE-754 basic
// operations (+, -, *, /, fma, and the exact frexp / ldexp) and a
// single-precision logarithm whose error the method absorbs, so that the
// same source gives the same bits on the host and on the device.
//
// The exponent of the reference's expression is c = RN(1/3) = (1 - 2^-54)/3,
// the double nearest 1/3, so
//     x^c = x^(1/3) * x^(-2^-54/3) = cbrt(x) * (1 - 2^-54 ln(x) / 3 + O(2^-108 ln(x)^2)).
// cbrt(x) is formed to about 2^-100 relative accuracy as a double plus a
// correction term:
//   1. x = f 2^e (frexp), e = 3q + r with r in {0, 1, 2}, m = f 2^r in [0.5, 4);
//   2. y ~ m^(-1/3) by Newton's iteration for the inverse cube root,
//      y <- y + y (1 - m y^3) / 3, from a quadratic start (no division);
//   3. z = m y^2 ~ m^(1/3); the residual z^3 - m is evaluated with the
//      error-free products of fma (z^2 = p_h + p_l exactly, p_h z = t_h + t_l
//      exactly, t_h - m exact by Sterbenz's lemma), and one Newton step in
//      double-double gives cbrt(m) = z - res y^2 / 3 (y^2 = 1 / z^2 to working
//      precision);
//   4. ln(x), which enters the result scaled by 2^-54 / 3: first from a
//      single-precision logarithm, which decides the rounding unless the
//      value lies within 2^-70 of a midpoint between doubles (checked from
//      the exact rounding error of the final sum); then, in those rare
//      cases, as e' ln 2 + 2 atanh(s), s = (f' - 1) / (f' + 1), f' in
//      [1/sqrt 2, sqrt 2), by its odd series (absolute error below 1e-15);
//   5. the double-double value times (1 - 2^-54 ln(x)/3) is rounded once to
//      double and scaled by 2^q (exact).
// The result differs from the correctly rounded x^c only when x^c lies within
// about 2^-100 relative of a midpoint between two doubles.
//
// The single-precision logarithm only chooses between the two evaluations
// of step 4 (the device's and the host's may differ; the result does not),
// so the strict kernels and the oracle (which evaluates the same expression
// as a correctly rounded pow) agree bit for bit.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define DGSWEM_HD __host__ __device__ __forceinline__
#else
#define DGSWEM_HD inline
#endif

namespace dgswem {

// ln(x) = e' ln 2 + 2 atanh(s) for x = f 2^e, to 1e-15 absolute (step 4)
DGSWEM_HD double ln_series(double f, int e) {
  double fp = f;
  int ep = e;
  if (fp < 0.70710678118654752440) {
    fp = fp + fp;
    ep = ep - 1;
  }
  const double s = (fp - 1.0) / (fp + 1.0);
  const double s2 = s * s;
  double poly = 1.0 / 19.0;
  poly = 1.0 / 17.0 + s2 * poly;
  poly = 1.0 / 15.0 + s2 * poly;
  poly = 1.0 / 13.0 + s2 * poly;
  poly = 1.0 / 11.0 + s2 * poly;
  poly = 1.0 / 9.0 + s2 * poly;
  poly = 1.0 / 7.0 + s2 * poly;
  poly = 1.0 / 5.0 + s2 * poly;
  poly = 1.0 / 3.0 + s2 * poly;
  const double lnf = 2.0 * s + 2.0 * s * (s2 * poly);
  // ln 2 = hi + lo, hi with 21 trailing zero bits so that ep * hi is exact
  const double ln2_hi = 0x1.62e42feep-1;
  const double ln2_lo = 1.9082149292705877e-10;
  return (double)ep * ln2_hi + ((double)ep * ln2_lo + lnf);
}

// kFastLog = false takes the series for ln(x) every time (the rare path
// alone, for tests).
template <bool kFastLog = true>
DGSWEM_HD double pow_third(double x) {
  if (!(x > 0.0) || !(x < INFINITY)) {
    // pow(x, c) of a zero, negative, infinite or NaN base: 0, NaN, inf, NaN
    if (x == 0.0) return 0.0;
    if (x > 0.0) return x;
    return NAN;
  }
  int e;
  const double f = frexp(x, &e);  // x = f 2^e, f in [0.5, 1)
  // e = 3q + r, r in {0, 1, 2} (floor division for negative e)
  int q = e >= 0 ? e / 3 : -((-e + 2) / 3);
  const int r = e - 3 * q;
  const double m = ldexp(f, r);  // [0.5, 4)
  // step 2: inverse cube root, quadratic start (least-squares fit of the
  // relative error over [0.5, 4), below 9 %; five steps reach rounding level)
  double y = 1.31600226 + m * (-0.3495224 + m * 0.04591333);
  const double third = 1.0 / 3.0;
  for (int it = 0; it < 5; ++it) {
    const double y3 = y * y * y;
    y = y + y * ((1.0 - m * y3) * third);
  }
  // step 3: z ~ m^(1/3) and its double-double Newton correction
  const double y2 = y * y;
  const double z = m * y2;
  const double p_h = z * z;
  const double p_l = fma(z, z, -p_h);
  const double t_h = p_h * z;
  const double t_l = fma(p_h, z, -t_h);
  const double res = (t_h - m) + (t_l + p_l * z);
  const double corr = (res * y2) * third;  // cbrt(m) = z - corr
  // steps 4-5, first with ln(x) from a single-precision logarithm (absolute
  // error below 2^-20 for f in [0.5, 1)): delta is then known to 2^-75, and
  // z + tail rounds to the same double as the exact value unless the exact
  // value lies within 2^-70 (relative) of a midpoint between two doubles.
  // s = RN(z + tail) and its rounding error err (exact, |tail| << z) show
  // that distance: |err| far from half an ulp of s keeps s.  Otherwise --
  // about once in 2^18 calls -- ln(x) to 1e-15 by its series.
  const double k54 = 5.5511151231257827e-17 * third;  // 2^-54 / 3
  if (kFastLog) {
#if defined(__CUDA_ARCH__)
    const float lnf_fast = __logf((float)f);
#else
    const float lnf_fast = std::log((float)f);
#endif
    const double lnx_fast = (double)e * 0.69314718055994531 + (double)lnf_fast;
    const double delta_fast = lnx_fast * k54;
    const double tail_fast = (-corr - z * delta_fast) + corr * delta_fast;
    const double s = z + tail_fast;
    const double err = tail_fast - (s - z);
    int es;
    const double fs = frexp(s, &es);                // s = fs 2^es, fs in [0.5, 1)
    const double half_ulp = ldexp(1.0, es - 54);    // half an ulp of s
    if (fs != 0.5 && fabs(fabs(err) - half_ulp) > s * 0x1p-70) return ldexp(s, q);
  }
  // step 4-5 with ln(x) to 1e-15 (also when s is a power of two, whose ulp
  // below is half the one above)
  const double delta = ln_series(f, e) * k54;
  const double tail = (-corr - z * delta) + corr * delta;
  return ldexp(z + tail, q);
}

// x / 3, correctly rounded, without a division: q = RN(x t), t = RN(1/3);
// r = x - 3q is exact (q is within 1 ulp of x/3, so r is a multiple of
// ulp(q) no larger than 3 ulp(q)) and fma(r, t, q) = RN(q + r t) is within
// 2^-53 ulp of x/3.  The exact quotient x/3 = M 2^e / 3 lies at least 1/6
// ulp from every midpoint between doubles (its remainder in ulps is a
// multiple of 1/3), so that rounding is the correctly rounded x/3 -- the IEEE
// division's result -- for every finite x.  The sign is x's (a zero quotient
// keeps the sign of x, as the division's does, which the sequence alone
// would lose: fma(+0, t, -0) = +0).  Four instructions instead of a division
// sequence.
DGSWEM_HD double div3(double x) {
  const double t = 1.0 / 3.0;
  const double q = x * t;
  const double r = fma(-q, 3.0, x);
  return copysign(fma(r, t, q), x);
}

}  // namespace dgswem
