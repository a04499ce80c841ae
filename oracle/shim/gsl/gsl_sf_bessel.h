/*
 * gsl/gsl_sf_bessel.h -- stand-in for the one GSL special function the
 * reference's Kaiser window calls (ctas src/common/lct.cpp:192-193), for
 * compiling lct.cpp without GSL.  Test infrastructure only.
 *
 * I0(x) = sum_k ((x/2)^2)^k / (k!)^2, the modified Bessel function of the
 * first kind of order 0, summed in double until the terms stop changing the
 * sum; GSL's own implementation (Chebyshev expansions) agrees with it to a few
 * ulps of double, far below the float the reference stores.
 */
#ifndef CTAS_ORACLE_SHIM_GSL_SF_BESSEL_H
#define CTAS_ORACLE_SHIM_GSL_SF_BESSEL_H

static inline double gsl_sf_bessel_I0(double x) {
  const double q = 0.25 * x * x;
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 500; k++) {
    term *= q / ((double)k * (double)k);
    const double next = sum + term;
    if (next == sum) break;
    sum = next;
  }
  return sum;
}

#endif
