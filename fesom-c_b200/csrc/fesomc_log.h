/*
 * fesomc_log.h -- natural logarithm built from correctly rounded IEEE
 * operations only (+, -, *, /, fma), so that the host and the device give
 * the same bits for the same argument.  It serves the one transcendental of
 * the FP64 time step, the bottom boundary value of the turbulence closure
 * log(delta_b / z0b_min) (src/fv_mixing.F90:238), in the device kernels and
 * in the CPU oracle alike; plain C, includable from C and CUDA C++.
 *
 * Method: argument reduction by the binary exponent and the atanh series.
 *   x = 2^k m, m in [sqrt(1/2), sqrt(2));  f = m - 1 (exact, Sterbenz);
 *   s = f / (2 + f), carried as a double-double sh + sl, |s| < 0.1716;
 *   log x = k ln2 + 2 atanh(s)
 *         = k ln2 + 2 s + 2 s^3 (1/3 + s^2/5 + s^4/7 + ... + s^20/23).
 * ln2 is split Cody-Waite style into a 40-bit head (k * LN2_HI is exact for
 * |k| < 2^13) and a tail.  The first omitted series term is below 2^-60 of
 * the result, the series tail is at most 1 % of the result, and the head
 * k ln2_hi + 2 sh is summed exactly, so the result is within one ulp of
 * log x; against glibc's log over 2e7 random arguments it differs in 0.16 %
 * of them, by one ulp, and is the closer of the two in about 40 % of those
 * (tests/test_oracle.py holds the one-ulp bound).
 *
 * The FP64 kernels are compiled without FMA contraction and the oracle with
 * -ffp-contract=off; the one fused operation here is the explicit fma().
 */
#ifndef FESOMC_LOG_H
#define FESOMC_LOG_H

#include <math.h>

#ifdef __CUDACC__
#define FESOMC_LOG_FN static __host__ __device__ inline
#else
#define FESOMC_LOG_FN static inline
#endif

/* ln 2 = 0.693147180559945309417232121458176568...: 40-bit head and tail */
#define FESOMC_LN2_HI 0x1.62e42fefa2p-1
#define FESOMC_LN2_LO 0x1.9ef35793c7673p-41

FESOMC_LOG_FN double fesomc_log(double x) {
    if (x == 0.0) return -HUGE_VAL;
    if (!(x > 0.0)) return (x - x) / (x - x);     /* negative or NaN: NaN */
    if (x == HUGE_VAL) return x;
    int k;
    double m = frexp(x, &k);                       /* x = m 2^k, m in [1/2, 1) */
    if (m < 0.70710678118654752440) {
        m = m + m;
        k = k - 1;
    }
    const double f = m - 1.0;
    const double dh = 2.0 + f;
    const double dl = f - (dh - 2.0);              /* 2 + f == dh + dl exactly */
    const double sh = f / dh;
    /* f - sh*dh is exact for the correctly rounded quotient sh */
    const double sl = (fma(-sh, dh, f) - sh * dl) / dh;
    const double z = sh * sh;
    const double p =
        (2.0 / 3.0) + z * ((2.0 / 5.0) + z * ((2.0 / 7.0) + z * ((2.0 / 9.0) + z * ((2.0 / 11.0) +
        z * ((2.0 / 13.0) + z * ((2.0 / 15.0) + z * ((2.0 / 17.0) + z * ((2.0 / 19.0) +
        z * ((2.0 / 21.0) + z * (2.0 / 23.0))))))))));
    const double t = (sh * z) * p;
    const double a = (double)k * FESOMC_LN2_HI;    /* exact */
    const double b = sh + sh;                      /* exact */
    const double s = a + b;
    const double bv = s - a;
    const double e = (a - (s - bv)) + (b - bv);    /* a + b == s + e exactly */
    return s + (e + (((double)k * FESOMC_LN2_LO + (sl + sl)) + t));
}

#endif /* FESOMC_LOG_H */
