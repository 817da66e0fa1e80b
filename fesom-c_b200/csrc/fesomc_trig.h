/*
 * fesomc_trig.h -- cosine built from correctly rounded IEEE operations only
 * (+, -, *, / and rint), so that the host and the device give the same bits
 * for the same argument.  It serves the harmonic open-boundary elevation of
 * compute_ssh_rhs_elem (src/fv_average_dynamic.F90:190-216), evaluated on
 * the device by the forcing kernel and on the host by the CPU oracle and the
 * host forcing path alike, and the equilibrium tide of potential
 * (src/fv_tide_potential.F90:1-107); plain C, includable from C and CUDA C++.
 *
 * Method: Cody-Waite reduction by pi/2 and the Taylor series.
 *   n = rint(x * 2/pi),  r = ((x - n P1) - n P2) - n P3,  |r| <= pi/4 + tiny,
 * with P1 + P2 + P3 = pi/2, P1 and P2 of 33 significant bits (n P1 and n P2
 * are exact for |n| < 2^20, i.e. |x| < 1.6e6) and P3 the rounded remainder;
 * r is carried as a head and a tail (the tail enters to first order).
 *   sin r = r + r z (-1/3! + z/5! - ... + z^7/17!),       z = r^2
 *   cos r = 1 - z/2 + z^2 (1/4! - z/6! + ... - z^7/18!)
 * (the first omitted terms are below 1e-19), the quadrant n mod 4 picks
 * +-sin / +-cos (for sin x the quadrant shifted by one).  The 1 - z/2 step keeps its rounding error (the difference
 * (1 - v) - z/2 is exact) and adds it back.  Within one ulp of cos x over
 * the range; against glibc's cos over 2e7 random arguments in [-1000, 1000]
 * it differs in 3 % of them, by one ulp (tests/test_oracle.py holds the
 * one-ulp bound).
 * Arguments beyond 1.6e6 in magnitude return NaN; the open-boundary phases
 * stay far below that (a year of M2 is about 4400 radians).
 *
 * The FP64 kernels are compiled without FMA contraction and the oracle with
 * -ffp-contract=off, so both evaluate the same sequence of roundings.
 */
#ifndef FESOMC_TRIG_H
#define FESOMC_TRIG_H

#include <math.h>

#ifdef __CUDACC__
#define FESOMC_TRIG_FN static __host__ __device__ inline
#else
#define FESOMC_TRIG_FN static inline
#endif

/* pi/2 = 1.5707963267948966192313216916397514...: two 33-bit heads and a tail */
#define FESOMC_PIO2_1 0x1.921fb544p+0
#define FESOMC_PIO2_2 0x1.0b4611a6p-34
#define FESOMC_PIO2_3 0x1.3198a2e037073p-69
#define FESOMC_2_OVER_PI 0x1.45f306dc9c883p-1

/* sin(rh + rl) and cos(rh + rl) for |rh| <= pi/4, |rl| <= ulp(rh) */
FESOMC_TRIG_FN double fesomc_sin_kernel(double rh, double rl) {
    const double z = rh * rh;
    const double p = -(1.0 / 6.0) + z * ((1.0 / 120.0) + z * (-(1.0 / 5040.0) + z * ((1.0 / 362880.0) +
                     z * (-(1.0 / 39916800.0) + z * ((1.0 / 6227020800.0) + z * (-(1.0 / 1307674368000.0) +
                     z * (1.0 / 355687428096000.0)))))));
    return rh + ((rh * z) * p + rl * (1.0 - 0.5 * z));
}

FESOMC_TRIG_FN double fesomc_cos_kernel(double rh, double rl) {
    const double z = rh * rh;
    const double q = (1.0 / 24.0) + z * (-(1.0 / 720.0) + z * ((1.0 / 40320.0) + z * (-(1.0 / 3628800.0) +
                     z * ((1.0 / 479001600.0) + z * (-(1.0 / 87178291200.0) + z * ((1.0 / 20922789888000.0) +
                     z * -(1.0 / 6402373705728000.0)))))));
    const double hz = 0.5 * z;
    const double v = 1.0 - hz;
    return v + (((1.0 - v) - hz) + ((z * z) * q - rh * rl));
}

/* x = n pi/2 + (rh + rl); returns n mod 4 (|x| < 1.6e6) */
FESOMC_TRIG_FN int fesomc_reduce_pio2(double x, double *rh_out, double *rl_out) {
    const double n = rint(x * FESOMC_2_OVER_PI);
    /* reduced argument as rh + rl: a is exact, a - b is split exactly (two-sum) */
    const double a = x - n * FESOMC_PIO2_1;
    const double b = n * FESOMC_PIO2_2;
    const double t = a - b;
    const double tb = t - a;
    const double e = (a - (t - tb)) - (b + tb);
    const double c = n * FESOMC_PIO2_3;
    const double rh = t - c;
    *rh_out = rh;
    *rl_out = ((t - rh) - c) + e;
    return (int)(((long long)n) & 3);
}

FESOMC_TRIG_FN double fesomc_cos(double x) {
    if (!(fabs(x) < 1.6e6)) return (x - x) / (x - x);     /* out of range, inf or NaN: NaN */
    double rh, rl;
    switch (fesomc_reduce_pio2(x, &rh, &rl)) {
        case 0: return fesomc_cos_kernel(rh, rl);
        case 1: return -fesomc_sin_kernel(rh, rl);
        case 2: return -fesomc_cos_kernel(rh, rl);
        default: return fesomc_sin_kernel(rh, rl);
    }
}

FESOMC_TRIG_FN double fesomc_sin(double x) {
    if (!(fabs(x) < 1.6e6)) return (x - x) / (x - x);
    double rh, rl;
    switch (fesomc_reduce_pio2(x, &rh, &rl)) {
        case 0: return fesomc_sin_kernel(rh, rl);
        case 1: return fesomc_cos_kernel(rh, rl);
        case 2: return -fesomc_sin_kernel(rh, rl);
        default: return -fesomc_cos_kernel(rh, rl);
    }
}

#endif /* FESOMC_TRIG_H */
