/*
 * fesomc_exp.h -- exponential built from correctly rounded IEEE operations
 * only (+, -, *, rint and exact scaling by powers of two), so that the host
 * and the device give the same bits for the same argument.  It serves the
 * shortwave absorption profiles of the surface heat source in the tracer
 * column solve with atmospheric forcing (swr_paul_sim and swr_soloviev,
 * src/fv_tracer.F90:1566-1631, called by calc_heat_flux_sw :1636-1697), in
 * the device kernels and in the CPU oracle alike; plain C, includable from C
 * and CUDA C++.
 *
 * Method: Cody-Waite reduction by ln 2 and the Taylor series.
 *   k = rint(x / ln2),  r = (x - k ln2_hi) - k ln2_lo,  |r| <= ln2/2 + tiny,
 * with ln2_hi of 40 significant bits (k ln2_hi exact for |k| < 2^13) and
 * ln2_lo the rounded remainder;
 *   e^r - 1 = r + r^2 (1/2! + r/3! + ... + r^13/15!)
 * (the first omitted term is below 2^-66 of the result), then
 * e^x = (1 + (e^r - 1)) * 2^k, the scaling exact for normal results and
 * one correctly rounded multiplication for subnormal ones.  Arguments below
 * -745.2 give +0, above 709.78 +inf.  Within one ulp of e^x; against glibc's
 * exp over random arguments it differs in a few per cent of them, by one ulp
 * (tests/test_oracle.py holds the one-ulp bound).
 *
 * The FP64 kernels are compiled without FMA contraction and the oracle with
 * -ffp-contract=off, so both evaluate the same sequence of roundings.
 */
#ifndef FESOMC_EXP_H
#define FESOMC_EXP_H

#include <math.h>

#ifdef __CUDACC__
#define FESOMC_EXP_FN static __host__ __device__ inline
#else
#define FESOMC_EXP_FN static inline
#endif

/* ln 2 = 0.693147180559945309417232121458176568...: 40-bit head and tail */
#define FESOMC_EXP_LN2_HI 0x1.62e42fefa2p-1
#define FESOMC_EXP_LN2_LO 0x1.9ef35793c7673p-41
#define FESOMC_EXP_INV_LN2 0x1.71547652b82fep+0

FESOMC_EXP_FN double fesomc_exp(double x) {
    if (x != x) return x;                          /* NaN */
    if (x > 709.782712893384) return HUGE_VAL;
    if (x < -745.2) return 0.0;
    const double k = rint(x * FESOMC_EXP_INV_LN2);
    const double r = (x - k * FESOMC_EXP_LN2_HI) - k * FESOMC_EXP_LN2_LO;
    /* (e^r - 1 - r) / r^2 by Horner, coefficients 1/n! for n = 2..15 */
    double p = 1.0 / 1307674368000.0;                                  /* 1/15! */
    p = 1.0 / 87178291200.0 + r * p;                                   /* 1/14! */
    p = 1.0 / 6227020800.0 + r * p;                                    /* 1/13! */
    p = 1.0 / 479001600.0 + r * p;                                     /* 1/12! */
    p = 1.0 / 39916800.0 + r * p;                                      /* 1/11! */
    p = 1.0 / 3628800.0 + r * p;                                       /* 1/10! */
    p = 1.0 / 362880.0 + r * p;                                        /* 1/9!  */
    p = 1.0 / 40320.0 + r * p;                                         /* 1/8!  */
    p = 1.0 / 5040.0 + r * p;                                          /* 1/7!  */
    p = 1.0 / 720.0 + r * p;                                           /* 1/6!  */
    p = 1.0 / 120.0 + r * p;                                           /* 1/5!  */
    p = 1.0 / 24.0 + r * p;                                            /* 1/4!  */
    p = 1.0 / 6.0 + r * p;                                             /* 1/3!  */
    p = 0.5 + r * p;                                                   /* 1/2!  */
    const double em1 = r + (r * r) * p;
    const double y = 1.0 + em1;
    const int ki = (int)k;
    if (ki > 1023) return (y * 2.0) * ldexp(1.0, ki - 1);
    if (ki >= -1022) return y * ldexp(1.0, ki);    /* exact power of two */
    /* subnormal range: two exact powers of two, the last product rounds once */
    return (y * ldexp(1.0, ki + 64)) * ldexp(1.0, -64);
}

#endif /* FESOMC_EXP_H */
