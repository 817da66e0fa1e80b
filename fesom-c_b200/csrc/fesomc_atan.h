/*
 * fesomc_atan.h -- arctangent built from correctly rounded IEEE operations
 * only (+, -, *, / and sqrt), so that the host and the device give the same
 * bits for the same argument.  It serves the stability function psi_m of the
 * bulk transfer coefficients (core_coeff_2z, src/fv_sbc.F90:643-662,
 * Large & Yeager 2004, eq. 8c), evaluated on the device by the surface-flux
 * kernel and on the host by the CPU oracle; plain C, includable from C and
 * CUDA C++.
 *
 * Method (the identities of the arctangent and its Taylor series):
 *   atan(-x) = -atan(x);
 *   x > 1:              atan(x) = pi/2 - atan(1/x);
 *   t > tan(pi/8):      atan(t) = pi/4 + atan((t - 1)/(t + 1));
 *   |u| <= tan(pi/8):   atan(u) = 2 atan(v),  v = u / (1 + sqrt(1 + u^2)),
 *                       |v| <= tan(pi/16) < 0.2;
 *   atan(v) = v - v^3/3 + v^5/5 - ... - v^27/27 (the first omitted term is
 *   below 0.04^14 / 29 of v, under 1e-21 relative).
 * pi/2 and pi/4 are carried as a head and a tail.  Within a few ulp of
 * atan over the reals (tests/test_oracle.py holds a 4-ulp bound against the
 * C library's atan).
 *
 * The FP64 kernels are compiled without FMA contraction and the oracle with
 * -ffp-contract=off, so both evaluate the same sequence of roundings.
 */
#ifndef FESOMC_ATAN_H
#define FESOMC_ATAN_H

#include <math.h>

#ifdef __CUDACC__
#define FESOMC_ATAN_FN static __host__ __device__ inline
#else
#define FESOMC_ATAN_FN static inline
#endif

/* pi/2 and pi/4: head and tail */
#define FESOMC_ATAN_PIO2_H 0x1.921fb54442d18p+0
#define FESOMC_ATAN_PIO2_L 0x1.1a62633145c07p-54
#define FESOMC_ATAN_PIO4_H 0x1.921fb54442d18p-1
#define FESOMC_ATAN_PIO4_L 0x1.1a62633145c07p-55
#define FESOMC_ATAN_TAN_PI8 0.41421356237309503

/* atan(v) for |v| < 0.2: the Taylor series to v^27 */
FESOMC_ATAN_FN double fesomc_atan_series(double v) {
    const double z = v * v;
    const double p = -(1.0 / 3.0) + z * ((1.0 / 5.0) + z * (-(1.0 / 7.0) + z * ((1.0 / 9.0) +
                     z * (-(1.0 / 11.0) + z * ((1.0 / 13.0) + z * (-(1.0 / 15.0) + z * ((1.0 / 17.0) +
                     z * (-(1.0 / 19.0) + z * ((1.0 / 21.0) + z * (-(1.0 / 23.0) + z * ((1.0 / 25.0) +
                     z * -(1.0 / 27.0))))))))))));
    return v + (v * z) * p;
}

/* atan(t) for 0 <= t <= 1 */
FESOMC_ATAN_FN double fesomc_atan01(double t) {
    if (t > FESOMC_ATAN_TAN_PI8) {
        const double u = (t - 1.0) / (t + 1.0);
        const double v = u / (1.0 + sqrt(1.0 + u * u));
        return FESOMC_ATAN_PIO4_H + (2.0 * fesomc_atan_series(v) + FESOMC_ATAN_PIO4_L);
    }
    const double v = t / (1.0 + sqrt(1.0 + t * t));
    return 2.0 * fesomc_atan_series(v);
}

FESOMC_ATAN_FN double fesomc_atan(double x) {
    if (x != x) return x;
    const double a = fabs(x);
    double r;
    if (a > 1.0) r = FESOMC_ATAN_PIO2_H + (FESOMC_ATAN_PIO2_L - fesomc_atan01(1.0 / a));
    else r = fesomc_atan01(a);
    return x < 0.0 ? -r : r;
}

#endif
