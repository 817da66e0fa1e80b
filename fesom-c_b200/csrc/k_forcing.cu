// Forcing on the device: the per-step inputs that the reference's forcing
// routines compute on the host (the harmonic open-boundary elevation of
// compute_ssh_rhs_elem, src/fv_average_dynamic.F90:190-216, and the river
// runoff of rivers_do with its 10-day ramp, src/fv_rivers.F90:263-299),
// evaluated by two small kernels at the head of every internal step, so
// that a step needs no host-to-device copy.  The device keeps its own copy
// of time_jd, advanced with the main loop's expression (fv_main.F90:400).
// The arithmetic is the host forcing path's, operation for operation
// (fesomc_cos is shared by both), so both give the same bits.  A third
// kernel evaluates the tidal potential (T_potential) into ssh_gp.
#include "device_common.cuh"
#include "forcing_dev.h"

namespace fesomc {

// time_jd = time_jd + dt/86400 (one thread)
__global__ void k_forcing_clock(ForcingDev f) {
    if (blockIdx.x == 0 && threadIdx.x == 0) f.clock[0] = f.clock[0] + f.dt / 86400.0;
}

// open-boundary elevation of the Mt sub-steps (slot sub*nobn + q) and the
// river runoff of the step
__global__ void k_forcing_values(ForcingDev f) {
    const double time_jd = f.clock[0];
    const double time = time_jd * 86400.0;
    const long long n_ob = f.tides_on ? (long long)f.Mt * f.nobn : 0;
    const long long n_riv = f.rivers_on ? f.n_rivers : 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_ob + n_riv;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < n_ob) {
            const int sub = (int)(i / f.nobn), q = (int)(i % f.nobn);
            const double time_2D = time + f.dt_2D * (sub + 1);
            double v = 0.0;
            for (int j = 0; j < 12; ++j)
                v = v + f.harm[j] * f.ampt[(size_t)f.nobn * j + q] *
                            fesomc_cos((time_2D - f.time_jd0 * 86400.0) * 2.0 * kPiRef / (f.harm[24 + j] * 3600.0) -
                                       (f.fazt[(size_t)f.nobn * j + q] + f.harm[12 + j]));
            if (!f.restart)
                if (time_jd - f.time_jd0 < 10.0) v = v * (time_jd - f.time_jd0) / 10.0;
            f.ob_val[i] = v;
        } else {
            const long long r = i - n_ob;
            double b = f.runoff_base[r];
            if (f.river_ramp && time_jd - f.time_jd0 < 10.0) b = b * (time_jd - f.time_jd0) / 10.0;
            f.runoff[r] = b;
        }
    }
}

__device__ __forceinline__ double control_360(double fr) {
    const int iz = (int)(fr / 360.0);
    if (iz >= 1) fr = fr - (double)iz * 360.0;
    return fr;
}

// potential (src/fv_tide_potential.F90:1-107): the equilibrium tide into
// ssh_gp, one node per thread.  The astronomical arguments h0, s0, p0 and
// the phases sxi depend on the step only; every thread forms them itself
// (a few dozen operations against the 11 cosines of a node).
__global__ void k_potential(PotentialDev p) {
    const double Apt[11] = {0.242334, 0.112841, 0.046398, 0.030704, 0.141565, 0.100514,
                            0.046843, 0.019256, 0.041742, 0.022026, 0.019446};
    const double Fpt[11] = {1.40519e-4, 1.45444e-4, 1.37880e-4, 1.45842e-4, 0.72921e-4, 0.67598e-4,
                            0.72523e-4, 0.64959e-4, 0.53234e-5, 0.26392e-5, 0.03982e-5};
    const double rad = kPiRef / 180.0;
    const double time_jd = p.clock[0];
    const double DY = time_jd - 2442413.5;             // days from 1975-01-01
    const double TY = (27392.500528 + 1.0000000356 * DY) / 36525.0;
    const double TY2 = TY * TY, TY3 = TY2 * TY;
    const double h0 = control_360(279.69668 + 36000.768930485 * TY + 3.03e-4 * TY2);
    const double s0 = control_360(270.434358 + 481267.88314137 * TY - 0.001133 * TY2 + 1.9e-6 * TY3);
    const double p0 = control_360(334.329653 + 4069.0340329575 * TY - 0.010325 * TY2 - 1.2e-5 * TY3);
    double sxi[11];
    sxi[0] = (h0 - s0) * 2.0 * rad;                    // M2
    sxi[1] = 0.0;                                      // S2
    sxi[2] = (2.0 * h0 - 3.0 * s0 + p0) * rad;         // N2
    sxi[3] = 2.0 * h0 * rad;                           // K2
    sxi[4] = (h0 + 90.0) * rad;                        // K1
    sxi[5] = (h0 - 2.0 * s0 - 90.0) * rad;             // O1
    sxi[6] = (h0 - 90.0) * rad;                        // P1
    sxi[7] = (h0 - 3.0 * s0 + p0 - 90.0) * rad;        // Q1
    sxi[8] = 2.0 * s0 * rad;                           // Mf
    sxi[9] = (s0 - p0) * rad;                          // Mm
    sxi[10] = 2.0 * h0 * rad;                          // Ssa
    double tcor[11];
    for (int j = 0; j < 11; ++j) tcor[j] = DY * 86400.0 - sxi[j] / Fpt[j];
    const bool ramp = time_jd - p.time_jd0 < 5.0;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < p.N;
         n += (long long)gridDim.x * blockDim.x) {
        const double2 c = p.coord[n];
        const double sl = fesomc_sin(0.5 * kPiRef - c.y);
        const double s2 = fesomc_sin(2.0 * (0.5 * kPiRef - c.y));
        double ssh_sd = 0.0, ssh_d = 0.0, ssh_lp = 0.0;
        for (int j = 0; j < 4; ++j)
            ssh_sd = ssh_sd + p.ath[j] * Apt[j] * sl * sl * fesomc_cos(Fpt[j] * tcor[j] + 2.0 * c.x + sxi[j]);
        for (int j = 4; j < 8; ++j)
            ssh_d = ssh_d + p.ath[j] * Apt[j] * s2 * fesomc_cos(Fpt[j] * tcor[j] + c.x + sxi[j]);
        for (int j = 8; j < 11; ++j)
            ssh_lp = ssh_lp + p.ath[j] * Apt[j] * (3.0 * (sl * sl) - 2.0) * fesomc_cos(Fpt[j] * tcor[j] + sxi[j]);
        double v = ssh_sd + ssh_d + ssh_lp;
        if (ramp) v = v * (time_jd - p.time_jd0) / 5.0;
        p.ssh_gp[n] = v;
    }
}

void launch_potential(const PotentialDev &p, cudaStream_t s) {
    const int block = 256;
    long long g = ((long long)p.N + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148 * 8) g = 148 * 8;
    k_potential<<<(int)g, block, 0, s>>>(p);
}

void launch_forcing(const ForcingDev &f, cudaStream_t s) {
    k_forcing_clock<<<1, 32, 0, s>>>(f);
    const long long n = (f.tides_on ? (long long)f.Mt * f.nobn : 0) + (f.rivers_on ? f.n_rivers : 0);
    const int block = 128;
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148) g = 148;
    k_forcing_values<<<(int)g, block, 0, s>>>(f);
}

}  // namespace fesomc
