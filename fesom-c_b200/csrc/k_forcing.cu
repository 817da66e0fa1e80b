// Forcing on the device: the per-step inputs that the reference's forcing
// routines compute on the host (the harmonic open-boundary elevation of
// compute_ssh_rhs_elem, src/fv_average_dynamic.F90:190-216, and the river
// runoff of rivers_do with its 10-day ramp, src/fv_rivers.F90:263-299),
// evaluated by two small kernels at the head of every internal step, so
// that a step needs no host-to-device copy.  The device keeps its own copy
// of time_jd, advanced with the main loop's expression (fv_main.F90:400).
// The arithmetic is the host forcing path's, operation for operation
// (fesomc_cos is shared by both), so both give the same bits.
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
