// Device view of the forcing that fesomc_gpu_set_device_forcing moves onto
// the GPU (kernels in k_forcing.cu, set-up in model.cu).
#pragma once
#include <cuda_runtime.h>

namespace fesomc {

// pi as the reference defines it (fv_var.F90:8), used in the tide phase
constexpr double kPiRef = 3.14159265358979;

struct ForcingDev {
    int nobn, n_rivers, Mt;
    int restart;                  // no 10-day tide ramp after a restart
    int tides_on, rivers_on, river_ramp;
    double dt, dt_2D, time_jd0;
    double *clock;                // [0]: time_jd of the step being computed
    const double *ampt, *fazt;    // (12, nobn) harmonic amplitudes / phases, harmonic-major
    const double *harm;           // amp_factor[12], phy_factor[12], period in hours[12]
    const double *runoff_base;    // n_rivers
    double *ob_val, *runoff;      // the model's step inputs
};

void launch_forcing(const ForcingDev &f, cudaStream_t s);

}  // namespace fesomc
