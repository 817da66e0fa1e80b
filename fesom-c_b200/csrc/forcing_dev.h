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

// Inputs of the tidal potential kernel: the step's time_jd from 'clock'
// (advanced by k_forcing_clock, or uploaded by the host path), node
// coordinates (lon, lat) in radians, the harmonic switches a_th of the 11
// equilibrium waves (M2, S2, N2, K2, K1, O1, P1, Q1, Mf, Mm, Ssa).
struct PotentialDev {
    int N;
    double time_jd0;
    double ath[11];
    const double *clock;
    const double2 *coord;
    double *ssh_gp;
};

void launch_potential(const PotentialDev &p, cudaStream_t s);

}  // namespace fesomc
