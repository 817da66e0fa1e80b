// Shared device-side definitions of the B200 FESOM-C time step.
//
// Layout in HBM (device order: the reference order, or with sfc_order the
// order of a Hilbert curve through the mesh, every index translated):
//   * 2D node / element fields: one double per entity.
//   * 2D vectors (U_n_2D, UAB, ...): double2 per element (u, v interleaved,
//     as the Fortran (2,E) arrays).
//   * Level fields: [entity][level] with levels contiguous, exactly the
//     Fortran (nsigma-1, N) / (nsigma, N) arrays, so a column is one
//     contiguous run of L (or NS) doubles.
//   * Connectivity: 0-based int4 / int2; absent neighbour / second element
//     of a boundary edge = -1.
//   * Edge scatters of the reference become gathers over CSR lists that are
//     sorted by the reference edge number, so every node / element receives
//     its contributions in the same order as the serial Fortran loop and the
//     FP64 sums are bit-identical (compiled with --fmad=false).
//   * Jc, Jd, Z, zbar (subroutine jacobian, fv_main.F90:1208-1267) are not
//     stored: they are recomputed with the same expressions from the
//     elevation at the last jacobian call (eta_jac) and sigma.  The element
//     quantities Je and the w_cv-weighted Z / zbar, which every element
//     kernel needs at every level, are stored once per jacobian call.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "fesomc_log.h"
#include "fesomc_trig.h"

// FP32 form: the closure's logarithm is the device logf (the FP64 path uses
// fesomc_log, bit-identical with the oracle's).
static __device__ __forceinline__ float fesomc_log(float x) { return logf(x); }

// Each kernel source is compiled twice: with FESOMC_FP32 = 0 into
// fesomc::f64 (the FP64 path, bit-exact with the reference's algorithm) and
// with FESOMC_FP32 = 1 into fesomc::f32 (the precision form: level fields,
// mesh geometry and the 3D arithmetic in FP32; the 2D sub-cycle state in
// FP64).
#ifndef FESOMC_FP32
#define FESOMC_FP32 0
#endif

namespace fesomc {

constexpr double kG64 = 9.8;
constexpr double kPref = 101325.0;   // P_ref, reference atmospheric pressure (fv_var.F90:17)

// Raises (never lowers) a kernel's dynamic shared-memory limit.  The
// attribute belongs to the kernel, and every model instance of the process
// (ensemble members of different level counts, both precision forms)
// launches the same kernels, so one instance must not shrink another's.
template <typename K>
inline cudaError_t raise_smem_limit(K kernel, size_t bytes) {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, kernel);
    if (e != cudaSuccess) return e;
    if (bytes <= (size_t)a.maxDynamicSharedSizeBytes) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// ---- max/min exactly as the Fortran MAX/MIN of two values -------------------
template <typename T>
__device__ __forceinline__ T dmax(T a, T b) { return a > b ? a : b; }
template <typename T>
__device__ __forceinline__ T dmin(T a, T b) { return a < b ? a : b; }

__host__ __device__ __forceinline__ double2 make_real2(double x, double y) { return make_double2(x, y); }
__host__ __device__ __forceinline__ float2 make_real2(float x, float y) { return make_float2(x, y); }
__host__ __device__ __forceinline__ double4 make_real4(double x, double y, double z, double w) {
    return make_double4(x, y, z, w);
}
__host__ __device__ __forceinline__ float4 make_real4(float x, float y, float z, float w) {
    return make_float4(x, y, z, w);
}

// Launch-shape knobs (fesomc_gpu_tune_*): threads per block of the kernels
// whose results do not depend on the block shape (one thread per entity or
// per (entity, level), grid-stride, no block-level reduction), and entities
// per block of the column kernels (pressure_col, bpg_elem, update3d, wvel),
// and the form of d3_end (1 column arrays in local memory, 2 in shared
// memory, 3 a level-parallel set-up kernel and a sweep kernel, 4 the same
// with the sweep's arrays in shared memory, 5 and 6 in registers for 11 or
// 21 levels), and the form of the tracers'
// implicit vertical diffusion (1 one thread per column reading the fields
// directly, 2 and 3 tiles of 128 or 64 columns staged in shared memory, for
// 10 or 20 layers; other layer counts take form 1), and the form of the
// implicit vertical viscosity (1 one thread per element column reading the
// fields directly, 2 tiles of 64 columns staged in shared memory: the fic
// variant, 10 or 20 layers).  A value of 0 selects the built-in default.
enum TuneKnob : int {
    TK_VELRHS, TK_VELGRAD3D, TK_ADV3, TK_PULS, TK_EL2NODES, TK_P1EDGE, TK_AB3, TK_VELGRAD2D, TK_SSHEDGE,
    TK_SSHNODE, TK_ADV2D, TK_U2D, TK_ROT, TK_ZEROFILT, TK_AB2, TK_MEGRAD, TK_MNGRAD, TK_MEDGE, TK_MH,
    TK_UPWIND, TK_AV, TK_COLUMNS, TK_D3END, TK_VDIFF, TK_IMPLVISC, kTuneKnobs
};

// sbc_do on the device (fesomc_gpu_set_atm_fields): the time-interpolation
// coefficients of the 8 atmospheric fields per node (device order, 8
// consecutive values per node), the device clock, a scratch for the stress
// per node (2 values per node), and the namelist's nm_net_flux and
// nm_prec_coef
struct AtmDev {
    const double *coef_a, *coef_b, *clock;
    double *tau_node;
    int net_flux;
    double prec_coef;
};

namespace f64 {
using real = double;
using real2 = double2;
using real4 = double4;
#include "dev_struct.inc"
}  // namespace f64
namespace f32 {
using real = float;
using real2 = float2;
using real4 = float4;
#include "dev_struct.inc"
}  // namespace f32

// full-warp mask of the level shuffles (levels on consecutive lanes)
constexpr unsigned kFull = 0xffffffffu;

// grid-stride helper
#define GRID_LOOP(i, n) for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); \
                             i += (long long)gridDim.x * blockDim.x)

// launch helpers (implemented in model.cu)
int grid_for(long long n, int block);


}  // namespace fesomc

#if FESOMC_FP32
#define FESOMC_PREC_BEGIN namespace fesomc { namespace f32 {
#else
#define FESOMC_PREC_BEGIN namespace fesomc { namespace f64 {
#endif
#define FESOMC_PREC_END } }

FESOMC_PREC_BEGIN
#include "dev_helpers.inc"
FESOMC_PREC_END
