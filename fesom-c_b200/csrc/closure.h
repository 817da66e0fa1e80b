// Learned vertical-mixing closure: a per-column network that stands in for
// d3_end (src/fv_mixing.F90:73-347).  No counterpart in the reference.
//
// Network: IN = 3*NS + 3 inputs, three hidden layers of 256 with SiLU,
// OUT = NS outputs; layer l computes Z = A W^T + b with W row-major
// (out x in); the flat parameter vector is W1 b1 W2 b2 W3 b3 W4 b4.
//
// Inputs per node column (NS interfaces, 0-based k; before the transform):
//   k in [0, NS):      squared shear at interface k, s^-2 (0 at the surface
//                      and the bottom interface)
//   k in [NS, 2NS):    buoyancy frequency squared at interface k - NS, s^-2
//   k in [2NS, 3NS):   depth of interface k - 2NS below the surface, m
//   3NS, 3NS+1, 3NS+2: surface TKE flux term 0.05 |wind|^2, bottom TKE value
//                      bott_R |U_b|^2, total depth, m
// Shear, N^2 and the two boundary terms enter as asinh(x / x0) with x0 =
// 1e-6 (they span many decades and N^2 changes sign); every input is then
// normalised by the training set's mean and standard deviation.
// Outputs: log bt (the turbulence energy d3_end advances) per interface,
// normalised the same way.  snu and Kv follow from bt exactly as d3_end
// forms them (snu = scale_t sqrt(bt) + snul, capped at 0.2; Kv = Pr_num snu),
// so the network's bt, snu and Kv are one consistent closure state, and the
// plain closure restarts from a bt inside its own range.
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace fesomc {

constexpr int kLcHidden = 256;
constexpr float kLcX0 = 1.0e-6f;
// fallback rules beyond the training envelope (fesomc_closure_set_rules)
constexpr int kLcRuleUnstable = 1;   // N^2 < 0 at an interior interface: the plain closure
constexpr int kLcRuleBoundary = 2;   // solid or open boundary node (index_nod2D != 0): the plain closure

inline int lc_in(int NS) { return 3 * NS + 3; }
inline int lc_out(int NS) { return NS; }
// nodes per block of the harvest's ordered compaction
constexpr int kLcHarvestBlock = 256;
// rows of the statistics array (each max(IN, OUT) floats)
constexpr int kLcStatRows = 8;

// the device-side pieces the step kernels need (features, application,
// envelope test and judge statistics); the state kernels are compiled per
// precision and read these through a plain struct
struct LcView {
    int NS, IN, OUT;
    int rules;                                // kLcRule* bits
    const float *mu_x, *sd_x, *mu_y, *sd_y;   // normalisation (IN / OUT)
    const float *lo_x, *hi_x;                 // training envelope of the normalised inputs
    const float *lo_y, *hi_y;                 // range of the training targets (log bt, not normalised)
    float *X;                                 // per node: normalised inputs (N x IN), FP32
    float *Y;                                 // per node: network outputs (N x OUT), normalised
    int *flag;                                // per node: 1 = network, 0 = plain closure
    int *list;                                // nodes handed to the plain closure
    int *blk;                                 // harvest: per block of kLcHarvestBlock nodes, its wet count, then its first slot
    unsigned long long *count;                // [0] list length
    unsigned long long *acc;                  // [0] wet columns [1] out of envelope [2] dry [3] steps
    double *judge;                            // [0] sum of squared log-errors [1] count [2] max
    // harvest: raw inputs / targets appended at hcount
    float *hx, *hy;
    int64_t hcap;
    unsigned long long *hcount;
};

}  // namespace fesomc
