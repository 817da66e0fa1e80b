// Shared device-side definitions of the B200 FESOM-C time step.
//
// Layout in HBM (device order == reference order in this version):
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


namespace fesomc {

constexpr double kG = 9.8;
constexpr double kREarth = 6400000.0;

struct Dev {
    // sizes
    int N, E, Ed, Ed_in, L, NS;
    int nobn, n_rivers;
    // scalar parameters
    double dt, dt_2D, Dmin, C_d, beta, epsilon, density_0, scale_area;
    double snul, z0b_min, z0s_min, Pr_num, beta_scale, cka, tau_inv_filt, K_hor, Cd_bz;
    double clim_relax, relax2clim_ac, river_salinity;
    int Mt, mom_adv_2D, mom_adv_3D, vert_adv, im_vert_visc, im_vert_visc_fic, fic_point;
    int tracer_adv, ver_mix, filt_2D, filt_3D, wet_dry_on, key_rivers, TF_presence, cl_relax;
    // mesh
    const double *sig;             // sigma(1:nsigma)
    const double *dsig;            // sigma(k)-sigma(k+1), k = 1..nsigma-1
    const int4 *elem_nodes, *elem_nb, *elem_edges;
    const int4 *elem_iedges;       // internal edges of the element, sorted, (edge<<1)|side, -1 pad
    const int2 *edge_nodes, *edge_tri;
    const int2 *edge_updn;         // MUSCL up/down-wind elements (or -1)
    const int *node_eptr, *node_eidx;   // CSR node -> (edge<<1)|side, sorted by edge
    const int *node_nptr, *node_nidx;   // CSR node -> elements (nod_in_elem2D order)
    const int *node_bptr, *node_bidx;   // CSR node -> boundary edges ((edge<<1)|side), sorted
    const int *node_rptr, *node_ridx;   // CSR node -> river entries (list order)
    const int *obn_of_node;        // open-boundary slot or -1
    const int *index_nod2D;
    const double4 *w_cv;
    const double4 *gs_x, *gs_y;    // gradient_sca(1:4), (5:8)
    const double4 *gv_x, *gv_y;    // gradient_vec(1:4), (5:8)
    const double *elem_area, *elem_cos, *coriolis, *area, *depth, *ac, *atp1, *atp2;
    const double *elem_acc;        // sum(w_cv*ac) per element
    const double *elem_bpfac;      // acc**Bp_bz * mask_bpr per element
    const double2 *edge_dxdy;
    const double4 *edge_cross;
    const double *node_tvol;       // sum(elem_area) over nod_in_elem2D (sequential)
    // 2D state
    double *eta_n, *eta_n_1, *eta_n_2, *eta_new, *etaAB, *ssh_gp, *eta_jac, *eta_jac_old;
    double2 *U_n_2D, *U_n_1, *U_n_2, *UAB, *U_rhs_2D_3D, *Bar_pr_2D;
    double4 *bfric;                       // per element for the sub-cycle: bottom U, V, a_Cd*|U|
    double2 *Fp;                          // per element: surface pressure force * elem_area (compute_vel_rhs)
    double *aux_elem, *dmean_n, *U_filt_2D, *V_filt_2D, *mask_wd, *mask_wd_node;
    double4 *vel_grad;
    double *taux, *tauy, *windx, *windy, *runoff, *ob_val;
    // 3D state (L per entity unless noted)
    double *U_n, *V_n, *U_rhsAB, *V_rhsAB, *U_n_filt, *V_n_filt, *U_rhs, *V_rhs;
    double *U_puls, *V_puls, *Unode, *Vnode, *Unode_p, *Vnode_p;
    double *vgux, *vguy, *vgvx, *vgvy, *Bar_pru, *Bar_prv;
    double *TF, *SF, *T_old, *S_old, *Tclim, *Sclim, *rho_c;
    double *hpressure, *bt, *snu, *Kv, *Ri, *tke_dissip, *Wvel;   // NS per node
    double *Av;                                                   // NS per element
    // element-level Jacobian quantities from eta_jac, refreshed by update3d
    // right after each jacobian call (and once at init):
    double *Je;                           // Je(k,e)                    L per element
    double *Ze;                           // SUM(w_cv*Z(k,nodes))       L per element
    double *ZBe;                          // SUM(w_cv*zbar(k,nodes))    L per element (interfaces 1..L)
    double *ttfold, *stfold;              // L per node, AB2 tracer minus its mean (this step)
    // MUSCL segment fluxes per (edge, level): (first, second segment) of
    // the T flux, the S flux and the continuity term
    double2 *mflT, *mflS, *mflC;
    double2 *adv2d;                       // per internal edge: upwind 2D momentum flux of the sub-step
    double2 *adv3;                        // per (internal edge, level): upwind 3D momentum flux (uu, vv)
    // tracer scratch
    double *TF_adv, *SF_adv, *Told_new, *Sold_new;
    double *ttx, *tty, *stx, *sty;       // L per element (MUSCL / Miura element gradients)
    double *tnx, *tny, *snx, *sny;       // L per node   (node-averaged gradients)
    double *tnow;                         // L per node: T minus its mean (Miura)
    double *mask_ad;                      // per node: advection-order mask (adv_tracer_mask)
    double *trhs_a, *trhs_b, *trhs_c;    // L per node scratch
    double *mm_part;                      // reduction partials
    double *aver;                         // [0]=T_aver [1]=S_aver
    unsigned int *status;                 // bit mask
    int *notconv;                         // columns with d3_end not converged
};

// ---- max/min exactly as the Fortran MAX/MIN of two values -------------------
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }

// ---- jacobian quantities (fv_main.F90:1228-1262) ------------------------------
// a = max(depth + eta, Dmin)
__device__ __forceinline__ double jac_a(const Dev &d, const double *eta, int n) {
    return dmax(d.depth[n] + eta[n], d.Dmin);
}
// Jc(k) with k 0-based layer index: a*(sigma(k)-sigma(k+1)) (dsig holds the
// difference, rounded exactly as the reference's sigma(1:L)-sigma(2:NS))
__device__ __forceinline__ double jc_of(const Dev &d, double a, int k) { return a * __ldg(d.dsig + k); }
// zbar(k), k 0-based interface index
__device__ __forceinline__ double zbar_of(const Dev &d, double a, int k) { return (1.0 - __ldg(d.sig + k)) * a; }
__device__ __forceinline__ double z_of(const Dev &d, double a, int k) {
    return 0.5 * (zbar_of(d, a, k) + zbar_of(d, a, k + 1));
}
// Je(k,e) = w1*Jc(k,n1) + w2*Jc(k,n2) + w3*Jc(k,n3) + w4*Jc(k,n4)
__device__ __forceinline__ double je_of(const Dev &d, const double4 &w, const double4 &a, int k) {
    return w.x * jc_of(d, a.x, k) + w.y * jc_of(d, a.y, k) + w.z * jc_of(d, a.z, k) + w.w * jc_of(d, a.w, k);
}
__device__ __forceinline__ double4 elem_jac_a(const Dev &d, const double *eta, const int4 &en) {
    return make_double4(jac_a(d, eta, en.x), jac_a(d, eta, en.y), jac_a(d, eta, en.z), jac_a(d, eta, en.w));
}
// Fortran SUM(w_cv(1:4,e)*x(nodes)) : sequential from 0
__device__ __forceinline__ double wsum(const double4 &w, double x1, double x2, double x3, double x4) {
    double s = 0.0;
    s = s + w.x * x1;
    s = s + w.y * x2;
    s = s + w.z * x3;
    s = s + w.w * x4;
    return s;
}
// explicit 4-term form w1*x1 + w2*x2 + w3*x3 + w4*x4
__device__ __forceinline__ double wexp(const double4 &w, double x1, double x2, double x3, double x4) {
    return w.x * x1 + w.y * x2 + w.z * x3 + w.w * x4;
}

// REAL(4) literal promoted to REAL(8)
#define R4(x) ((double)(x##f))

// densityJM, fv_pressure_new.F90:340-414 (no sediment)
__device__ __forceinline__ double density_jm(double t, double s, double pz, double density_0) {
    double ss3 = sqrt(s * s * s);
    double bulk = 19092.56 + t * (209.8925 - t * (3.041638 - t * (-R4(1.852732e-3) - t * (R4(1.361629e-5)))))
                + s * (104.4077 - t * (6.500517 - t * (.1553190 - t * (-R4(2.326469e-4)))))
                + ss3 * (-5.587545 + t * (0.7390729 - t * (R4(1.909078e-2))))
                - pz * (R4(4.721788e-1) + t * (R4(1.028859e-2) + t * (-R4(2.512549e-4) - t * (R4(5.939910e-7)))))
                - pz * s * (-R4(1.571896e-2) - t * (R4(2.598241e-4) + t * (-R4(7.267926e-6))))
                - pz * ss3 * R4(2.042967e-3)
                + pz * pz * (R4(1.045941e-5) - t * (R4(5.782165e-10) - t * (R4(1.296821e-7))))
                + pz * pz * s * (-R4(2.595994e-7) + t * (-R4(1.248266e-9) + t * (-R4(3.508914e-9))));
    double rhopot = 999.842594
                  + t * (R4(6.793952e-2) + t * (-R4(9.095290e-3) + t * (R4(1.001685e-4)
                  + t * (-R4(1.120083e-6) + t * R4(6.536332e-9)))))
                  + s * (0.824493 + t * (-R4(4.08990e-3) + t * (R4(7.64380e-5)
                  + t * (-R4(8.24670e-7) + t * R4(5.38750e-9)))))
                  + ss3 * (-R4(5.72466e-3) + t * (R4(1.02270e-4) + t * (-R4(1.65460e-6))))
                  + R4(4.8314e-4) * s * s;
    return rhopot * bulk / (bulk + 0.1 * pz) - density_0;
}

// ---- one warp per entity, lane = level ----------------------------------------
constexpr unsigned kFull = 0xffffffffu;
#define WARP_LOOP(ent, count)                                                                           \
    for (long long ent = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; ent < (long long)(count); \
         ent += ((long long)gridDim.x * blockDim.x) >> 5)

// levels handled by the chunk of 32 starting at z0
__device__ __forceinline__ int chunk_len(int L, int z0) { return L - z0 < 32 ? L - z0 : 32; }

// acc = (((acc + v_0) + v_1) + ... + v_{n-1}) with v_j held by lane j:
// the sequential Fortran sum, evaluated identically in every lane.
__device__ __forceinline__ double warp_seq_sum(double acc, double v, int n) {
    for (int j = 0; j < n; ++j) acc = acc + __shfl_sync(kFull, v, j);
    return acc;
}

// inclusive sequential prefix: lane j receives acc + v_0 + ... + v_j (left
// to right); acc is advanced past all n values in every lane.
__device__ __forceinline__ double warp_seq_scan(double &acc, double v, int n) {
    const int lane = threadIdx.x & 31;
    double mine = 0.0;
    for (int j = 0; j < n; ++j) {
        acc = acc + __shfl_sync(kFull, v, j);
        if (lane == j) mine = acc;
    }
    return mine;
}

// grid-stride helper
#define GRID_LOOP(i, n) for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); \
                             i += (long long)gridDim.x * blockDim.x)

// launch helpers (implemented in model.cu)
int grid_for(long long n, int block);

}  // namespace fesomc
