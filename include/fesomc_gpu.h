/*
 * fesomc_gpu.h -- C-ABI of the B200 (sm_100a) FESOM-C ocean time step.
 *
 * The reference hot path (FESOM-C, Fortran 90) consists of argument-less
 * subroutines that read and write module globals (o_PARAM / o_MESH /
 * o_ARRAYS, src/fv_var.F90:1-438).  The Fortran driver calls them from
 * oce_timestep (src/fv_main.F90:1877-2106).  This library replaces the body
 * of oce_timestep for type_task 3 (src/fv_main.F90:1983-2095): the driver
 * keeps reading namelists, the mesh and forcing, and keeps writing output;
 * it hands the already-built module arrays to fesomc_gpu_init once, pushes
 * forcing each internal step with fesomc_gpu_set_forcing, advances with
 * fesomc_gpu_step and pulls state back with fesomc_gpu_sync_to_host before
 * output, energy diagnostics and restarts.
 *
 * Conventions
 *  - All arrays are in the reference's Fortran layout: a field dimensioned
 *    (K, M) in Fortran is passed as a C pointer to K*M values with the first
 *    index fastest (levels contiguous per node / element).
 *  - Connectivity arrays carry 1-based indices exactly as the Fortran module
 *    arrays hold them; boundary markers (edge_tri(2,:) = -999,
 *    elem_neighbors <= 0) are kept.  The library converts on the host.
 *  - Every entry point returns 0 on success or one of FESOMC_E* (> 0).
 *  - The whole mesh lives on one GPU: there is no halo exchange (the MPI
 *    g_comm / exchange_* calls of the reference drop out).  The caller passes
 *    its MPI rank count in fesomc_params.npes; fesomc_gpu_init returns
 *    FESOMC_EINVAL for npes > 1 (0 is read as 1).
 *  - Call from one host thread, outside any OpenMP parallel region.
 */
#ifndef FESOMC_GPU_H
#define FESOMC_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes -------------------------------------------------------- */
#define FESOMC_OK            0
#define FESOMC_EINVAL        1  /* bad argument / unsupported option          */
#define FESOMC_ENOMEM        2  /* device or host allocation failed          */
#define FESOMC_ECUDA         3  /* a CUDA runtime call failed                */
#define FESOMC_ESTATE        4  /* call out of order (e.g. step before init) */
#define FESOMC_ENEGSALT      5  /* negative salinity  (fv_tracer.F90:1469-1473) */
#define FESOMC_ELOWTEMP      6  /* temperature < -3 C (fv_tracer.F90:1478-1482) */
#define FESOMC_ENONFINITE    7  /* NaN / Inf found in the prognostic state    */
#define FESOMC_ENOTCONV      8  /* d3_end hit its 200-iteration cap (reported,
                                   not fatal; see fesomc_gpu_last_status)   */
#define FESOMC_EMESH         9  /* mesh builder: inconsistent node list
                                   (test_elem "Node list problem", fv_mesh_array.F90:62-66) */

/* ---- status word bits (device side, read back once per step) ------------ */
#define FESOMC_ST_NEGSALT    0x1u
#define FESOMC_ST_LOWTEMP    0x2u
#define FESOMC_ST_NONFINITE  0x4u
#define FESOMC_ST_NOTCONV    0x8u

/* ---- field masks for sync ----------------------------------------------- */
#define FESOMC_F_ETA      0x0001u /* eta_n, eta_n_1, eta_n_2, etaAB           */
#define FESOMC_F_UV2D     0x0002u /* U_n_2D, U_n_1, U_n_2, U_filt_2D, V_filt_2D */
#define FESOMC_F_UV3D     0x0004u /* U_n, V_n, U_rhsAB, V_rhsAB, U_n_filt, V_n_filt */
#define FESOMC_F_TS       0x0008u /* TF, SF, T_old, S_old                     */
#define FESOMC_F_MIX      0x0010u /* bt, snu, Kv, Av, Ri, tke_dissip           */
#define FESOMC_F_WVEL     0x0020u /* Wvel                                     */
#define FESOMC_F_MASK     0x0040u /* mask_wd, mask_wd_node                     */
#define FESOMC_F_CLIM     0x0080u /* Tclim, Sclim                              */
#define FESOMC_F_DIAG     0x0100u /* rho_c, hpressure, Bar_pr_2D               */
#define FESOMC_F_ALL      0xFFFFu

/* ---- option values (fv_run.dat keys, src/fv_read_run.F90) --------------- */
#define FESOMC_TRACER_UPWIND 1    /* tracer_adv = 1 : solve_tracer_upwind     */
#define FESOMC_TRACER_MUSCL  2    /* tracer_adv = 2 : solve_tracer_muscl      */
#define FESOMC_TRACER_MIURA  4    /* tracer_adv = 4 : solve_tracer_miura      */

/*
 * Mesh, as left in o_MESH by read_mesh_ser / find_edges / find_elem_neighbors
 * / mesh_arrays1 / mesh_arrays2 / SET_SIGMA (src/fv_main.F90:787-945,
 * src/fv_mesh_array.F90:1-1386, src/fv_vert_coord.F90:135-280).
 */
typedef struct fesomc_mesh {
    int32_t nod2D, elem2D, edge2D, edge2D_in, nsigma;
    int32_t nod_in_elem2D_max;        /* leading dimension of nod_in_elem2D   */
    const int32_t *index_nod2D;       /* (nod2D) 0 interior, 1 solid, 2 open   */
    const int32_t *elem2D_nodes;      /* (4,elem2D); triangles: node4 = node1 */
    const int32_t *edge_nodes;        /* (2,edge2D)                           */
    const int32_t *edge_tri;          /* (2,edge2D); el2 = -999 on boundary   */
    const int32_t *elem_edges;        /* (4,elem2D)                           */
    const int32_t *elem_neighbors;    /* (4,elem2D); <= 0 on the boundary     */
    const int32_t *nod_in_elem2D_num; /* (nod2D)                              */
    const int32_t *nod_in_elem2D;     /* (nod_in_elem2D_max,nod2D)            */
    const int32_t *edge_up_dn_tri;    /* (2,edge2D) or NULL (MUSCL only)      */
    const double  *coord_nod2D;       /* (2,nod2D) radians                    */
    const double  *depth;             /* (nod2D)                              */
    const double  *area;              /* (nod2D)                              */
    const double  *elem_area;         /* (elem2D)                             */
    const double  *elem_cos;          /* (elem2D)                             */
    const double  *coriolis;          /* (elem2D)                             */
    const double  *w_cv;              /* (4,elem2D)                           */
    const double  *gradient_sca;      /* (8,elem2D)                           */
    const double  *gradient_vec;      /* (8,elem2D)                           */
    const double  *edge_dxdy;         /* (2,edge2D)                           */
    const double  *edge_cross_dxdy;   /* (4,edge2D)                           */
    const double  *sigma;             /* (nsigma)                             */
    const double  *a_tp;              /* (nod2D,2)  (fv_ini.F90:94-107)       */
    const double  *ac;                /* (nod2D) sponge factor, 1 = none      */
    /* open-boundary nodes (my_in_obn, read_mesh_ser fv_main.F90:841-851)    */
    int32_t nobn;
    const int32_t *in_obn;            /* (nobn) 1-based node ids              */
    /* river nodes (my_nod_rivers, fv_rivers.F90)                            */
    int32_t n_rivers;
    const int32_t *nod_rivers;        /* (n_rivers) 1-based node ids          */
} fesomc_mesh;

/*
 * Resolved run parameters (o_PARAM after READ_DATA_RUN and initial_state).
 * Booleans are 0/1.  Times in seconds unless noted.
 */
typedef struct fesomc_params {
    double dt, dt_2D;             /* Mt = int(dt/dt_2D) (fv_read_run.F90:1060) */
    int32_t Mt;
    double Dmin;
    double C_d;                   /* C_d_el = C_d (fv_average_dynamic.F90:262) */
    double beta, epsilon;         /* AB3 / AB2 coefficients (fv_var.F90:108,110) */
    double density_0;             /* set by initial_state (fv_ini.F90:187-199)  */
    double scale_area;            /* sum(elem_area)/elem2D (fv_ini.F90:81)      */
    double snul, z0b_min, z0s_min, Pr_num, beta_scale, cka;
    double tau_inv_filt, K_hor, Cd_bz, Bp_bz;
    double clim_relax, relax2clim_ac;   /* already in 1/s (fv_read_run.F90:884,894) */
    double river_salinity;        /* 0.2 psu in the reference (fv_main.F90:1818) */
    double time_jd0;              /* JD0 (days)                                 */
    int32_t mom_adv_2D;           /* 2 = upwind (only value on the path)       */
    int32_t mom_adv_3D;           /* 1 = upwind                                */
    int32_t vert_adv;             /* 1 = upwind QUICK                          */
    int32_t im_vert_visc;         /* momentum_vert_impl_visc                   */
    int32_t im_vert_visc_fic;     /* momentum_vert_impl_visc_tmp (fictitious point) */
    int32_t fic_point;            /* 0, 1, 2                                   */
    int32_t tracer_adv;           /* FESOMC_TRACER_*                           */
    int32_t ver_mix;              /* 3 = d3_end (only closure that runs)       */
    int32_t filt_2D, filt_3D;     /* viscosity_filt_2D / _3D / _3D_to_2D        */
    int32_t wet_dry_on;
    int32_t key_rivers;
    int32_t TF_presence;          /* open-boundary tides                       */
    int32_t restart;              /* hot start: no 10-day OB ramp              */
    int32_t cl_relax;
    int32_t cl_solid_boder_relax; /* not supported: must be 0                  */
    int32_t temp_on, salinity_on; /* type_task 3 when either is set            */
    int32_t n_harm;               /* number of tidal harmonics in use (<=12)    */
    int32_t harm_index[12];       /* 0-based index into the 12 reference waves  */
    /* Arithmetic form (no counterpart in the reference, which is FP64):
     * 0 = plain FP64 (bit-exact with the reference algorithm);
     * 1 = FP32 form: level fields, the 2D momentum, mesh geometry and the
     *     flux / advection / viscosity / tracer / mixing arithmetic in FP32;
     *     the elevation, SSH and total-depth accumulation, wet/dry tests
     *     and the energy integral stay FP64.  Its kernels are compiled
     *     with FMA contraction and FP32 division / square root to 2 ulp;
     *     its results are deterministic but not those of form 0.          */
    int32_t fp32_form;
    /* biharmonic viscosity of the 3D momentum (bih_3D, Abh0 of fv_run.dat,
     * src/fv_read_run.F90:320-326,396-401; biharmonic_viscosity,
     * src/fv_viscosity.F90:104-334)                                        */
    int32_t bih_3D;
    double Abh0;
    /* filter-2x viscosities (filt_bi_3D / filt_bi_2D, tau_c of fv_run.dat,
     * src/fv_read_run.F90:336-342; viscosity_filt2x_3D / _2D,
     * src/fv_viscosity.F90:570-767)                                         */
    int32_t filt_bi_3D, filt_bi_2D;
    double tau_c;
    /* biharmonic viscosity of the 2D momentum (bih_2D; biharmonic_2D,
     * src/fv_viscosity.F90:338-568), with Abh0                              */
    int32_t bih_2D;
    /* tidal potential (T_potential of fv_run.dat, src/fv_read_run.F90:651):
     * potential (src/fv_tide_potential.F90:1-107, called at the head of
     * oce_timestep, src/fv_main.F90:1899) writes the equilibrium tide of
     * the harmonics in harm_index (M2..Ssa) into ssh_gp every step, on the
     * device; build the mesh with the same flag for its a_tp
     * (src/fv_ini.F90:94-107).                                              */
    int32_t T_potential;
    /* number of MPI ranks of the calling driver (npes, g_PARSUP).  The whole
     * mesh lives on one GPU, so fesomc_gpu_init rejects npes > 1 with
     * FESOMC_EINVAL; 0 (a zero-initialised struct) is read as 1.           */
    int32_t npes;
    /* atmospheric forcing (key_atm of fv_run.dat, src/fv_read_run.F90:768):
     * the sea-level pressure and E - P in the elevation gradient of
     * update_2D_vel (src/fv_average_dynamic.F90:278-286) and in the surface
     * pressure force of compute_vel_rhs (src/fv_3D_vel.F90:40-53), and the
     * shortwave / non-solar heat source and the E - P freshwater source of
     * tracer_impl_vert_diff (src/fv_tracer.F90:1376,1396-1418;
     * calc_heat_flux_sw :1636-1697, calc_evap_precip :1699-1752, sw_cp
     * :1775-1908) from the fesomc_forcing fields mslp, emp, qsr, qns.
     * type_swr_body: 1 = Paulson-Simpson / Jerlov two-band profile, 2 =
     * Soloviev (src/fv_read_run.F90:793-803); with type_swr_body 1 and
     * jer_const = 1 the water type is Rjc, ajc, bjc (the R, a, b keys,
     * :825-856), with jer_const = 0 the per-node Rj, aj, bj of the forcing
     * (required before the first step, else FESOMC_ESTATE).               */
    int32_t key_atm;
    int32_t type_swr_body;
    int32_t jer_const;
    double Rjc, ajc, bjc;
    /* Storage order on the device (no counterpart in the reference):
     * 0 = the reference numbering; 1 = nodes, elements and edges stored
     * along a Hilbert curve through their positions (internal and boundary
     * edges each in their own range), so that neighbour gathers of meshes
     * numbered in file order touch nearby memory.  The permutation is kept
     * by the library: every array crossing the C-ABI stays in the reference
     * numbering, and every edge-ordered sum still runs in reference edge
     * order, so results are the same bits in both orders.  Needs
     * coord_nod2D.                                                          */
    int32_t sfc_order;
} fesomc_params;

/*
 * Prognostic state (o_ARRAYS) exchanged with the host.  Every pointer may be
 * NULL on sync_to_host when its field group is not requested.
 */
typedef struct fesomc_state {
    double *eta_n, *eta_n_1, *eta_n_2, *etaAB;        /* (nod2D)              */
    double *U_n_2D, *U_n_1, *U_n_2;                   /* (2,elem2D)           */
    double *U_filt_2D, *V_filt_2D;                    /* (elem2D)             */
    double *U_n, *V_n, *U_rhsAB, *V_rhsAB;            /* (nsigma-1,elem2D)    */
    double *U_n_filt, *V_n_filt;                      /* (nsigma-1,elem2D)    */
    double *TF, *SF, *T_old, *S_old;                  /* (nsigma-1,nod2D)     */
    double *Tclim, *Sclim;                            /* (nsigma-1,nod2D)     */
    double *bt, *snu, *Kv, *Ri, *tke_dissip;          /* (nsigma,nod2D)       */
    double *Av;                                       /* (nsigma,elem2D)      */
    double *Wvel;                                     /* (nsigma,nod2D)       */
    double *mask_wd;                                  /* (elem2D)             */
    double *mask_wd_node;                             /* (nod2D)              */
    double *ssh_gp;                                   /* (nod2D) tidal geopotential */
    double *rho_c;                                    /* (nsigma-1,nod2D)     */
    double *hpressure;                                /* (nsigma,nod2D)       */
    double *Bar_pr_2D;                                /* (2,elem2D)           */
    int32_t lfirst;                                   /* AB start flag (fv_var.F90:244) */
    double time_jd;                                   /* model time (days)    */
} fesomc_state;

/*
 * Per-internal-step forcing (what rivers_do / sbc_do / obc_do leave in
 * o_ARRAYS, src/fv_main.F90:412-431).  NULL = keep previous values.
 */
typedef struct fesomc_forcing {
    const double *taux, *tauy;      /* (elem2D) surface stress, N/m^2          */
    const double *windx, *windy;    /* (nod2D) 10 m wind, m/s                  */
    const double *runoff_rivers;    /* (n_rivers) m^3/s, ramp already applied  */
    const double *Tclim, *Sclim;    /* (nsigma-1,nod2D)                        */
    const double *ampt, *fazt;      /* (nobn,12) OB tidal amplitude / phase    */
    const double *amp_factor, *phy_factor; /* (12)                             */
    /* key_atm only (what sbc_do leaves in o_ARRAYS, src/fv_main.F90:419);
     * before the first one the library holds mslp = P_ref = 101325 Pa
     * (src/fv_main.F90:1006) and zero emp, qsr, qns (:1050-1053)         */
    const double *mslp;             /* (nod2D) sea-level pressure, Pa          */
    const double *emp;              /* (nod2D) evaporation - precipitation     */
    const double *qsr;              /* (nod2D) downward shortwave, W/m^2       */
    const double *qns;              /* (nod2D) downward non-solar heat, W/m^2  */
    const double *Rj, *aj, *bj;     /* (nod2D) Jerlov water type per node (jer_const = 0) */
} fesomc_forcing;

/* Opaque model instance. */
typedef struct fesomc_model fesomc_model;

/* ---- drop-in entry points -------------------------------------------------
 * fesomc_gpu_init replaces: array_setup .. initial_state state as left at
 *   src/fv_main.F90:157-362 (jacobian is recomputed on the device).
 * fesomc_gpu_set_forcing replaces: the module-array writes of rivers_do,
 *   sbc_do and obc_do (src/fv_main.F90:412-431).
 * fesomc_gpu_step replaces: oce_timestep, case(3) (src/fv_main.F90:1983-2095)
 *   together with the time update at src/fv_main.F90:400-401.
 * fesomc_gpu_sync_to_host / _from_host: before ncoutput(mpi)_do, energy and
 *   write_restart_separate / after read_restart_separate.
 * fesomc_gpu_energy replaces: energy(eout) (src/fv_average_dynamic.F90:476-554).
 * fesomc_gpu_init accepts 5 <= nsigma <= 127 (per-column scratch of the
 * vertical solvers is held in shared memory) and returns FESOMC_EINVAL
 * otherwise.
 */
int  fesomc_gpu_init(const fesomc_mesh *mesh, const fesomc_params *par,
                     const fesomc_state *state, fesomc_model **out);
int  fesomc_gpu_set_forcing(fesomc_model *m, const fesomc_forcing *f);
/* Forcing on the device, replacing the per-step host side of rivers_do
 * (src/fv_rivers.F90:263-299) and of the harmonic open-boundary elevation
 * of compute_ssh_rhs_elem (src/fv_average_dynamic.F90:190-216).  After this
 * call every internal step advances a device copy of time_jd (the main
 * loop's time_jd + dt/86400, src/fv_main.F90:400) and evaluates on the
 * device, with the same arithmetic as the host path, the open-boundary
 * elevation of its Mt sub-steps (from the ampt / fazt / amp_factor /
 * phy_factor last given to fesomc_gpu_set_forcing; later calls that change
 * them are picked up) and the river runoff: runoff_base (n_rivers values,
 * required when rivers are on), scaled by (time_jd - time_jd0)/10 during
 * the first 10 days when river_ramp != 0.  Steps then copy nothing from
 * the host; runoff given to fesomc_gpu_set_forcing is ignored.  The mode
 * stays on for the life of the model.  Returns FESOMC_EINVAL when rivers
 * are on and runoff_base is NULL. */
int  fesomc_gpu_set_device_forcing(fesomc_model *m, const double *runoff_base, int32_t river_ramp);
int  fesomc_gpu_step(fesomc_model *m, int32_t n_dt);
int  fesomc_gpu_run(fesomc_model *m, int32_t n_dt0, int32_t nsteps);
int  fesomc_gpu_sync_to_host(fesomc_model *m, uint32_t field_mask, fesomc_state *state);
/* Asynchronous output, the non-blocking counterpart of fesomc_gpu_sync_to_host
 * for the output and restart writers (ncoutput(mpi)_do,
 * src/fv_ncoutputmpi.F90:1164; write_restart_separate, src/fv_restart.F90:399):
 * _begin takes a device-side copy of the masked fields after every step
 * enqueued so far and starts copying it, on a second stream, into the
 * non-NULL arrays of state (FP64, reference layout), then returns; the
 * caller may keep stepping while the copy runs, and must not read or free
 * those arrays before _end.  _end waits for the copy, converts the FP32
 * fields of the FP32 form, and sets state's time_jd and lfirst to the
 * snapshot's.  The destination arrays are page-locked (cudaHostRegister) on
 * their first use and stay so until fesomc_gpu_finalize, so pass the same
 * arrays each time (the driver's module arrays) and keep them allocated
 * until then.  One snapshot at a time: _begin while one is pending, or _end
 * without one, returns FESOMC_ESTATE. */
int  fesomc_gpu_snapshot_begin(fesomc_model *m, uint32_t field_mask, fesomc_state *state);
int  fesomc_gpu_snapshot_end(fesomc_model *m);
int  fesomc_gpu_sync_from_host(fesomc_model *m, uint32_t field_mask, const fesomc_state *state);
int  fesomc_gpu_energy(fesomc_model *m, double *eout);
/* Tracer range of a decomposed mesh: range = {Tmin, Tmax, Smin, Smax} over
 * the whole domain (the min / max of solve_tracers, src/fv_tracer.F90:18-27,
 * which the reference takes over all ranks), used by the following steps
 * in place of the min / max over this model's own nodes: T_aver and S_aver
 * are formed from it as from the model's own.  Give it before every step
 * (the ranks' tracers change); NULL goes back to the model's own min / max.
 * FESOMC_EINVAL for packed members or a range with min > max or NaN.  No
 * counterpart in the reference (one MPI reduction there). */
int  fesomc_gpu_set_tracer_range(fesomc_model *m, const double *range);
/* sbc_do on the device (src/fv_sbc.F90:1012-1046 with data_timeinterp,
 * :838-868, and apply_atm_fluxes, :368-482, with the Large & Yeager (2004)
 * transfer coefficients of core_coeff_2z, :484-662): from the coefficients
 * that getcoeffld computes from the forcing files (coef_a, coef_b: 8 per
 * node in the reference layout coef(i_totfl, nod2D): x / y wind at 10 m,
 * specific humidity, shortwave, longwave, 2 m air temperature,
 * precipitation, sea-level pressure), every following step forms the fields
 * at its time_jd (now_date * coef_a + coef_b), the winds, the wind stress
 * against the surface current (per node, then per element with w_cv), the
 * non-solar heat flux (longwave less emission when net_flux == 0, as
 * nm_net_flux), E - P (precipitation divided by prec_coef, nm_prec_coef),
 * the shortwave and the sea-level pressure, before the step, as the
 * reference's main loop calls sbc_do before oce_timestep; fesomc_gpu_
 * set_forcing then leaves those fields alone.  Call again whenever
 * getcoeffld gives new coefficients.  type_task 3 without sea ice.
 * FESOMC_EINVAL without key_atm, in the FP32 form or for prec_coef 0. */
int  fesomc_gpu_set_atm_fields(fesomc_model *m, const double *coef_a, const double *coef_b, int32_t net_flux,
                               double prec_coef);
/* Halo exchange of a decomposed mesh on the device (the packed form of
 * exchange_nod / exchange_elem, src/gen_halo_exchange_c.F90:130-165,663-793,
 * for every field of the restart set at once).  A plan lists nodes and
 * elements of this model (0-based, reference numbering, host arrays);
 * _size gives the doubles of its buffer; _pack gathers the state of the
 * listed entities (the fesomc_state fields in declaration order, each
 * entity's values consecutive, FP32 fields widened) into a device buffer,
 * _unpack writes such a buffer back (and, as a full upload does, the
 * jacobian state from the elevation); both return when the device is done.
 * _range gives {Tmin, Tmax, Smin, Smax} over the plan's nodes (a rank's own
 * nodes: its part of the range fesomc_gpu_set_tracer_range takes).  Plans
 * belong to the model they were made for; free them before it. */
typedef struct fesomc_halo fesomc_halo;
int  fesomc_gpu_halo_plan(fesomc_model *m, int32_t n_nodes, const int32_t *nodes, int32_t n_elems,
                          const int32_t *elems, fesomc_halo **plan);
int  fesomc_gpu_halo_size(const fesomc_halo *plan, int64_t *count);
int  fesomc_gpu_halo_pack(fesomc_model *m, const fesomc_halo *plan, double *dev_buf);
int  fesomc_gpu_halo_unpack(fesomc_model *m, const fesomc_halo *plan, const double *dev_buf);
int  fesomc_gpu_halo_range(fesomc_model *m, const fesomc_halo *plan, double *range);
void fesomc_gpu_halo_free(fesomc_halo *plan);
int  fesomc_gpu_last_status(fesomc_model *m, uint32_t *status, int32_t *notconv_columns);
int  fesomc_gpu_finalize(fesomc_model *m);
const char *fesomc_gpu_error_string(int code);

/* ---- host mesh builder ----------------------------------------------------
 * Restates read_mesh_ser (triangles first, coordinate scaling,
 * fv_main.F90:787-945), test_elem (fv_mesh_array.F90:1-82), find_edges
 * (:395-718), find_elem_neighbors (:791-946), mesh_arrays1 (:948-1139),
 * mesh_arrays2 (:1155-1386), find_up_downwind_triangles (:1390-1618) and
 * SET_SIGMA cases 1 and 2 (fv_vert_coord.F90:135-280).  Produces the arrays
 * a fesomc_mesh points to.  Inputs: node coordinates as in nod2d.out
 * (metres if cartesian, degrees otherwise), node flags, and elements as in
 * elem2d.out (4 nodes per row, node4 = node1 for triangles; 1-based).
 */
typedef struct fesomc_mesh_builder fesomc_mesh_builder;

typedef struct fesomc_mesh_opts {
    int32_t cartesian;
    int32_t coriolis_on;          /* Coriolis_TF                              */
    double  lat_cartesian_deg;    /* latitude for cartesian Coriolis          */
    double  cyclic_length_deg;    /* 360 in the reference test case           */
    int32_t nsigma;
    int32_t ind_sigma;            /* 1 or 2                                   */
    double  pow_sig, lev_bot, lev_sur;
    int32_t T_potential;          /* a_tp = (0.918, 0.69) instead of (1, 0)    */
    int32_t with_up_dn_tri;       /* compute edge_up_dn_tri (MUSCL)           */
} fesomc_mesh_opts;

int  fesomc_mesh_build(int32_t nod2D, const double *xy, const int32_t *index_nod2D,
                       int32_t elem2D, const int32_t *elem_nodes4,
                       const double *depth, const fesomc_mesh_opts *opts,
                       fesomc_mesh_builder **out);
/* Fills *mesh with pointers owned by the builder (valid until free). */
int  fesomc_mesh_view(const fesomc_mesh_builder *b, fesomc_mesh *mesh);
/* scale_area = sum(elem_area)/elem2D, sequential sum (fv_ini.F90:81). */
double fesomc_mesh_scale_area(const fesomc_mesh_builder *b);
int  fesomc_mesh_set_rivers(fesomc_mesh_builder *b, int32_t n, const int32_t *nodes);
/* Sponge layer of radius (m) at the open boundary: ac_create
 * (src/fv_utilit.F90:184-220, distance Dist2in1 :53-88), as the reference
 * builds it when SL_obn is set (src/fv_main.F90:224-250). */
int  fesomc_mesh_set_sponge(fesomc_mesh_builder *b, double radius);
void fesomc_mesh_free(fesomc_mesh_builder *b);

/* Jackett-McDougall density anomaly rho(t,s,pz) - density_0 on the host, as
 * initial_state needs it to set density_0 = 1000 + densityJM(T_const, S_const, 0)
 * (src/fv_ini.F90:187-199; densityJM src/fv_pressure_new.F90:340-414). */
double fesomc_host_density_jm(double t, double s, double pz, double density_0);

/* ---- measurement ----------------------------------------------------------
 * fesomc_gpu_time_run: like fesomc_gpu_run, but returns the device time of
 * the nsteps internal steps measured with CUDA events on the library stream.
 * fesomc_gpu_profile: runs nsteps internal steps without the CUDA graph, with
 * an event pair around every kernel, and reports per kernel (names: 32-byte
 * entries) the mean device time per launch, the algorithmic bytes per launch
 * (every array the kernel must touch, counted once) and the launch count.
 * Neither has a counterpart in the reference; they replace its per-routine
 * omp_get_wtime prints (src/fv_main.F90:2084-2095). */
int  fesomc_gpu_time_run(fesomc_model *m, int32_t nsteps, double *ms);
/* fesomc_gpu_d3end_iterations: advances nsteps internal steps (forcing as
 * last set) and returns in iters (nod2D values) the number of sweeps the
 * turbulence closure d3_end needed on each node column in the last of them
 * (200 = not converged), in the device's storage order, i.e. in the order
 * consecutive GPU threads take the columns (32 consecutive values share a
 * warp).  Measurement only; no counterpart in the reference. */
int  fesomc_gpu_d3end_iterations(fesomc_model *m, int32_t nsteps, int32_t *iters);
int  fesomc_gpu_profile(fesomc_model *m, int32_t nsteps, int32_t max_kernels, int32_t *n_kernels,
                        char *names, double *ms_per_launch, double *bytes_per_launch, int64_t *launches);

/* Ensemble: advances n_members independent model instances (meshes of any
 * size, either precision form) by nsteps internal steps each, concurrently
 * on one GPU.  Every member keeps its own stream and its own captured step
 * graph; the call interleaves the members' steps (member order as given,
 * largest first is best), then waits for all.  status[i] (may be NULL)
 * receives member i's step status (FESOMC_OK, FESOMC_ENEGSALT, ...); the
 * return value is the first non-OK member status, or a call error.  With
 * ms != NULL the device time from the first enqueued step to the last
 * finished one is measured with CUDA events (fork / join across the
 * member streams).  Members must live on the current device and must not
 * be used by another thread during the call.  No counterpart in the
 * reference, which runs one mesh per executable. */
int  fesomc_ensemble_run(fesomc_model *const *members, int32_t n_members, int32_t nsteps, double *ms,
                         int32_t *status);

/* Launch shapes.  A knob is the threads per block of one kernel whose
 * results do not depend on the block shape (one thread per entity or per
 * (entity, level), grid-stride, no block-level reduction), or ("columns")
 * the nodes / elements per block of the column kernels; any setting gives
 * the same bits.  fesomc_gpu_tune_knobs returns the number of knobs;
 * fesomc_gpu_tune_knob their names and the fesomc_gpu_profile records that
 * time each (comma-separated; buffers of *_len bytes, NULL to skip).
 * fesomc_gpu_tune_get fills values (the shapes in use) and limits (the
 * largest each knob accepts on this device), either may be NULL.
 * fesomc_gpu_tune_set takes one value per knob (0 = the default) and
 * returns FESOMC_EINVAL, changing nothing, when a thread count is not a
 * multiple of 32 or a value exceeds its limit ("d3end_arrays" takes 1 to 6:
 * d3_end's column arrays in local or in shared memory, or a set-up and a
 * sweep kernel with the sweep's arrays in local memory, in shared memory, or
 * (11 or 21 levels) in registers at 6 or 8 blocks of 64 columns per SM;
 * "vdiff_form" 1 to 3: the tracers' implicit vertical diffusion with each
 * column read directly by its thread, or on tiles of 128 or 64 (the
 * default) columns staged in shared memory, for 10 or 20 layers;
 * "implvisc_form" 1 or 2: the implicit vertical viscosity with each element
 * column read directly, or on tiles of 64 columns staged in shared memory,
 * the default for the fic variant at 10 or 20 layers); the next step
 * captures its
 * graph again.  The search over the knobs and its cache per mesh size and
 * level count live with the host driver (fesomc/autotune.py).  No
 * counterpart in the reference. */
int  fesomc_gpu_tune_knobs(void);
int  fesomc_gpu_tune_knob(int32_t k, char *name, int32_t name_len, char *records, int32_t records_len);
int  fesomc_gpu_tune_get(fesomc_model *m, int32_t *values, int32_t *limits);
int  fesomc_gpu_tune_set(fesomc_model *m, const int32_t *values);

/* Packed members: several meshes advanced as one model, so that every
 * kernel of a step covers all members in one launch.  The caller
 * concatenates the members' fesomc_mesh arrays (indices offset; all
 * members' internal edges first, then all boundary edges), fesomc_state
 * and fesomc_forcing arrays in member order; the members share nsigma,
 * sigma and every fesomc_params field except scale_area, given per member
 * here.  Each member then advances bit for bit as it does alone: the tracer
 * means of solve_tracers (fv_tracer.F90:18-27) and scale_area are taken per
 * member.  No counterpart in the reference, which runs one mesh per
 * executable. */
typedef struct fesomc_members {
    int32_t n;                    /* members                                       */
    const int32_t *node_off;      /* (n+1) first node of each member, 0-based; node_off[n] = nod2D */
    const int32_t *elem_off;      /* (n+1) first element of each member; elem_off[n] = elem2D */
    const double *scale_area;     /* (n) sum(elem_area)/elem2D of each member (fv_ini.F90:81) */
} fesomc_members;

/* fesomc_gpu_init for a packed mesh; members = NULL or n = 1 is one mesh.
 * Returns FESOMC_EINVAL when the ranges do not start at 0, grow strictly and
 * end at nod2D / elem2D, when a scale_area is not positive, or when an
 * element, edge or node-element list reaches into another member. */
int  fesomc_gpu_init_packed(const fesomc_mesh *mesh, const fesomc_params *par, const fesomc_state *st,
                            const fesomc_members *members, fesomc_model **out);

/* Selects the CUDA device used by subsequent fesomc_gpu_init calls of the
 * calling thread (one process per GPU).  No counterpart in the reference,
 * where each MPI rank owns a mesh partition instead. */
int  fesomc_gpu_set_device(int32_t device);

/* No counterpart in the reference.  The domain energy (the same quantity
 * fesomc_gpu_energy returns) of a state held in caller-owned DEVICE arrays,
 * without creating a model and without allocating device memory.  It serves
 * callers that own the state in their own device buffers (another
 * framework's memory pool, whose allocator they must not bypass) or that
 * have reserved all device memory up front and may not allocate more.  Arrays use the
 * reference shapes: eta_n, depth, area (nod2D); elem2D_nodes (4,elem2D),
 * 1-based; w_cv (4,elem2D); U_n_2D (2,elem2D); elem_area (elem2D).  stream
 * is a cudaStream_t (NULL = default stream); the call returns after the
 * result is on the host.  The reduction scratch is a fixed 14,232-byte
 * device array shared by all calls on a device: it needs no initial zeroing,
 * and calls that overlap in time race on it.  The first call on a device
 * (with that device current) looks up the array once and keeps its address
 * for the life of the process; make it before any stream capture begins,
 * and do not call it again on a device after cudaDeviceReset there.
 * Returns FESOMC_EINVAL for bad arguments (counts below 1, NULL arrays). */
int  fesomc_energy_device(int32_t nod2D, int32_t elem2D, double Dmin, const double *eta_n,
                          const double *depth, const double *area, const int32_t *elem2D_nodes,
                          const double *w_cv, const double *U_n_2D, const double *elem_area,
                          void *stream, double *eout);

/* ---- learned vertical-mixing closure ----------------------------------------
 * No counterpart in the reference.  A per-column network stands in for the
 * turbulence closure d3_end (src/fv_mixing.F90:73-347): inputs per node
 * column are, at the nsigma interfaces, the squared shear, the buoyancy
 * frequency squared and the interface depth, plus the surface TKE flux term,
 * the bottom TKE value and the total depth (3*nsigma + 3 values; shear, N^2
 * and the boundary terms through asinh(x/1e-6), then normalised by the
 * training set); three hidden layers of 256 with SiLU; outputs log bt, the
 * turbulence energy d3_end advances, at the interfaces (nsigma, normalised).
 * It is trained on the GPU, on columns harvested from the plain closure, by
 * FP32 forward / backward / Adam kernels.  In the time step
 * (fesomc_closure_attach) a wet column whose inputs lie inside the training
 * envelope takes the network's bt, held to the range of the training
 * targets, and snu and Kv formed from it as d3_end forms them (snu =
 * scale_t sqrt(bt) + snul, at most 0.2; Kv = Pr_num snu); dry columns and
 * columns outside the envelope take the plain closure; every judge_every-th
 * step the plain closure runs on all columns and the network's viscosity is
 * compared with it.
 *
 * _create: nsigma 5..32, room for 'capacity' harvested columns.
 * _harvest: advances the model nsteps internal steps (forcing as last set,
 *   like fesomc_gpu_run) with the plain closure, appending the wet columns of
 *   every 'every'-th step to the training set.
 * _fit: normalisation and envelope (per-input min / max) of the training set.
 * _train: epochs of Adam over the training set in minibatches of 'batch'
 *   (<= 8192); losses (may be NULL) receives the mean loss per epoch.
 * _params / _norm: copy the parameters (W1 b1 W2 b2 W3 b3 W4 b4, W row-major
 *   out x in) / the statistics (8 arrays of max(in, out) floats: input mean,
 *   input sd, output mean, output sd, envelope low, envelope high of the
 *   normalised inputs, lowest and highest training target) out of (get) and
 *   into (set) the closure.
 * _forward / _grad: the network on host arrays of normalised inputs (tests),
 *   _forward with bf16 = 1 on the tensor cores (BF16 weights and
 *   activations, FP32 accumulation; nsigma <= 32), else in FP32;
 *   _grad takes n <= 8192 samples and returns the mean squared error and its
 *   gradient in the parameter layout.
 * _attach: the model's steps use the closure (NULL: the plain closure
 *   again), its inference on the tensor cores when bf16 = 1 (else FP32);
 *   judge_every 0 never judges.  _stats: counts since attach.             */
typedef struct fesomc_closure fesomc_closure;
typedef struct fesomc_closure_report {
    int64_t steps, judge_steps;       /* steps since attach, of which judge steps */
    int64_t wet_columns;              /* wet column-steps seen                   */
    int64_t out_of_envelope;          /* wet column-steps given to the plain closure */
    int64_t dry_columns;              /* dry column-steps (plain closure)        */
    int64_t judge_values;             /* interface values compared by the judge  */
    double judge_rms_log, judge_max_log; /* network vs plain closure, log snu   */
} fesomc_closure_report;
int  fesomc_closure_create(int32_t nsigma, int64_t capacity, uint64_t seed, fesomc_closure **out);
void fesomc_closure_free(fesomc_closure *c);
int  fesomc_closure_info(const fesomc_closure *c, int64_t *harvested, int64_t *nparams, int32_t *n_in,
                         int32_t *n_out);
int  fesomc_closure_harvest(fesomc_closure *c, fesomc_model *m, int32_t nsteps, int32_t every);
int  fesomc_closure_fit(fesomc_closure *c);
int  fesomc_closure_train(fesomc_closure *c, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                          float *losses);
int  fesomc_closure_params(fesomc_closure *c, float *get, const float *set);
int  fesomc_closure_norm(fesomc_closure *c, float *get, const float *set);
int  fesomc_closure_forward(fesomc_closure *c, const float *X, int64_t n, float *Y, int32_t bf16);
int  fesomc_closure_grad(fesomc_closure *c, const float *X, const float *T, int32_t n, double *loss,
                         float *grads);
int  fesomc_closure_attach(fesomc_model *m, fesomc_closure *c, int32_t judge_every, int32_t bf16);
/* measurement: the network on n device-resident pseudo-random columns,
 * reps times after one warm-up, *ms = mean device time per pass (CUDA
 * events); bf16 selects the tensor-core kernel. */
int  fesomc_closure_time(fesomc_closure *c, int64_t n, int32_t reps, int32_t bf16, double *ms);
int  fesomc_closure_stats(fesomc_model *m, fesomc_closure_report *r);
/* fesomc_closure_set_rules: fallback rules the model applies, beyond the
 * training envelope, with this network from the next fesomc_closure_attach
 * on.  FESOMC_LC_RULE_UNSTABLE (1): a column with N^2 < 0 at an interior
 * interface (statically unstable, convecting) goes to the plain closure;
 * FESOMC_LC_RULE_BOUNDARY (2): a column at a solid or open boundary node
 * (index_nod2D != 0) goes to the plain closure.  Such columns are counted
 * as out of the envelope.  Other bits: FESOMC_EINVAL. */
#define FESOMC_LC_RULE_UNSTABLE 1
#define FESOMC_LC_RULE_BOUNDARY 2
int  fesomc_closure_set_rules(fesomc_closure *c, int32_t rules);

/* ---- version / introspection --------------------------------------------- */
const char *fesomc_gpu_version(void);
/* Number of kernels launched by this instance since init. */
int64_t fesomc_gpu_kernel_launches(fesomc_model *m);

#ifdef __cplusplus
}
#endif
#endif /* FESOMC_GPU_H */
