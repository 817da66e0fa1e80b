// Tracer kernels of solve_tracers (src/fv_main.F90:1707-1836):
//   minmax      : global T/S min/max -> T_aver, S_aver (two-pass reduction)
//   miura_*     : solve_tracer_miura (fv_tracer.F90:930-1316), T only
//   upwind_h    : solve_tracer_upwind (fv_tracer.F90:390-923) per (node, level):
//                 edge fluxes gathered in edge order, QUICK vertical fluxes,
//                 open-boundary relaxation, AB2 update (T and S together)
//   muscl_*     : solve_tracer_muscl (fv_tracer.F90:8-379) for T and S:
//                 element gradients, node-averaged gradients
//                 (fill_up_dn_grad fallback), segment fluxes per (edge,
//                 level), node gather in edge order + vertical + update
//   vdiff_col   : river salinity source + tracer_impl_vert_diff
//                 (fv_tracer.F90:1319-1494) per node column, with the
//                 negative-salinity / low-temperature checks as status bits
//   energy      : energy diagnostic (fv_average_dynamic.F90:476-554),
//                 compensated deterministic two-pass reduction
#include "device_common.cuh"
#include "fesomc_exp.h"
#include "fesomc_atan.h"

FESOMC_PREC_BEGIN

constexpr int kRedBlock = 256;
constexpr int kRedGrid = 592;  // 4 x 148 SMs

// ---------------------------------------------------------------------------
// global min / max of TF and SF
// ---------------------------------------------------------------------------
// One partial per (block, member): blockIdx.y is the member, whose nodes
// are member_node_off[m] .. member_node_off[m+1] (all nodes for one member).
__global__ void k_minmax_part(Dev d) {
    __shared__ real s[4][kRedBlock];
    const int mb = blockIdx.y;
    const long long n0 = d.member_node_off ? d.member_node_off[mb] : 0;
    const long long n1 = d.member_node_off ? d.member_node_off[mb + 1] : d.N;
    const long long first = n0 * d.L, total = (n1 - n0) * d.L;
    real tmin = d.TF[first], tmax = d.TF[first], smin = d.SF[first], smax = d.SF[first];
    GRID_LOOP(j, total) {
        const long long i = first + j;
        const real t = d.TF[i], x = d.SF[i];
        tmin = dmin(tmin, t); tmax = dmax(tmax, t);
        smin = dmin(smin, x); smax = dmax(smax, x);
    }
    s[0][threadIdx.x] = tmin; s[1][threadIdx.x] = tmax; s[2][threadIdx.x] = smin; s[3][threadIdx.x] = smax;
    __syncthreads();
    for (int o = kRedBlock / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s[0][threadIdx.x] = dmin(s[0][threadIdx.x], s[0][threadIdx.x + o]);
            s[1][threadIdx.x] = dmax(s[1][threadIdx.x], s[1][threadIdx.x + o]);
            s[2][threadIdx.x] = dmin(s[2][threadIdx.x], s[2][threadIdx.x + o]);
            s[3][threadIdx.x] = dmax(s[3][threadIdx.x], s[3][threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) d.mm_part[((size_t)mb * gridDim.x + blockIdx.x) * 4 + k] = s[k][0];
}

// one warp per member; min / max are exact, so the order in which the
// partials are combined does not change the result
__global__ void k_minmax_final(Dev d, int nparts) {
    const int lane = threadIdx.x & 31;
    const real *part = d.mm_part + (size_t)blockIdx.x * nparts * 4;
    real tmin = part[0], tmax = part[1], smin = part[2], smax = part[3];
    for (int b = lane; b < nparts; b += 32) {
        tmin = dmin(tmin, part[4 * b + 0]);
        tmax = dmax(tmax, part[4 * b + 1]);
        smin = dmin(smin, part[4 * b + 2]);
        smax = dmax(smax, part[4 * b + 3]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        tmin = dmin(tmin, __shfl_xor_sync(kFull, tmin, o));
        tmax = dmax(tmax, __shfl_xor_sync(kFull, tmax, o));
        smin = dmin(smin, __shfl_xor_sync(kFull, smin, o));
        smax = dmax(smax, __shfl_xor_sync(kFull, smax, o));
    }
    if (lane == 0) {
        d.aver[2 * blockIdx.x] = real(0.5) * (tmin + tmax);
        d.aver[2 * blockIdx.x + 1] = real(0.5) * (smin + smax);
    }
}

// AB2 value of a tracer at (node, level) minus its mean (fv_tracer.F90:433)
__device__ __forceinline__ real ab2(const Dev &d, const real *Tn, const real *To, size_t i, real aver) {
    return -(real(0.5) + d.epsilon) * To[i] + (real(1.5) + d.epsilon) * Tn[i] - aver;
}

// Vel_nor at node n from its boundary edges (fv_tracer.F90:862-873)
__device__ __forceinline__ real vel_nor(const Dev &d, int n) {
    real v = real(0.0);
    for (int p = d.node_bptr[n]; p < d.node_bptr[n + 1]; ++p) {
        const int code = d.node_bidx[p];
        const int ed = code >> 1;
        const int2 nn = d.edge_nodes[ed];
        const int e1 = d.edge_tri[ed].x;
        const real dmean = dmax<real>(d.Dmin, real(0.5) * (d.eta_n[nn.x] + d.depth[nn.x] + d.eta_n[nn.y] + d.depth[nn.y]));
        const real4 X = d.edge_cross[ed];
        const real un1 = (d.V_filt_2D[e1] * X.x - d.U_filt_2D[e1] * X.y) * dmean;
        if (code & 1) v = v - un1 / d.area[n];
        else v = v + un1 / d.area[n];
    }
    return v;
}

// QUICK vertical flux tvert(k) of solve_tracer_upwind at interface k
// (0-based, 0..NS-1) of node n; TO(m) returns the AB2 tracer of layer m.
template <typename F>
__device__ __forceinline__ real tvert_upwind(const Dev &d, int k, real a, const real *W, F TO) {
    const int NS = d.NS;
    if (k == NS - 1) return real(0.0);
    if (k == 0) return -W[0] * TO(0);
    const int nz = k + 1;  // 1-based
    // Z(m), zbar(m) 1-based
    auto Z = [&](int m) { return z_of(d, a, m - 1); };
    auto ZB = [&](int m) { return zbar_of(d, a, m - 1); };
    auto T = [&](int m) { return TO(m - 1); };
    const real w = W[nz - 1];
    if (nz == 2) {
        if (w > real(0.0)) {
            const real dg = (ZB(2) - Z(1)) * (Z(2) - ZB(2)) / ((Z(3) - Z(1)) * (Z(2) - Z(3)));
            const real db = -(ZB(2) - Z(1)) * (Z(3) - ZB(2)) / ((Z(2) - Z(1)) * (Z(2) - Z(3)));
            return -(T(1) * (real(1.0) - dg - db) + T(2) * db + T(3) * dg) * w;
        }
        return -T(1) * w;
    }
    if (nz <= NS - 2) {
        if (w >= real(0.0)) {
            const real dg = (ZB(nz) - Z(nz - 1)) * (Z(nz) - ZB(nz)) / ((Z(nz + 1) - Z(nz - 1)) * (Z(nz) - Z(nz + 1)));
            const real db = -(ZB(nz) - Z(nz - 1)) * (Z(nz + 1) - ZB(nz)) / ((Z(nz) - Z(nz - 1)) * (Z(nz) - Z(nz + 1)));
            return -(T(nz - 1) * (real(1.0) - dg - db) + T(nz) * db + T(nz + 1) * dg) * w;
        }
        const real dg = (Z(nz) - ZB(nz)) * (ZB(nz) - Z(nz - 1)) / ((Z(nz) - Z(nz - 2)) * (Z(nz - 2) - Z(nz - 1)));
        const real db = -(Z(nz) - ZB(nz)) * (ZB(nz) - Z(nz - 2)) / ((Z(nz) - Z(nz - 1)) * (Z(nz - 2) - Z(nz - 1)));
        return -(T(nz) * (real(1.0) - dg - db) + T(nz - 1) * db + T(nz - 2) * dg) * w;
    }
    // nz == NS-1
    if (w >= real(0.0)) return -T(nz) * w;
    const real dg = (Z(nz) - ZB(nz)) * (ZB(nz) - Z(nz - 1)) / ((Z(nz) - Z(nz - 2)) * (Z(nz - 2) - Z(nz - 1)));
    const real db = -(Z(nz) - ZB(nz)) * (ZB(nz) - Z(nz - 2)) / ((Z(nz) - Z(nz - 1)) * (Z(nz - 2) - Z(nz - 1)));
    return -(T(nz) * (real(1.0) - dg - db) + T(nz - 1) * db + T(nz - 2) * dg) * w;
}

// tvert_upwind of T and S of the same column: the interface weights, the
// same for both tracers, are formed once (same expressions, same bits)
template <typename F, typename G>
__device__ __forceinline__ void tvert_upwind2(const Dev &d, int k, real a, const real *W, F TO, G SO, real &tv,
                                              real &sv) {
    const int NS = d.NS;
    if (k == NS - 1) { tv = real(0.0); sv = real(0.0); return; }
    if (k == 0) { tv = -W[0] * TO(0); sv = -W[0] * SO(0); return; }
    const int nz = k + 1;  // 1-based
    auto Z = [&](int m) { return z_of(d, a, m - 1); };
    auto ZB = [&](int m) { return zbar_of(d, a, m - 1); };
    const real w = W[nz - 1];
    // a quadratic over layers m0, m1, m2 (1-based) with weights 1-dg-db, db,
    // dg, or the single layer m0
    int m0, m1 = 0, m2 = 0;
    real dg = real(0.0), db = real(0.0);
    bool quad = true;
    if (nz == 2) {
        if (w > real(0.0)) {
            dg = (ZB(2) - Z(1)) * (Z(2) - ZB(2)) / ((Z(3) - Z(1)) * (Z(2) - Z(3)));
            db = -(ZB(2) - Z(1)) * (Z(3) - ZB(2)) / ((Z(2) - Z(1)) * (Z(2) - Z(3)));
            m0 = 1; m1 = 2; m2 = 3;
        } else {
            m0 = 1; quad = false;
        }
    } else if (nz <= NS - 2 && w >= real(0.0)) {
        dg = (ZB(nz) - Z(nz - 1)) * (Z(nz) - ZB(nz)) / ((Z(nz + 1) - Z(nz - 1)) * (Z(nz) - Z(nz + 1)));
        db = -(ZB(nz) - Z(nz - 1)) * (Z(nz + 1) - ZB(nz)) / ((Z(nz) - Z(nz - 1)) * (Z(nz) - Z(nz + 1)));
        m0 = nz - 1; m1 = nz; m2 = nz + 1;
    } else if (nz == NS - 1 && w >= real(0.0)) {
        m0 = nz; quad = false;
    } else {
        dg = (Z(nz) - ZB(nz)) * (ZB(nz) - Z(nz - 1)) / ((Z(nz) - Z(nz - 2)) * (Z(nz - 2) - Z(nz - 1)));
        db = -(Z(nz) - ZB(nz)) * (ZB(nz) - Z(nz - 2)) / ((Z(nz) - Z(nz - 1)) * (Z(nz - 2) - Z(nz - 1)));
        m0 = nz; m1 = nz - 1; m2 = nz - 2;
    }
    if (quad) {
        tv = -(TO(m0 - 1) * (real(1.0) - dg - db) + TO(m1 - 1) * db + TO(m2 - 1) * dg) * w;
        sv = -(SO(m0 - 1) * (real(1.0) - dg - db) + SO(m1 - 1) * db + SO(m2 - 1) * dg) * w;
    } else {
        tv = -TO(m0 - 1) * w;
        sv = -SO(m0 - 1) * w;
    }
}

// AB2 tracers of this step minus their means, stored once per (node, level)
// for the gathers below (fv_tracer.F90:433,435 and :39-47)
__global__ void k_ab2_node(Dev d) {
    const long long total = (long long)d.N * d.L;
    GRID_LOOP(i, total) {
        const int n = (int)(i / d.L);
        d.ttfold[i] = ab2(d, d.TF, d.T_old, i, t_aver_of(d, n));
        d.stfold[i] = ab2(d, d.SF, d.S_old, i, s_aver_of(d, n));
    }
}

// ---------------------------------------------------------------------------
// solve_tracer_upwind: one thread per (node, level), levels on consecutive
// lanes of a flat index (no lane idles when L < 32); level data coalesced.
// ---------------------------------------------------------------------------
__global__ void k_upwind_h(Dev d) {
    const int lane = threadIdx.x & 31;
    const int L = d.L, NS = d.NS;
    const long long total = (long long)d.N * L;
    // each warp takes 31 (node, level) outputs; lane 31 forms the flux at its
    // own index, the interface below lane 30's layer, for the shuffle, so no
    // lane forms a second flux
    const long long nwarp = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c * 31 < total; c += nwarp) {
        const long long iw = c * 31 + lane;
        const bool valid = lane < 31 && iw < total;
        const long long i_ = iw < total ? iw : total - 1;
        const int n = (int)(i_ / L);
        const int z = (int)(i_ % L), zc = z;
        const real T_aver = t_aver_of(d, n), S_aver = s_aver_of(d, n);
        const real a = jac_a(d, d.eta_jac, n);
        const real *W = d.Wvel + (size_t)n * NS;
        const size_t base = (size_t)n * L;
        const real area_inv = real(1.0) / d.area[n];
        const int p0 = d.node_eptr[n], p1 = d.node_eptr[n + 1];
        {
            real acc_t = real(0.0), acc_s = real(0.0), acc_c = real(0.0);
            for (int p = p0; p < p1; ++p) {
                const int code = d.node_eidx[p];
                const int ed = code >> 1;
                const int2 nn = d.edge_nodes[ed];
                const int2 et = d.edge_tri[ed];
                const real4 X = d.edge_cross[ed];
                const size_t i1 = (size_t)nn.x * L + zc, i2 = (size_t)nn.y * L + zc;
                const real t1 = d.ttfold[i1], t2 = d.ttfold[i2];
                const real s1 = d.stfold[i1], s2 = d.stfold[i2];
                const size_t e1 = (size_t)et.x * L + zc;
                const real J1 = d.Je[e1];
                const real c1 = d.V_n_filt[e1] * X.x - d.U_n_filt[e1] * X.y;
                real aux_c, t_aux, s_aux;
                if (ed < d.Ed_in) {
                    const size_t e2 = (size_t)et.y * L + zc;
                    const real J2 = d.Je[e2];
                    const real c2 = -d.V_n_filt[e2] * X.z + d.U_n_filt[e2] * X.w;
                    aux_c = J1 * c1 + J2 * c2;
                    if (c1 > real(0.0) && c2 > real(0.0)) {
                        t_aux = J1 * c1 * t2 + J2 * c2 * t2;
                        s_aux = J1 * c1 * s2 + J2 * c2 * s2;
                    } else if (c1 > real(0.0)) {
                        t_aux = J1 * c1 * t2 + J2 * c2 * t1;
                        s_aux = J1 * c1 * s2 + J2 * c2 * s1;
                    } else if (c2 > real(0.0)) {
                        t_aux = J1 * c1 * t1 + J2 * c2 * t2;
                        s_aux = J1 * c1 * s1 + J2 * c2 * s2;
                    } else {
                        t_aux = J1 * c1 * t1 + J2 * c2 * t1;
                        s_aux = J1 * c1 * s1 + J2 * c2 * s1;
                    }
                } else {
                    aux_c = J1 * c1;
                    if (c1 > real(0.0)) { t_aux = aux_c * t2; s_aux = aux_c * s2; }
                    else { t_aux = aux_c * t1; s_aux = aux_c * s1; }
                }
                if (code & 1) { acc_c = acc_c - aux_c; acc_t = acc_t - t_aux; acc_s = acc_s - s_aux; }
                else { acc_c = acc_c + aux_c; acc_t = acc_t + t_aux; acc_s = acc_s + s_aux; }
            }
            auto TO = [&](int m) { return d.ttfold[base + m]; };
            auto SO = [&](int m) { return d.stfold[base + m]; };
            real tv0, sv0;
            tvert_upwind2(d, zc, a, W, TO, SO, tv0, sv0);
            real tv1 = __shfl_down_sync(kFull, tv0, 1), sv1 = __shfl_down_sync(kFull, sv0, 1);
            if (zc == L - 1) { tv1 = real(0.0); sv1 = real(0.0); }   // the bottom interface carries no flux
            if (valid) {
                const bool relax = d.cl_relax && d.index_nod2D[n] == 2;
                const size_t ii = base + z;
                const real to = d.ttfold[ii], so = d.stfold[ii];
                const real jc = jc_of(d, a, z);
                real tr = ((acc_t - to * acc_c) * area_inv + to * (W[z] - W[z + 1]) + (tv0 - tv1)) / jc;
                real sr = ((acc_s - so * acc_c) * area_inv + so * (W[z] - W[z + 1]) + (sv0 - sv1)) / jc;
                if (relax) {
                    if (vel_nor(d, n) > real(0.0)) {
                        tr = tr + d.relax2clim_ac * (d.Tclim[ii] - (to + T_aver));
                        sr = sr + d.relax2clim_ac * (d.Sclim[ii] - (so + S_aver));
                    } else {
                        tr = d.clim_relax * (d.Tclim[ii] - (to + T_aver));
                        sr = d.clim_relax * (d.Sclim[ii] - (so + S_aver));
                    }
                }
                const real ttf = d.TF[ii] - T_aver, stf = d.SF[ii] - S_aver;
                d.Told_new[ii] = ttf + T_aver;
                d.TF_adv[ii] = ttf + tr * d.dt + T_aver;
                d.Sold_new[ii] = stf + S_aver;
                d.SF_adv[ii] = stf + sr * d.dt + S_aver;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// MUSCL (fv_tracer.F90:8-379) for T and S
// ---------------------------------------------------------------------------
// tracer_gradient_elements of the AB2 tracer, thread per (element, level)
__global__ void k_muscl_egrad(Dev d) {
    const long long total = (long long)d.E * d.L;
    GRID_LOOP(ii, total) {
        const int e = (int)(ii / d.L);
        const int z = (int)(ii % d.L);
        const int L = d.L;
        const int4 en = d.elem_nodes[e];
        const size_t i1 = (size_t)en.x * L + z, i2 = (size_t)en.y * L + z, i3 = (size_t)en.z * L + z,
                     i4 = (size_t)en.w * L + z;
        const real t1 = d.ttfold[i1], t2 = d.ttfold[i2], t3 = d.ttfold[i3], t4 = d.ttfold[i4];
        const real s1 = d.stfold[i1], s2 = d.stfold[i2], s3 = d.stfold[i3], s4 = d.stfold[i4];
        const real4 gx = d.gs_x[e], gy = d.gs_y[e];
        d.ttx[ii] = wsum(gx, t1, t2, t3, t4);
        d.tty[ii] = wsum(gy, t1, t2, t3, t4);
        d.stx[ii] = wsum(gx, s1, s2, s3, s4);
        d.sty[ii] = wsum(gy, s1, s2, s3, s4);
    }
}

// area-weighted node mean of the element gradients (fill_up_dn_grad fallback,
// fv_gradients.F90:292-318: tx/tvol with running sums)
__global__ void k_muscl_ngrad(Dev d) {
    const long long total = (long long)d.N * d.L;
    GRID_LOOP(ii, total) {
        const int n = (int)(ii / d.L);
        const int z = (int)(ii % d.L);
        const int L = d.L;
        real tvol = real(0.0), a = real(0.0), b = real(0.0), c = real(0.0), e4 = real(0.0);
        for (int p = d.node_nptr[n]; p < d.node_nptr[n + 1]; ++p) {
            const int el = d.node_nidx[p];
            const real ar = d.elem_area[el];
            const size_t i = (size_t)el * L + z;
            tvol = tvol + ar;
            a = a + d.ttx[i] * ar;
            b = b + d.tty[i] * ar;
            c = c + d.stx[i] * ar;
            e4 = e4 + d.sty[i] * ar;
        }
        d.tnx[ii] = a / tvol;
        d.tny[ii] = b / tvol;
        d.snx[ii] = c / tvol;
        d.sny[ii] = e4 / tvol;
    }
}

// Vertical QUICK flux shared by solve_tracer_muscl (fv_tracer.F90:225-271)
// and solve_tracer_miura (fv_tracer.F90:1171-1207) at interface k (0-based)
// of a column with tracer TO(m); Tmean carries over interfaces with W == 0
// as in the reference.  MUSCL groups the weights as a*b/(c+a)/(b-c), Miura
// as a*b/((c+a)*(b-c)).
template <bool MUSCL, typename F>
__device__ __forceinline__ real tvert_quick(const Dev &d, int k, real a, const real *W, F TO) {
    const int NS = d.NS;
    if (k == NS - 1) return real(0.0);
    if (k == 0) return -W[0] * TO(0);
    real Tmean = real(0.0);
    // replay interfaces back to the last one with W /= 0 (carried Tmean)
    int start = k + 1;
    while (start > 2 && W[start - 1] == real(0.0)) --start;
    for (int nz = start; nz <= k + 1; ++nz) {
        const real w = W[nz - 1];
        auto Z = [&](int m) { return z_of(d, a, m - 1); };
        auto ZB = [&](int m) { return zbar_of(d, a, m - 1); };
        if (w > real(0.0)) {
            if (nz == NS - 1) Tmean = TO(nz - 1);
            else {
                const real aa = ZB(nz) - Z(nz - 1), bb = Z(nz) - ZB(nz), cc = Z(nz + 1) - ZB(nz);
                const real dg = MUSCL ? aa * bb / (cc + aa) / (bb - cc) : aa * bb / ((cc + aa) * (bb - cc));
                const real db = MUSCL ? -aa * cc / (bb + aa) / (bb - cc) : -aa * cc / ((bb + aa) * (bb - cc));
                const real da = real(1.0) - dg - db;
                Tmean = TO(nz - 2) * da + TO(nz - 1) * db + TO(nz) * dg;
            }
        }
        if (w < real(0.0)) {
            if (nz == 2) Tmean = TO(nz - 2);
            else {
                const real aa = Z(nz) - ZB(nz), bb = ZB(nz) - Z(nz - 1), cc = ZB(nz) - Z(nz - 2);
                const real dg = MUSCL ? aa * bb / (cc + aa) / (bb - cc) : aa * bb / ((cc + aa) * (bb - cc));
                const real db = MUSCL ? -aa * cc / (bb + aa) / (bb - cc) : -aa * cc / ((bb + aa) * (bb - cc));
                const real da = real(1.0) - dg - db;
                Tmean = TO(nz - 1) * da + TO(nz - 2) * db + TO(nz - 3) * dg;
            }
        }
    }
    return -Tmean * W[k];
}

// tvert_quick of T and S of the same column: the weights, the same for both
// tracers, are formed once (same expressions, same bits)
template <bool MUSCL, typename F, typename G>
__device__ __forceinline__ void tvert_quick2(const Dev &d, int k, real a, const real *W, F TO, G SO, real &tv,
                                             real &sv) {
    const int NS = d.NS;
    if (k == NS - 1) { tv = real(0.0); sv = real(0.0); return; }
    if (k == 0) { tv = -W[0] * TO(0); sv = -W[0] * SO(0); return; }
    real Tmean = real(0.0), Smean = real(0.0);
    int start = k + 1;
    while (start > 2 && W[start - 1] == real(0.0)) --start;
    for (int nz = start; nz <= k + 1; ++nz) {
        const real w = W[nz - 1];
        auto Z = [&](int m) { return z_of(d, a, m - 1); };
        auto ZB = [&](int m) { return zbar_of(d, a, m - 1); };
        if (w > real(0.0)) {
            if (nz == NS - 1) {
                Tmean = TO(nz - 1);
                Smean = SO(nz - 1);
            } else {
                const real aa = ZB(nz) - Z(nz - 1), bb = Z(nz) - ZB(nz), cc = Z(nz + 1) - ZB(nz);
                const real dg = MUSCL ? aa * bb / (cc + aa) / (bb - cc) : aa * bb / ((cc + aa) * (bb - cc));
                const real db = MUSCL ? -aa * cc / (bb + aa) / (bb - cc) : -aa * cc / ((bb + aa) * (bb - cc));
                const real da = real(1.0) - dg - db;
                Tmean = TO(nz - 2) * da + TO(nz - 1) * db + TO(nz) * dg;
                Smean = SO(nz - 2) * da + SO(nz - 1) * db + SO(nz) * dg;
            }
        }
        if (w < real(0.0)) {
            if (nz == 2) {
                Tmean = TO(nz - 2);
                Smean = SO(nz - 2);
            } else {
                const real aa = Z(nz) - ZB(nz), bb = ZB(nz) - Z(nz - 1), cc = ZB(nz) - Z(nz - 2);
                const real dg = MUSCL ? aa * bb / (cc + aa) / (bb - cc) : aa * bb / ((cc + aa) * (bb - cc));
                const real db = MUSCL ? -aa * cc / (bb + aa) / (bb - cc) : -aa * cc / ((bb + aa) * (bb - cc));
                const real da = real(1.0) - dg - db;
                Tmean = TO(nz - 1) * da + TO(nz - 2) * db + TO(nz - 3) * dg;
                Smean = SO(nz - 1) * da + SO(nz - 2) * db + SO(nz - 3) * dg;
            }
        }
    }
    tv = -Tmean * W[k];
    sv = -Smean * W[k];
}

__device__ __forceinline__ real muscl_mean(bool upw2, real Tm1, real Tm2) {
    return upw2 ? real(0.15) * Tm2 + real(0.85) * (Tm1 + Tm2) / real(2.0) : real(0.15) * Tm1 + real(0.85) * (Tm1 + Tm2) / real(2.0);
}

// MUSCL segment fluxes of one (edge, level) (fv_tracer.F90:59-170 for T and
// S, :172-209 for the continuity term); thread per (edge, level), levels on
// consecutive threads.  Each flux is computed once here and gathered by both
// end nodes below.  64 registers: 32 resident warps per SM instead of 24
// (17 % faster).
__global__ void __maxnreg__(64) k_muscl_edge(Dev d) {
    const long long total = (long long)d.Ed * d.L;
    const int L = d.L;
    GRID_LOOP(ii, total) {
        const int ed = (int)(ii / L);
        const int z = (int)(ii % L);
        const int2 nn = d.edge_nodes[ed];
        const int2 et = d.edge_tri[ed];
        const int2 ud = d.edge_updn[ed];
        const real4 X = d.edge_cross[ed];
        const real2 exy = d.edge_dxdy[ed];
        const size_t i1 = (size_t)nn.x * L + z, i2 = (size_t)nn.y * L + z;
        const real T1 = d.ttfold[i1], T2 = d.ttfold[i2];
        const real S1 = d.stfold[i1], S2 = d.stfold[i2];
        real g1, g2, g3, g4, h1, h2, h3, h4;
        if (ud.x >= 0 && ud.y >= 0) {
            const size_t u = (size_t)ud.x * L + z, w = (size_t)ud.y * L + z;
            g1 = d.ttx[u]; g2 = d.ttx[w]; g3 = d.tty[u]; g4 = d.tty[w];
            h1 = d.stx[u]; h2 = d.stx[w]; h3 = d.sty[u]; h4 = d.sty[w];
        } else {
            g1 = d.tnx[i1]; g2 = d.tnx[i2]; g3 = d.tny[i1]; g4 = d.tny[i2];
            h1 = d.snx[i1]; h2 = d.snx[i2]; h3 = d.sny[i1]; h4 = d.sny[i2];
        }
        real2 fT, fS, fC;
        {
            const real a = kREarth * d.elem_cos[et.x];
            const size_t e1 = (size_t)et.x * L + z;
            const real J1 = d.Je[e1];
            const real U1 = d.U_n_filt[e1], V1 = d.V_n_filt[e1];
            const bool up1 = V1 * X.x - U1 * X.y > 0;
            const real Tm2 = T2 - (real(2.0) * (T2 - T1) + exy.x * a * g2 + exy.y * kREarth * g4) / real(6.0);
            const real Tm1 = T1 + (real(2.0) * (T2 - T1) + exy.x * a * g1 + exy.y * kREarth * g3) / real(6.0);
            const real Tm = muscl_mean(up1, Tm1, Tm2);
            fT.x = (J1 * V1 * Tm) * X.x - (J1 * U1 * Tm) * X.y;
            const real Sm2 = S2 - (real(2.0) * (S2 - S1) + exy.x * a * h2 + exy.y * kREarth * h4) / real(6.0);
            const real Sm1 = S1 + (real(2.0) * (S2 - S1) + exy.x * a * h1 + exy.y * kREarth * h3) / real(6.0);
            const real Sm = muscl_mean(up1, Sm1, Sm2);
            fS.x = (J1 * V1 * Sm) * X.x - (J1 * U1 * Sm) * X.y;
            fC.x = J1 * V1 * X.x - J1 * U1 * X.y;
        }
        if (et.y >= 0) {
            const real b = kREarth * d.elem_cos[et.y];
            const size_t e2 = (size_t)et.y * L + z;
            const real J2 = d.Je[e2];
            const real U2f = d.U_n_filt[e2], V2f = d.V_n_filt[e2];
            const bool up2 = V2f * X.z - U2f * X.w < 0;
            const real Tm2 = T2 - (real(2.0) * (T2 - T1) + exy.x * b * g2 + exy.y * kREarth * g4) / real(6.0);
            const real Tm1 = T1 + (real(2.0) * (T2 - T1) + exy.x * b * g1 + exy.y * kREarth * g3) / real(6.0);
            const real Tm = muscl_mean(up2, Tm1, Tm2);
            const real Sm2 = S2 - (real(2.0) * (S2 - S1) + exy.x * b * h2 + exy.y * kREarth * h4) / real(6.0);
            const real Sm1 = S1 + (real(2.0) * (S2 - S1) + exy.x * b * h1 + exy.y * kREarth * h3) / real(6.0);
            const real Sm = muscl_mean(up2, Sm1, Sm2);
            // second segment uses U_n / V_n (fv_tracer.F90:158-159)
            const real Un2 = d.U_n[e2], Vn2 = d.V_n[e2];
            fT.y = -(J2 * Vn2 * Tm) * X.z + (J2 * Un2 * Tm) * X.w;
            fS.y = -(J2 * Vn2 * Sm) * X.z + (J2 * Un2 * Sm) * X.w;
            fC.y = -J2 * V2f * X.z + J2 * U2f * X.w;
        } else {
            fT.y = real(0.0); fS.y = real(0.0); fC.y = real(0.0);
        }
        d.mflT[ii] = fT;
        d.mflS[ii] = fS;
        d.mflC[ii] = fC;
    }
}

// node gather of the edge fluxes in edge order + vertical + update, one
// thread per (node, level) with levels on consecutive lanes of a flat index
// (no lane idles when L < 32; a warp may span two or three nodes).  The edge
// loop is unrolled so the flux loads of several edges are in flight
// together; the sums stay in edge order.  The vertical flux at interface
// z+1 comes from the next lane when that lane holds the same node.
__global__ void __launch_bounds__(128, 8) k_muscl_h(Dev d) {
    const long long total = (long long)d.N * d.L;
    const int lane = threadIdx.x & 31;
    const int L = d.L, NS = d.NS;
    // each warp takes 31 (node, level) outputs; lane 31 forms the flux at its
    // own index, the interface below lane 30's layer, for the shuffle, so no
    // lane forms a second flux
    const long long nwarp = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c * 31 < total; c += nwarp) {
        const long long iw = c * 31 + lane;
        const bool valid = lane < 31 && iw < total;
        const long long i_ = iw < total ? iw : total - 1;
        const int n = (int)(i_ / L);
        const int z = (int)(i_ % L);
        const real T_aver = t_aver_of(d, n), S_aver = s_aver_of(d, n);
        const real an = jac_a(d, d.eta_jac, n);
        const real *W = d.Wvel + (size_t)n * NS;
        const size_t base = (size_t)n * L;
        const int p0 = d.node_eptr[n], p1 = d.node_eptr[n + 1];
        real rt = real(0.0), rs = real(0.0), rc = real(0.0);
#pragma unroll 4
        for (int p = p0; p < p1; ++p) {
            const int code = d.node_eidx[p];
            const int ed = code >> 1;
            const size_t i = (size_t)ed * L + z;
            const real2 fT = d.mflT[i], fS = d.mflS[i], fC = d.mflC[i];
            const bool internal = ed < d.Ed_in;
            if (code & 1) {
                rt = rt - fT.x; rs = rs - fS.x; rc = rc - fC.x;
                if (internal) { rt = rt - fT.y; rs = rs - fS.y; rc = rc - fC.y; }
            } else {
                rt = rt + fT.x; rs = rs + fS.x; rc = rc + fC.x;
                if (internal) { rt = rt + fT.y; rs = rs + fS.y; rc = rc + fC.y; }
            }
        }
        auto TO = [&](int m) { return d.ttfold[base + m]; };
        auto SO = [&](int m) { return d.stfold[base + m]; };
        real tv0, sv0;
        tvert_quick2<true>(d, z, an, W, TO, SO, tv0, sv0);
        real tv1 = __shfl_down_sync(kFull, tv0, 1), sv1 = __shfl_down_sync(kFull, sv0, 1);
        if (z == L - 1) { tv1 = real(0.0); sv1 = real(0.0); }   // the bottom interface carries no flux
        if (valid) {
            const bool relax = d.cl_relax && d.index_nod2D[n] == 2;
            const size_t ii = base + z;
            const real jc = jc_of(d, an, z);
            const real aj = d.area[n] * jc;
            const real to = d.ttfold[ii], so = d.stfold[ii];
            real tr = rt / aj - to * rc / aj + to * (W[z] - W[z + 1]) / jc + (tv0 - tv1) / jc;
            real sr = rs / aj - so * rc / aj + so * (W[z] - W[z + 1]) / jc + (sv0 - sv1) / jc;
            const real ttf = d.TF[ii] - T_aver, stf = d.SF[ii] - S_aver;
            if (relax) {
                if (vel_nor(d, n) > real(0.0)) {
                    tr = tr + d.relax2clim_ac * (d.Tclim[ii] - (ttf + T_aver));
                    sr = sr + d.relax2clim_ac * (d.Sclim[ii] - (stf + S_aver));
                } else {
                    tr = d.clim_relax * (d.Tclim[ii] - (ttf + T_aver));
                    sr = d.clim_relax * (d.Sclim[ii] - (stf + S_aver));
                }
            }
            d.Told_new[ii] = ttf + T_aver;
            d.TF_adv[ii] = ttf + tr * d.dt + T_aver;
            d.Sold_new[ii] = stf + S_aver;
            d.SF_adv[ii] = stf + sr * d.dt + S_aver;
        }
    }
}

// ---------------------------------------------------------------------------
// solve_tracer_miura (fv_tracer.F90:930-1316): temperature only, as in the
// reference driver (fv_main.F90:1790-1799); salinity passes through.
// ---------------------------------------------------------------------------
// AB2 of T minus its mean (ttfold), T minus its mean (tnow) and the
// advection-order mask of adv_tracer_mask (fv_main.F90:1309-1335,
// H_advtr_crit = 0.1, H_advtr_min = 0)
__global__ void k_miura_prep(Dev d) {
    const long long total = (long long)d.N * d.L;
    GRID_LOOP(i, total) {
        const real T_aver = t_aver_of(d, (int)(i / d.L));
        d.ttfold[i] = ab2(d, d.TF, d.T_old, i, T_aver);
        d.tnow[i] = d.TF[i] - T_aver;
        if (i % d.L == 0) {
            const int n = (int)(i / d.L);
            const real crit = real(0.1), hmin = real(0.0);
            const real dmean = dmax<real>(d.Dmin, d.depth[n] + d.eta_n[n]);
            real m;
            if (dmean > crit) m = real(1.0);
            else if (dmean < hmin) m = real(0.0);
            else m = (dmean - hmin) / (crit - hmin);
            d.mask_ad[n] = m;
        }
    }
}

// tracer_gradient_elements of T - T_aver (fv_gradients.F90:180-214)
__global__ void k_miura_egrad(Dev d) {
    const long long total = (long long)d.E * d.L;
    GRID_LOOP(ii, total) {
        const int e = (int)(ii / d.L);
        const int z = (int)(ii % d.L);
        const int L = d.L;
        const int4 en = d.elem_nodes[e];
        const real t1 = d.tnow[(size_t)en.x * L + z], t2 = d.tnow[(size_t)en.y * L + z];
        const real t3 = d.tnow[(size_t)en.z * L + z], t4 = d.tnow[(size_t)en.w * L + z];
        d.ttx[ii] = wsum(d.gs_x[e], t1, t2, t3, t4);
        d.tty[ii] = wsum(d.gs_y[e], t1, t2, t3, t4);
    }
}

// tracer_gradient_nodes (fv_gradients.F90:217-260): area-weighted sums
// times the reciprocal of the summed area
__global__ void k_miura_ngrad(Dev d) {
    const long long total = (long long)d.N * d.L;
    GRID_LOOP(ii, total) {
        const int n = (int)(ii / d.L);
        const int z = (int)(ii % d.L);
        const int L = d.L;
        real s = real(0.0);
        for (int p = d.node_nptr[n]; p < d.node_nptr[n + 1]; ++p) s = s + d.elem_area[d.node_nidx[p]];
        const real tvol = real(1.0) / s;
        real tx = real(0.0), ty = real(0.0);
        for (int p = d.node_nptr[n]; p < d.node_nptr[n + 1]; ++p) {
            const int el = d.node_nidx[p];
            const real ar = d.elem_area[el];
            tx = tx + d.ttx[(size_t)el * L + z] * ar;
            ty = ty + d.tty[(size_t)el * L + z] * ar;
        }
        d.tnx[ii] = tx * tvol;
        d.tny[ii] = ty * tvol;
    }
}

// Miura segment fluxes of one (edge, level) (fv_tracer.F90:1010-1140) and the
// continuity terms (:1141-1168); thread per (edge, level)
__global__ void k_miura_edge(Dev d) {
    const long long total = (long long)d.Ed * d.L;
    const int L = d.L;
    const real dt = d.dt;
    GRID_LOOP(ii, total) {
        const int ed = (int)(ii / L);
        const int z = (int)(ii % L);
        const int2 nn = d.edge_nodes[ed];
        const int2 et = d.edge_tri[ed];
        const real4 X = d.edge_cross[ed];
        const real2 exy = d.edge_dxdy[ed];
        const real crt1 = real(0.5) * (d.mask_ad[nn.x] + d.mask_ad[nn.y]);
        const bool two = et.y >= 0;
        const real a = real(1.0), b = real(1.0);
        real Kh = d.elem_area[et.x];
        if (two) Kh = real(0.5) * (Kh + d.elem_area[et.y]);
        Kh = d.K_hor * Kh / scale_area_of(d, et.x);
        const size_t e1 = (size_t)et.x * L + z;
        const size_t i1 = (size_t)nn.x * L + z, i2 = (size_t)nn.y * L + z;
        real Tx, Ty;
        if (two) {
            const size_t e2 = (size_t)et.y * L + z;
            Tx = real(0.5) * Kh * (d.ttx[e1] + d.ttx[e2]);
            Ty = real(0.5) * Kh * (d.tty[e1] + d.tty[e2]);
        } else {
            Tx = Kh * d.ttx[e1];
            Ty = Kh * d.tty[e1];
        }
        const real J1 = d.Je[e1];
        const real U1 = d.U_n_filt[e1], V1 = d.V_n_filt[e1];
        real Tmean;
        if (V1 * X.x - U1 * X.y > 0) {
            // no dt on the V term in this branch (fv_tracer.F90:1057)
            Tmean = d.tnow[i2] + (real(0.5) * (-exy.x * a + X.x - U1 * dt) * d.tnx[i2] +
                                  real(0.5) * (-exy.y * kREarth + X.y - V1) * d.tny[i2]) * crt1;
        } else {
            Tmean = d.tnow[i1] + (real(0.5) * (exy.x * a + X.x - U1 * dt) * d.tnx[i1] +
                                  real(0.5) * (exy.y * kREarth + X.y - V1 * dt) * d.tny[i1]) * crt1;
        }
        real2 fT, fC;
        fT.x = (J1 * V1 * Tmean - Ty) * X.x - (J1 * U1 * Tmean - Tx) * X.y;
        fC.x = J1 * V1 * X.x - J1 * U1 * X.y;
        if (two) {
            const size_t e2 = (size_t)et.y * L + z;
            const real J2 = d.Je[e2];
            const real U2 = d.U_n_filt[e2], V2 = d.V_n_filt[e2];
            if (V2 * X.z - U2 * X.w < 0) {
                Tmean = d.tnow[i2] + (real(0.5) * (-exy.x * b + X.z - U2 * dt) * d.tnx[i2] +
                                      real(0.5) * (-exy.y * kREarth + X.w - V2 * dt) * d.tny[i2]) * crt1;
            } else {
                Tmean = d.tnow[i1] + (real(0.5) * (exy.x * b + X.z - U2 * dt) * d.tnx[i1] +
                                      real(0.5) * (exy.y * kREarth + X.w - V2 * dt) * d.tny[i1]) * crt1;
            }
            fT.y = -(J2 * V2 * Tmean - Ty) * X.z + (J2 * U2 * Tmean - Tx) * X.w;
            fC.y = -J2 * V2 * X.z + J2 * U2 * X.w;
        } else {
            fT.y = real(0.0); fC.y = real(0.0);
        }
        d.mflT[ii] = fT;
        d.mflC[ii] = fC;
    }
}

// node gather of the Miura fluxes in edge order + vertical + update (T),
// salinity passed through; one thread per (node, level), levels on
// consecutive lanes of a flat index
__global__ void __launch_bounds__(128, 8) k_miura_h(Dev d) {
    const int lane = threadIdx.x & 31;
    const int L = d.L, NS = d.NS;
    const long long total = (long long)d.N * L;
    // each warp takes 31 (node, level) outputs; lane 31 forms the flux at its
    // own index, the interface below lane 30's layer, for the shuffle, so no
    // lane forms a second flux
    const long long nwarp = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c * 31 < total; c += nwarp) {
        const long long iw = c * 31 + lane;
        const bool valid = lane < 31 && iw < total;
        const long long i_ = iw < total ? iw : total - 1;
        const int n = (int)(i_ / L);
        const int z = (int)(i_ % L), zc = z;
        const real T_aver = t_aver_of(d, n);
        const real an = jac_a(d, d.eta_jac, n);
        const real *W = d.Wvel + (size_t)n * NS;
        const size_t base = (size_t)n * L;
        const int p0 = d.node_eptr[n], p1 = d.node_eptr[n + 1];
        {
            real rt = real(0.0), rc = real(0.0);
#pragma unroll 4
            for (int p = p0; p < p1; ++p) {
                const int code = d.node_eidx[p];
                const int ed = code >> 1;
                const size_t i = (size_t)ed * L + zc;
                const real2 fT = d.mflT[i], fC = d.mflC[i];
                const bool internal = ed < d.Ed_in;
                if (code & 1) {
                    rt = rt - fT.x; rc = rc - fC.x;
                    if (internal) { rt = rt - fT.y; rc = rc - fC.y; }
                } else {
                    rt = rt + fT.x; rc = rc + fC.x;
                    if (internal) { rt = rt + fT.y; rc = rc + fC.y; }
                }
            }
            auto TN = [&](int m) { return d.tnow[base + m]; };
            const real tv0 = tvert_quick<false>(d, zc, an, W, TN);
            real tv1 = __shfl_down_sync(kFull, tv0, 1);
            if (zc == L - 1) tv1 = real(0.0);   // the bottom interface carries no flux
            if (valid) {
                const bool relax = d.cl_relax && d.index_nod2D[n] == 2;
                const real area = d.area[n];
                const size_t ii = base + z;
                const real jc = jc_of(d, an, z);
                const real to = d.ttfold[ii];
                const real ttf = d.tnow[ii];
                real tr = ((rt - to * rc) / area + to * (W[z] - W[z + 1]) + tv0 - tv1) / jc;
                if (relax) {
                    if (vel_nor(d, n) > real(0.0)) tr = tr + d.relax2clim_ac * (d.Tclim[ii] - (ttf + T_aver));
                    else tr = d.clim_relax * (d.Tclim[ii] - (ttf + T_aver));
                }
                d.Told_new[ii] = ttf + T_aver;
                d.TF_adv[ii] = ttf + tr * d.dt + T_aver;
                d.Sold_new[ii] = d.S_old[ii];
                d.SF_adv[ii] = d.SF[ii];
            }
        }
    }
}

// Tracer after advection and the river source, minus its mean: T(k) / S(k)
// of tracer_impl_vert_diff.  The river source (fv_main.F90:1804-1823) adds
// its terms to S in river-list order.
// S: SF_adv of (n, z); Sn: Sold_new of (n, z), read only at river nodes
__device__ __forceinline__ real vd_salt_of(const Dev &d, int n, int z, real aj, real S, real Sn, real S_aver) {
    if (d.key_rivers) {
        for (int p = d.node_rptr[n]; p < d.node_rptr[n + 1]; ++p) {
            const real r = d.runoff[d.node_ridx[p]];
            const real coeff = r * __ldg(d.dsig + z) * d.dt / (d.area[n] * jc_of(d, aj, z));
            const real delta = (d.river_salinity - Sn);
            S = S + delta * coeff;
        }
    }
    return S - S_aver;
}
__device__ __forceinline__ real vd_salt(const Dev &d, int n, size_t base, int z, real aj, real S_aver) {
    const bool river = d.key_rivers && d.node_rptr[n] < d.node_rptr[n + 1];
    return vd_salt_of(d, n, z, aj, d.SF_adv[base + z], river ? d.Sold_new[base + z] : real(0.0), S_aver);
}

// Tridiagonal coefficients a(k), b(k), c(k) of layer k (0-based) of node
// column n (fv_tracer.F90:1380-1420).
__device__ __forceinline__ void vd_coef(const Dev &d, const real *Kv, real aj, int k, real &a, real &b,
                                        real &c) {
    const int L = d.L, NS = d.NS;
    const real dt = d.dt;
    auto Zc = [&](int m) { return z_of(d, aj, m); };
    auto ZBc = [&](int m) { return zbar_of(d, aj, m); };
    if (k == 0) {
        c = -dt * Kv[1] / ((Zc(0) - Zc(1)) * (ZBc(0) - ZBc(1)));
        a = real(0.0);
        b = -c + real(1.0);
    } else if (k == L - 1) {
        a = -dt * Kv[L - 1] / ((Zc(L - 2) - Zc(L - 1)) * (ZBc(L - 1) - ZBc(NS - 1)));
        b = -a + real(1.0);
        c = real(0.0);
    } else {
        a = -dt * Kv[k] / ((Zc(k - 1) - Zc(k)) * (ZBc(k) - ZBc(k + 1)));
        c = -dt * Kv[k] / ((Zc(k) - Zc(k + 1)) * (ZBc(k) - ZBc(k + 1)));
        b = -a - c + real(1.0);
    }
}

// rivers + tracer_impl_vert_diff (fv_tracer.F90:1319-1494), one thread per
// node column.  The sweep coefficients live in shared memory
// ([array][level][thread]); T and S are re-read instead of stored.
constexpr int kVdBlock = 128;
// ---- atmospheric forcing of the column solve (key_atm) -------------------
// sw_cp (fv_tracer.F90:1775-1908): heat capacity of sea water, UNESCO 1983
// polynomial; literals without _WP in the Fortran are REAL(4) (R4).
__device__ real sw_cp(real S, real Ti, real Pr) {
    const real T = (Ti < real(0.0)) ? real(0.0) : Ti;
    real S0, sS;
    if (S < real(0.0)) { S0 = real(0.0); sS = real(0.0); }
    else { S0 = S; sS = S * sqrt(S); }
    const real P = Pr;
    const real T68 = T * real(1.00024);
    real c0 = real(4217.4), c1 = real(-3.720283), c2 = real(0.1412855), c3 = -R4(2.654387e-3), c4 = R4(2.093236e-5);
    real a0 = real(-7.64357), a1 = real(0.1072763), a2 = -R4(1.38385e-3);
    real b0 = real(0.1770383), b1 = -R4(4.07718e-3), b2 = R4(5.148e-5);
    const real Cpst0 = (((c4 * T68 + c3) * T68 + c2) * T68 + c1) * T68 + c0 + (a0 + a1 * T68 + a2 * (T68 * T68)) * S0 +
                       (b0 + b1 * T68 + b2 * (T68 * T68)) * sS;
    a0 = -R4(4.9592e-1); a1 = R4(1.45747e-2); a2 = -R4(3.13885e-4);
    const real a3 = R4(2.0357e-6), a4 = R4(1.7168e-8);
    b0 = R4(2.4931e-4); b1 = -R4(1.08645e-5); b2 = R4(2.87533e-7);
    const real b3 = -R4(4.0027e-9), b4 = R4(2.2956e-11);
    c0 = -R4(5.422e-8); c1 = R4(2.6380e-9); c2 = -R4(6.5637e-11); c3 = R4(6.136e-13);
    const real del_Cp0t0 = (((((c3 * T68 + c2) * T68 + c1) * T68 + c0) * P +
                             ((((b4 * T68 + b3) * T68 + b2) * T68 + b1) * T68 + b0)) * P +
                            ((((a4 * T68 + a3) * T68 + a2) * T68 + a1) * T68 + a0)) * P;
    const real d0 = R4(4.9247e-3), d1 = -R4(1.28315e-4), d2 = R4(9.802e-7), d3 = R4(2.5941e-8), d4 = -R4(2.9179e-10);
    const real e0 = -R4(1.2331e-4), e1 = -R4(1.517e-6), e2 = R4(3.122e-8);
    const real f0 = -R4(2.9558e-6), f1 = R4(1.17054e-7), f2 = -R4(2.3905e-9), f3 = R4(1.8448e-11);
    const real g0 = R4(9.971e-8);
    const real h0 = R4(5.540e-10), h1 = -R4(1.7682e-11), h2 = R4(3.513e-13);
    const real j1 = -R4(1.4300e-12);
    const real S3_2 = sS;
    // P**2 and P**3 as the products P*P and (P*P)*P
    const real del_Cpstp = (((((d4 * T68 + d3) * T68 + d2) * T68 + d1) * T68 + d0) * S0 +
                            ((e2 * T68 + e1) * T68 + e0) * S3_2) * P +
                           ((((f3 * T68 + f2) * T68 + f1) * T68 + f0) * S0 + g0 * S3_2) * (P * P) +
                           (((h2 * T68 + h1) * T68 + h0) * S0 + j1 * T68 * S3_2) * ((P * P) * P);
    return Cpst0 + del_Cp0t0 + del_Cpstp;
}

// fraction of the surface shortwave left at depth z < 0: swr_paul_sim
// (type_swr_body 1) or swr_soloviev (2), fv_tracer.F90:1566-1631
__device__ __forceinline__ real swr_frac(const Dev &d, int n, real z) {
    if (d.type_swr_body == 1) {
        const real R = d.jer_const ? d.Rjc : (real)d.Rj[n];
        const real a = d.jer_const ? d.ajc : (real)d.aj[n];
        const real b = d.jer_const ? d.bjc : (real)d.bj[n];
        return R * (real)fesomc_exp((double)(z / a)) + (real(1.0) - R) * (real)fesomc_exp((double)(z / b));
    }
    // a = (1, 0, 0), b = (10, 0, 0): sum(a*exp(b*z)), exp(0*z) = 1
    return (real(1.0) * (real)fesomc_exp((double)(real(10.0) * z)) + real(0.0) * real(1.0)) + real(0.0) * real(1.0);
}

// calc_heat_flux_sw (fv_tracer.F90:1636-1697) for layer z (0-based) of node
// n: the shortwave absorbed in the layer (and the non-solar flux in the top
// one, the bottom-reflected rest in the lowest), as a temperature tendency.
// As in the reference: T and S are T_old + T_aver and S_old + S_aver (the
// tracers of the previous step, which are not shifted by their means at
// this point), and sw_cp receives them in the order (T, S) against its
// (S, T) arguments.
__device__ real heat_source(const Dev &d, int n, size_t base, int z, real aj, real T_aver, real S_aver) {
    const real d1 = zbar_of(d, aj, z), d2 = zbar_of(d, aj, z + 1);
    const real T = d.Told_new[base + z] + T_aver;
    const real S = d.Sold_new[base + z] + S_aver;
    const real aux = (d1 + d2) * real(0.5);
    const real rho = d.rho_c[base + z] + d.density_0;
    const real ms = (real)d.mslp[n];
    const real P = (ms == real(0.0)) ? (rho * kG * aux + real(kPref)) * real(10.0e-5) : (rho * kG * aux + ms) * real(10.0e-5);
    const real c_p = sw_cp(T, S, P);
    const real swr1 = swr_frac(d, n, -d1), swr2 = swr_frac(d, n, -d2);
    const real jc = jc_of(d, aj, z);
    const real qsr = (real)d.qsr[n];
    real src;
    if (z == 0) src = (qsr * (swr1 - swr2) + (real)d.qns[n]) / (jc * c_p * rho);
    else src = qsr * (swr1 - swr2) / (jc * c_p * rho);
    // the rest of the shortwave, 0.2 of it reflected by the bottom (REAL(4) 0.2)
    if (z == d.L - 1) src = src + R4(0.2) * qsr * (swr2) / (jc * c_p * rho);
    return src;
}

// calc_evap_precip (fv_tracer.F90:1699-1752): freshwater (E - P) source of
// the top layer; T0 and S0 are the top layer minus their means.
__device__ real evap_precip(const Dev &d, int n, real aj, real T0, real S0, real T_aver, real S_aver) {
    const real T = T0 + T_aver;
    const real S = S0 + S_aver;
    const real rho = density_jm(T, real(0.0), -zbar_of(d, aj, 0), d.density_0);
    const real den = (rho + d.density_0) * jc_of(d, aj, 0);
    real frw = real(0.0);
    if (den != real(0.0)) {
        frw = S * (real)d.emp[n] / den;
        if (S <= real(0.2) && frw < real(0.0)) frw = real(0.0);
    }
    return frw;
}

// kAtm: the atmospheric sources (key_atm) compiled in; the plain kernel keeps
// its register count without them
template <bool kAtm>
__global__ void __launch_bounds__(kVdBlock) k_vdiff_col(Dev d) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    real *sm = reinterpret_cast<real *>(sm_raw);
    const int L = d.L, NS = d.NS;
    real *col = sm + threadIdx.x;
    const int bd = blockDim.x;
    auto CP = [&](int k) -> real & { return col[((size_t)0 * L + k) * bd]; };
    auto TP = [&](int k) -> real & { return col[((size_t)1 * L + k) * bd]; };
    auto SP = [&](int k) -> real & { return col[((size_t)2 * L + k) * bd]; };
    GRID_LOOP(ii, d.N) {
        const int n = (int)ii;
        const real T_aver = t_aver_of(d, n), S_aver = s_aver_of(d, n);
        const size_t base = (size_t)n * L;
        const real aj = jac_a(d, d.eta_jac, n);
        const real *Kv = d.Kv + (size_t)n * NS;
        auto Tz = [&](int z) { return d.TF_adv[base + z] - T_aver; };
        auto Sz = [&](int z) { return vd_salt(d, n, base, z, aj, S_aver); };
        // forward elimination; the right-hand side of layer k uses T(k-1..k+1)
        real Tm = real(0.0), T0 = Tz(0), Tp = Tz(1);
        real Sm = real(0.0), S0 = Sz(0), Sp = Sz(1);
        real cpv = real(0.0), tpv = real(0.0), spv = real(0.0);  // the recurrences, in registers
        // surface sources on wet nodes with atmospheric forcing (fv_tracer.F90:1376,1396-1418)
        const bool atm = kAtm && d.mask_wd_node[n] != real(0.0);
        const real frw = atm ? evap_precip(d, n, aj, T0, S0, T_aver, S_aver) : real(0.0);
        for (int k = 0; k < L; ++k) {
            real a, b, c, tr, sr;
            vd_coef(d, Kv, aj, k, a, b, c);
            if (k == 0) {
                tr = c * (-Tp + T0);
                sr = c * (-Sp + S0);
            } else if (k == L - 1) {
                tr = a * (T0 - Tm);
                sr = a * (S0 - Sm);
            } else {
                tr = -a * Tm - c * Tp + (a + c) * T0;
                sr = -a * Sm - c * Sp + (a + c) * S0;
            }
            if (atm) {
                tr = tr + d.dt * heat_source(d, n, base, k, aj, T_aver, S_aver);
                if (k == 0) sr = sr + d.dt * frw;
            }
            if (k == 0) {
                cpv = c / b;
                tpv = tr / b;
                spv = sr / b;
            } else {
                const real m = real(1.0) / (b - cpv * a);
                cpv = c * m;
                tpv = (tr - tpv * a) * m;
                spv = (sr - spv * a) * m;
            }
            CP(k) = cpv;
            TP(k) = tpv;
            SP(k) = spv;
            Tm = T0; T0 = Tp;
            Sm = S0; S0 = Sp;
            if (k + 2 < L) { Tp = Tz(k + 2); Sp = Sz(k + 2); }
        }
        // back substitution and update, bottom to top
        unsigned int st = 0;
        real tr = real(0.0), sr = real(0.0);
        for (int z = L - 1; z >= 0; --z) {
            if (z == L - 1) { tr = TP(z); sr = SP(z); }
            else { tr = TP(z) - CP(z) * tr; sr = SP(z) - CP(z) * sr; }
            const size_t i = base + z;
            real t = Tz(z) + tr + T_aver;
            real s = Sz(z) + sr + S_aver;
            if (fabs(s) < real(1.0e-12)) s = fabs(s);
            if (s < real(0.0)) st |= 0x1u;
            if (t < -real(3.0)) st |= 0x2u;
            if (!isfinite(t) || !isfinite(s)) st |= 0x4u;
            d.TF[i] = t;
            d.SF[i] = s;
            d.T_old[i] = d.Told_new[i];
            d.S_old[i] = d.Sold_new[i];
        }
        if (!isfinite(d.eta_n[n])) st |= 0x4u;
        if (st) atomicOr(d.status, st);
    }
}

// ---------------------------------------------------------------------------
// energy: compensated (Neumaier) partial sums per block, then one block.
// FP64 accumulation in both precision forms.
// ---------------------------------------------------------------------------
struct KSum {
    double s, c;
    __device__ void add(double x) {
        double t = s + x;
        if (fabs(s) >= fabs(x)) c += (s - t) + x;
        else c += (x - t) + s;
        s = t;
    }
    __device__ double value() const { return s + c; }
};

__global__ void k_energy_part(Dev d, double *part) {
    __shared__ double sh[3][kRedBlock];
    KSum pe{0.0, 0.0}, ke{0.0, 0.0}, ar{0.0, 0.0};
    GRID_LOOP(i, d.N) {
        const double e = d.eta_n[i];
        const double a = d.area[i];
        pe.add(0.5 * kG64 * a * (e * e));
        ar.add(a);
    }
    GRID_LOOP(i, d.E) {
        const int4 en = d.elem_nodes[i];
        const real4 w = d.w_cv[i];
        const double s = wsum_d(w, dmax(d.Dmin_d, (double)d.depth[en.x] + d.eta_n[en.x]),
                                dmax(d.Dmin_d, (double)d.depth[en.y] + d.eta_n[en.y]),
                                dmax(d.Dmin_d, (double)d.depth[en.z] + d.eta_n[en.z]),
                                dmax(d.Dmin_d, (double)d.depth[en.w] + d.eta_n[en.w]));
        const real2 u = d.U_n_2D[i];
        const double ux = u.x, uy = u.y;
        ke.add(0.5 * s * (double)d.elem_area[i] * (ux * ux + uy * uy));
    }
    sh[0][threadIdx.x] = pe.value();
    sh[1][threadIdx.x] = ke.value();
    sh[2][threadIdx.x] = ar.value();
    __syncthreads();
    if (threadIdx.x < 3) {
        KSum t{0.0, 0.0};
        for (int k = 0; k < kRedBlock; ++k) t.add(sh[threadIdx.x][k]);
        part[(size_t)blockIdx.x * 3 + threadIdx.x] = t.value();
    }
}

__global__ void k_energy_final(const double *part, int nparts, double *out) {
    if (threadIdx.x < 3 && blockIdx.x == 0) {
        KSum t{0.0, 0.0};
        for (int b = 0; b < nparts; ++b) t.add(part[(size_t)b * 3 + threadIdx.x]);
        out[threadIdx.x] = t.value();
    }
}

// ---- launch wrappers --------------------------------------------------------
// partials per member of the tracer min / max: kRedGrid for one mesh, fewer
// per member for packed members (at least 8)
int minmax_parts(int n_members) { return n_members <= 1 ? kRedGrid : (kRedGrid / n_members > 8 ? kRedGrid / n_members : 8); }
void launch_minmax(const Dev &d, cudaStream_t s) {
    const int parts = minmax_parts(d.n_members);
    k_minmax_part<<<dim3(parts, d.n_members), kRedBlock, 0, s>>>(d);
    k_minmax_final<<<d.n_members, 32, 0, s>>>(d, parts);
}
// ---- sbc_do on the device: bulk surface fluxes ------------------------------
// psi_h / psi_m of Large & Yeager (2004), eq. 8c-8e (fv_sbc.F90:620-662);
// SIGN(0.5, x) is copysign.  FP64 throughout.
__device__ __forceinline__ double sbc_psi_h(double zta) {
    double X2 = sqrt(fabs(1.0 - 16.0 * zta));
    X2 = fmax(X2, 1.0);
    const double stabit = 0.5 + copysign(0.5, zta);
    return -5.0 * zta * stabit + (1.0 - stabit) * (2.0 * fesomc_log((1.0 + X2) / 2.0));
}
__device__ __forceinline__ double sbc_psi_m(double zta) {
    double X2 = sqrt(fabs(1.0 - 16.0 * zta));
    X2 = fmax(X2, 1.0);
    const double X = sqrt(X2);
    const double stabit = 0.5 + copysign(0.5, zta);
    const double pi = 3.141592653589793;
    return -5.0 * zta * stabit + (1.0 - stabit) * (2.0 * fesomc_log((1.0 + X) / 2.0) + fesomc_log((1.0 + X2) / 2.0) -
                                                    2.0 * fesomc_atan(X) + pi / 2.0);
}

// core_coeff_2z (fv_sbc.F90:484-641): transfer coefficients for momentum,
// sensible and latent heat, and the air temperature and humidity shifted
// from zt to zu, in 5 iterations on the Monin-Obukhov length
__device__ void sbc_core_coeff_2z(double zt, double zu, double sst, double T_zt, double q_sat, double q_zt, double dU,
                                  double &Cd, double &Ch, double &Ce, double &T_zu, double &q_zu) {
    const double grav = 9.8, kappa = 0.4;
    const double dU10 = fmax(0.5, dU);
    double dT = T_zt - sst;
    double dq = q_zt - q_sat;
    double stab = 0.5 + copysign(0.5, dT);
    double Cd_n10 = 1E-3 * (2.7 / dU10 + 0.142 + dU10 / 13.09);
    double sqrt_Cd_n10 = sqrt(Cd_n10);
    double Ce_n10 = 1E-3 * (34.6 * sqrt_Cd_n10);
    double Ch_n10 = 1E-3 * sqrt_Cd_n10 * (18.0 * stab + 32.7 * (1.0 - stab));
    Cd = Cd_n10;
    Ce = Ce_n10;
    Ch = Ch_n10;
    double sqrt_Cd = sqrt(Cd);
    T_zu = T_zt;
    q_zu = q_zt;
    const double log_zt_zu = fesomc_log(zt / zu), log_zu_10 = fesomc_log(zu / 10.0);
    for (int j_itt = 1; j_itt <= 5; ++j_itt) {
        dT = T_zu - sst;
        dq = q_zu - q_sat;
        const double T_vpot = T_zu * (1.0 + 0.608 * q_zu);
        const double U_star = sqrt_Cd * dU10;
        const double T_star = Ch / sqrt_Cd * dT;
        const double q_star = Ce / sqrt_Cd * dq;
        const double L = (U_star * U_star) / (kappa * grav / T_vpot * (T_star * (1.0 + 0.608 * q_zu) + 0.608 * T_zu * q_star));
        double zeta_u = zu / L;
        zeta_u = copysign(fmin(fabs(zeta_u), 10.0), zeta_u);
        double zeta_t = zt / L;
        zeta_t = copysign(fmin(fabs(zeta_t), 10.0), zeta_t);
        const double zpsi_hu = sbc_psi_h(zeta_u);
        const double zpsi_ht = sbc_psi_h(zeta_t);
        const double zpsi_m = sbc_psi_m(zeta_u);
        const double U_n10 = fmax(0.25, dU10 / (1.0 + sqrt_Cd_n10 / kappa * (log_zu_10 - zpsi_m)));
        T_zu = T_zt - T_star / kappa * (log_zt_zu + zpsi_hu - zpsi_ht);
        q_zu = q_zt - q_star / kappa * (log_zt_zu + zpsi_hu - zpsi_ht);
        stab = 0.5 + copysign(0.5, q_zu);
        q_zu = stab * q_zu;
        Cd_n10 = 1E-3 * (2.7 / U_n10 + 0.142 + U_n10 / 13.09);
        sqrt_Cd_n10 = sqrt(Cd_n10);
        Ce_n10 = 1E-3 * (34.6 * sqrt_Cd_n10);
        stab = 0.5 + copysign(0.5, zeta_u);
        Ch_n10 = 1E-3 * sqrt_Cd_n10 * (18.0 * stab + 32.7 * (1.0 - stab));
        double xct = 1.0 + sqrt_Cd_n10 / kappa * (log_zu_10 - zpsi_m);
        Cd = Cd_n10 / (xct * xct);
        sqrt_Cd = sqrt(Cd);
        const double xlogt = log_zu_10 - zpsi_hu;
        xct = 1.0 + Ch_n10 * xlogt / kappa / sqrt_Cd_n10;
        Ch = Ch_n10 * sqrt_Cd / sqrt_Cd_n10 / xct;
        xct = 1.0 + Ce_n10 * xlogt / kappa / sqrt_Cd_n10;
        Ce = Ce_n10 * sqrt_Cd / sqrt_Cd_n10 / xct;
    }
}

// data_timeinterp + apply_atm_fluxes (fv_sbc.F90:838-868, 368-482) per node,
// type_task 3 without sea ice: the fields at the step's time, the winds,
// the heat and freshwater fluxes, the stress per node.  The relative wind
// subtracts the surface Unode / Vnode of the previous step, the surface
// temperature is TF's top layer.  rhoa, albo, emiss_wat are REAL(4).
__global__ void k_atm_nodes(Dev d, AtmDev a) {
    const double now_date = a.clock[0];
    const double rhoa = (double)1.3f, cpa = 1005.0, Lv = 2.5e6, Stef = 5.67e-8, albo = (double)0.1f,
                 emiss_wat = (double)0.97f;
    const int L = d.L;
    GRID_LOOP(ii, d.N) {
        const int i = (int)ii;
        const double *ca = a.coef_a + (size_t)i * 8, *cb = a.coef_b + (size_t)i * 8;
        double atm[8];
#pragma unroll
        for (int f = 0; f < 8; ++f) atm[f] = now_date * ca[f] + cb[f];
        d.windx[i] = (real)atm[0];
        d.windy[i] = (real)atm[1];
        const double wdx = atm[0] - (double)d.Unode[(size_t)i * L];
        const double wdy = atm[1] - (double)d.Vnode[(size_t)i * L];
        const double wndm = sqrt(wdx * wdx + wdy * wdy);
        const double tf0 = (double)d.TF[(size_t)i * L];
        const double zst = tf0 + 273.15;
        const double q_sat = 0.98 * 640380.0 / rhoa * fesomc_exp(-5107.4 / zst);
        double Cd, Ch, Ce, t_zu, q_zu;
        sbc_core_coeff_2z(2.0, 10.0, zst, atm[5], q_sat, atm[2], wndm, Cd, Ch, Ce, t_zu, q_zu);
        const double rtmp = rhoa * wndm * Cd;
        a.tau_node[2 * (size_t)i] = rtmp * wdx;
        a.tau_node[2 * (size_t)i + 1] = rtmp * wdy;
        const double zevap = fmax(0.0, rhoa * Ce * (q_sat - q_zu) * wndm);
        const double zqsb = rhoa * cpa * Ch * (zst - t_zu) * wndm;
        const double zqlw = a.net_flux == 0 ? atm[4] - emiss_wat * Stef * zst * zst * zst * zst : atm[4];
        const double zqla = Lv * zevap;
        double qns = zqlw - zqsb - zqla;
        if (tf0 < -2.0 && qns < 0.0) qns = 0.0;
        d.qns[i] = qns;
        d.emp[i] = zevap - atm[6] / a.prec_coef;
        d.qsr[i] = (1.0 - albo) * atm[3];
        d.mslp[i] = atm[7];
    }
}
// the stress per element: sum(w_cv * taux_node(elem2D_nodes)) in node order
__global__ void k_atm_stress(Dev d, AtmDev a) {
    GRID_LOOP(ee, d.E) {
        const int e = (int)ee;
        const int4 en = d.elem_nodes[e];
        const real4 w = d.w_cv[e];
        const int nd[4] = {en.x, en.y, en.z, en.w};
        const double wv[4] = {(double)w.x, (double)w.y, (double)w.z, (double)w.w};
        double sx = 0.0, sy = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            sx = sx + wv[k] * a.tau_node[2 * (size_t)nd[k]];
            sy = sy + wv[k] * a.tau_node[2 * (size_t)nd[k] + 1];
        }
        d.taux[e] = (real)sx;
        d.tauy[e] = (real)sy;
    }
}
void launch_atm(const Dev &d, const AtmDev &a, cudaStream_t s) {
    k_atm_nodes<<<grid_for(d.N, 128), 128, 0, s>>>(d, a);
    k_atm_stress<<<grid_for(d.E, 256), 256, 0, s>>>(d, a);
}

// T_aver / S_aver from a range the host gives (fesomc_gpu_set_tracer_range:
// the min / max over the whole domain of a decomposed mesh), with
// k_minmax_final's expression
__global__ void k_aver_from_range(Dev d, const double *r) {
    if (threadIdx.x == 0) {
        d.aver[0] = real(0.5) * ((real)r[0] + (real)r[1]);
        d.aver[1] = real(0.5) * ((real)r[2] + (real)r[3]);
    }
}
void launch_aver_from_range(const Dev &d, const double *range, cudaStream_t s) {
    k_aver_from_range<<<1, 32, 0, s>>>(d, range);
}
void launch_ab2(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_AB2, 256);
    k_ab2_node<<<grid_for((long long)d.N * d.L, b), b, 0, s>>>(d);
}
void launch_upwind(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_UPWIND, 128);
    k_upwind_h<<<grid_for((long long)d.N * d.L, b), b, 0, s>>>(d);
}
void launch_muscl_egrad(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_MEGRAD, 256);
    k_muscl_egrad<<<grid_for((long long)d.E * d.L, b), b, 0, s>>>(d);
}
void launch_muscl_ngrad(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_MNGRAD, 256);
    k_muscl_ngrad<<<grid_for((long long)d.N * d.L, b), b, 0, s>>>(d);
}
void launch_miura(const Dev &d, cudaStream_t s) {
    k_miura_prep<<<grid_for((long long)d.N * d.L, 256), 256, 0, s>>>(d);
    k_miura_egrad<<<grid_for((long long)d.E * d.L, 256), 256, 0, s>>>(d);
    k_miura_ngrad<<<grid_for((long long)d.N * d.L, 256), 256, 0, s>>>(d);
    k_miura_edge<<<grid_for((long long)d.Ed * d.L, 256), 256, 0, s>>>(d);
    k_miura_h<<<grid_for((long long)d.N * d.L, 128), 128, 0, s>>>(d);
}
void launch_muscl_edge(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_MEDGE, 256);
    k_muscl_edge<<<grid_for((long long)d.Ed * d.L, b), b, 0, s>>>(d);
}
void launch_muscl_h(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_MH, 128);
    k_muscl_h<<<grid_for((long long)d.N * d.L, b), b, 0, s>>>(d);
}
// ---- tracer_impl_vert_diff on tiles of columns (knob vdiff_form = 2) -------
// k_vdiff_col reads each column with one thread, so a warp's loads of one
// layer touch 32 rows L values apart.  Here a block takes kVtCols (128 or
// 64)
// consecutive nodes, whose columns are one contiguous range of every
// [node][layer] field: it stages T - T_aver, the river-adjusted S - S_aver
// and Kv in shared memory with coalesced loads (copying Told_new / Sold_new
// to T_old / S_old on the way; each thread loads a batch of items before
// storing any), solves each column with one thread from
// shared memory (rows of odd stride: no bank conflicts) with the sweep's
// recurrences in registers (the layer count LC is fixed at compile time),
// writes the new tracers over the staged ones and stores them coalesced.
// The arithmetic and its order are k_vdiff_col's.
constexpr int kVtBatch = 4;
__host__ __device__ __forceinline__ int vd_odd(int x) { return x | 1; }

template <bool kAtm, int LC, int kVtCols>
__global__ void __launch_bounds__(kVtCols) k_vdiff_tile(Dev d) {
    extern __shared__ __align__(16) unsigned char vt_smem[];
    constexpr int L = LC, LP = LC | 1;
    const int NS = d.NS, KP = vd_odd(d.NS), N = d.N;
    real *sT = reinterpret_cast<real *>(vt_smem);  // row j: node n0 + j
    real *sS = sT + kVtCols * LP;
    real *sK = sS + kVtCols * LP;
    // with the atmospheric sources: the heat source of every (node, layer),
    // formed in the staging phase by all threads instead of in the serial
    // column solve
    real *sH = sK + kVtCols * KP;
    for (long long n0 = (long long)blockIdx.x * kVtCols; n0 < N; n0 += (long long)gridDim.x * kVtCols) {
        const int nt = (int)(N - n0 < kVtCols ? N - n0 : kVtCols);
        // staging: kVtBatch items per thread loaded before any is used, so
        // that each thread keeps several loads in flight
        for (int i0 = threadIdx.x; i0 < nt * NS; i0 += kVtBatch * kVtCols) {
            real kv[kVtBatch];
#pragma unroll
            for (int u = 0; u < kVtBatch; ++u) {
                const int i = i0 + u * kVtCols;
                kv[u] = i < nt * NS ? d.Kv[(size_t)n0 * NS + i] : real(0.0);
            }
#pragma unroll
            for (int u = 0; u < kVtBatch; ++u) {
                const int i = i0 + u * kVtCols, j = i / NS;
                if (i < nt * NS) sK[j * KP + (i - j * NS)] = kv[u];
            }
        }
        for (int i0 = threadIdx.x; i0 < nt * L; i0 += kVtBatch * kVtCols) {
            real ta[kVtBatch], sa[kVtBatch], tn[kVtBatch], sn[kVtBatch];
#pragma unroll
            for (int u = 0; u < kVtBatch; ++u) {
                const int i = i0 + u * kVtCols;
                const size_t g = (size_t)n0 * L + (i < nt * L ? i : 0);
                ta[u] = d.TF_adv[g];
                sa[u] = d.SF_adv[g];
                tn[u] = d.Told_new[g];
                sn[u] = d.Sold_new[g];
            }
#pragma unroll
            for (int u = 0; u < kVtBatch; ++u) {
                const int i = i0 + u * kVtCols;
                if (i >= nt * L) continue;
                const int j = i / L, z = i - j * L;
                const int n = (int)n0 + j;
                const size_t g = (size_t)n0 * L + i;
                const real ajn = jac_a(d, d.eta_jac, n);
                sT[j * LP + z] = ta[u] - t_aver_of(d, n);
                sS[j * LP + z] = vd_salt_of(d, n, z, ajn, sa[u], sn[u], s_aver_of(d, n));
                if (kAtm)
                    sH[j * LP + z] = d.mask_wd_node[n] != real(0.0)
                                         ? heat_source(d, n, (size_t)n * L, z, ajn, t_aver_of(d, n), s_aver_of(d, n))
                                         : real(0.0);
                d.T_old[g] = tn[u];
                d.S_old[g] = sn[u];
            }
        }
        __syncthreads();
        if ((int)threadIdx.x < nt) {
            const int j = threadIdx.x, n = (int)n0 + j;
            const real T_aver = t_aver_of(d, n), S_aver = s_aver_of(d, n);
            const size_t base = (size_t)n * L;
            const real aj = jac_a(d, d.eta_jac, n);
            const real *Kv = sK + j * KP;
            real *T = sT + j * LP, *S = sS + j * LP;
            real CP[LC], TP[LC], SP[LC];
            real cpv = real(0.0), tpv = real(0.0), spv = real(0.0);
            const bool atm = kAtm && d.mask_wd_node[n] != real(0.0);
            const real frw = atm ? evap_precip(d, n, aj, T[0], S[0], T_aver, S_aver) : real(0.0);
#pragma unroll
            for (int k = 0; k < L; ++k) {
                real a, b, c, tr, sr;
                vd_coef(d, Kv, aj, k, a, b, c);
                const real T0 = T[k], S0 = S[k];
                if (k == 0) {
                    tr = c * (-T[1] + T0);
                    sr = c * (-S[1] + S0);
                } else if (k == L - 1) {
                    tr = a * (T0 - T[k - 1]);
                    sr = a * (S0 - S[k - 1]);
                } else {
                    tr = -a * T[k - 1] - c * T[k + 1] + (a + c) * T0;
                    sr = -a * S[k - 1] - c * S[k + 1] + (a + c) * S0;
                }
                if (atm) {
                    tr = tr + d.dt * sH[j * LP + k];
                    if (k == 0) sr = sr + d.dt * frw;
                }
                if (k == 0) {
                    cpv = c / b;
                    tpv = tr / b;
                    spv = sr / b;
                } else {
                    const real m = real(1.0) / (b - cpv * a);
                    cpv = c * m;
                    tpv = (tr - tpv * a) * m;
                    spv = (sr - spv * a) * m;
                }
                CP[k] = cpv;
                TP[k] = tpv;
                SP[k] = spv;
            }
            unsigned int st = 0;
            real tr = real(0.0), sr = real(0.0);
#pragma unroll
            for (int z = L - 1; z >= 0; --z) {
                if (z == L - 1) { tr = TP[z]; sr = SP[z]; }
                else { tr = TP[z] - CP[z] * tr; sr = SP[z] - CP[z] * sr; }
                real t = T[z] + tr + T_aver;
                real s = S[z] + sr + S_aver;
                if (fabs(s) < real(1.0e-12)) s = fabs(s);
                if (s < real(0.0)) st |= 0x1u;
                if (t < -real(3.0)) st |= 0x2u;
                if (!isfinite(t) || !isfinite(s)) st |= 0x4u;
                T[z] = t;
                S[z] = s;
            }
            if (!isfinite(d.eta_n[n])) st |= 0x4u;
            if (st) atomicOr(d.status, st);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nt * L; i += kVtCols) {
            const int j = i / L, z = i - j * L;
            const size_t g = (size_t)n0 * L + i;
            d.TF[g] = sT[j * LP + z];
            d.SF[g] = sS[j * LP + z];
        }
        __syncthreads();
    }
}

// columns per tile: 128 (vdiff_form 2) or 64 (3, the default)
static int vdiff_cols(const Dev &d) { return d.tune[TK_VDIFF] == 2 ? 128 : 64; }
static size_t vdiff_tile_smem(const Dev &d, int cols, bool atm) {
    return (size_t)cols * ((atm ? 3 : 2) * vd_odd(d.L) + vd_odd(d.NS)) * sizeof(real);
}
// the tiled form is compiled for 10 and 20 layers (11 and 21 sigma levels)
static bool vdiff_tiled(const Dev &d) { return d.tune[TK_VDIFF] != 1 && (d.L == 10 || d.L == 20); }

static int vdiff_block(const Dev &d) { return d.L <= 48 ? kVdBlock : 32; }
static size_t vdiff_smem(const Dev &d) { return (size_t)3 * d.L * vdiff_block(d) * sizeof(real); }
template <int LC, int C>
static bool config_vdiff_tile(const Dev &d) {
    return raise_smem_limit(k_vdiff_tile<false, LC, C>, vdiff_tile_smem(d, C, false)) == cudaSuccess &&
           raise_smem_limit(k_vdiff_tile<true, LC, C>, vdiff_tile_smem(d, C, true)) == cudaSuccess;
}
int config_vdiff(const Dev &d) {
    if (raise_smem_limit(k_vdiff_col<false>, vdiff_smem(d)) != cudaSuccess ||
        raise_smem_limit(k_vdiff_col<true>, vdiff_smem(d)) != cudaSuccess)
        return 1;
    if (d.L == 10) return config_vdiff_tile<10, 128>(d) && config_vdiff_tile<10, 64>(d) ? 0 : 1;
    if (d.L == 20) return config_vdiff_tile<20, 128>(d) && config_vdiff_tile<20, 64>(d) ? 0 : 1;
    return 0;
}
template <int LC, int C>
static void launch_vdiff_tile(const Dev &d, cudaStream_t s) {
    const long long tiles = ((long long)d.N + C - 1) / C;
    const int g = (int)(tiles < (1LL << 30) ? tiles : (1LL << 30));
    if (d.key_atm) k_vdiff_tile<true, LC, C><<<g, C, vdiff_tile_smem(d, C, true), s>>>(d);
    else k_vdiff_tile<false, LC, C><<<g, C, vdiff_tile_smem(d, C, false), s>>>(d);
}
void launch_vdiff(const Dev &d, cudaStream_t s) {
    if (vdiff_tiled(d)) {
        const bool c64 = vdiff_cols(d) == 64;
        if (d.L == 10 && c64) launch_vdiff_tile<10, 64>(d, s);
        else if (d.L == 10) launch_vdiff_tile<10, 128>(d, s);
        else if (c64) launch_vdiff_tile<20, 64>(d, s);
        else launch_vdiff_tile<20, 128>(d, s);
        return;
    }
    if (d.key_atm) k_vdiff_col<true><<<grid_for(d.N, vdiff_block(d)), vdiff_block(d), vdiff_smem(d), s>>>(d);
    else k_vdiff_col<false><<<grid_for(d.N, vdiff_block(d)), vdiff_block(d), vdiff_smem(d), s>>>(d);
}
int energy_parts() { return kRedGrid; }
void launch_energy(const Dev &d, double *part, double *out, cudaStream_t s) {
    k_energy_part<<<kRedGrid, kRedBlock, 0, s>>>(d, part);
    k_energy_final<<<1, 32, 0, s>>>(part, kRedGrid, out);
}


// Largest block (threads) each tunable kernel of this file can launch with
// (its registers and launch bounds): lim[knob] lowered to that.
static void tune_lower(int *lim, int knob, const void *k) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, k) == cudaSuccess && a.maxThreadsPerBlock < lim[knob]) lim[knob] = a.maxThreadsPerBlock;
}
void tune_limits_tracer(int *lim) {
    tune_lower(lim, TK_AB2, (const void *)k_ab2_node);
    tune_lower(lim, TK_MEGRAD, (const void *)k_muscl_egrad);
    tune_lower(lim, TK_MNGRAD, (const void *)k_muscl_ngrad);
    tune_lower(lim, TK_MEDGE, (const void *)k_muscl_edge);
    tune_lower(lim, TK_MH, (const void *)k_muscl_h);
    tune_lower(lim, TK_UPWIND, (const void *)k_upwind_h);
}

FESOMC_PREC_END
