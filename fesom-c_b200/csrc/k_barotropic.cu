// External-mode (barotropic) sub-cycle kernels: one sub-step of
// timestep_AB_2D (src/fv_main.F90:1372-1634) is
//   ab3_elem  : AB3 extrapolation of U, element mean total depth (aux_elem)
//               and the least-squares velocity gradients of UAB
//   ssh_node  : edge-flux divergence gathered per node in edge order
//               (compute_ssh_rhs_elem), rivers, OB tide, eta update, AM4
//   [sub-step 1 only: puls_elem, el2nodes, p1_elem]
//   u2d_elem  : update_2D_vel (pressure gradient, Coriolis, wind, upwind
//               momentum advection gathered per element, filter viscosity,
//               3D->2D forcing, implicit friction, wet/dry mask) fused with
//               the time-level rotation of U and the U_filt accumulation
//   rot_nodes : eta time-level rotation
// All kernels are HBM-bandwidth bound.  Both precision forms compile them:
// the elevation, total depths and the wet/dry tests are FP64 in both (the
// *_d scalars, wsum_d / wexp_d), the 2D momentum follows 'real'.
#include "device_common.cuh"

FESOMC_PREC_BEGIN

// AB3 coefficients, timestep_AB_2D fv_main.F90:1403,1408
template <typename T>
__device__ __forceinline__ T ab3(T b, T x0, T x1, T x2) {
    return (T(1.5) + b) * x0 - (T(0.5) + T(2.0) * b) * x1 + b * x2;
}
__device__ __forceinline__ real2 ab3v(real b, real2 x0, real2 x1, real2 x2) {
    return make_real2(ab3(b, x0.x, x1.x, x2.x), ab3(b, x0.y, x1.y, x2.y));
}

// ---------------------------------------------------------------------------
// ab3_elem: UAB (fv_main.F90:1407-1410) and aux_elem
// (fv_average_dynamic.F90:66-86); vel_gradients_2D(UAB) follows in
// k_velgrad2d, which reads the neighbours' UAB (a third faster than forming
// their AB3 again in this kernel).
// ---------------------------------------------------------------------------
__global__ void k_ab3_elem(Dev d) {
    GRID_LOOP(ii, d.E) {
        const int e = (int)ii;
        const real b = d.beta;
        const real2 uab = ab3v(b, d.U_n_2D[e], d.U_n_1[e], d.U_n_2[e]);
        d.UAB[e] = uab;
        const int4 en = d.elem_nodes[e];
        const int nd[4] = {en.x, en.y, en.z, en.w};
        double ad[4];
        for (int i = 0; i < 4; ++i) {
            const int n = nd[i];
            const double etaab = ab3<double>(d.beta_d, d.eta_n[n], d.eta_n_1[n], d.eta_n_2[n]);
            ad[i] = d.Dmin_d;
            const double ttl = etaab + (double)d.depth[n];
            if (ttl > d.Dmin_d) ad[i] = ttl;
        }
        const real4 w = d.w_cv[e];
        d.aux_elem[e] = (real)wexp_d(w, ad[0], ad[1], ad[2], ad[3]);
    }
}

// edge flux c1 of compute_ssh_rhs_elem (fv_average_dynamic.F90:119-120, 152-153)
__device__ __forceinline__ real ssh_edge_flux(const Dev &d, int ed) {
    const int2 et = d.edge_tri[ed];
    const real4 X = d.edge_cross[ed];
    const real2 u1 = d.UAB[et.x];
    real c1 = (u1.y * X.x - u1.x * X.y) * d.aux_elem[et.x];
    if (ed < d.Ed_in) {
        const real2 u2 = d.UAB[et.y];
        c1 = c1 + (-u2.y * X.z + u2.x * X.w) * d.aux_elem[et.y];
    }
    return c1;
}

// the SSH edge flux of every edge, once, for both end nodes to gather (the
// flux array stays in L2; a quarter faster than forming it per node)
__global__ void k_ssh_edge(Dev d) {
    GRID_LOOP(ed, d.Ed) d.sshfl[ed] = ssh_edge_flux(d, (int)ed);
}

// ---------------------------------------------------------------------------
// ssh_node: ssh_rhs gather (serial scatter order), rivers, open boundary,
// eta_new = eta_n + dt_2D*rhs/area (fv_main.F90:1432-1435), then the AM4
// elevation of update_2D_vel (fv_average_dynamic.F90:290-295) into etaAB and
// the node wet/dry mask (wad_mask, fv_main.F90:1302-1304).
// ob_val holds the open-boundary elevation of this sub-step (reference formula
// fv_average_dynamic.F90:190-216), written before the step either by the host
// (fesomc_gpu_set_forcing) or by k_forcing_values (device forcing).
// ---------------------------------------------------------------------------
// 40 registers: 6 resident blocks per SM instead of 5 (3 % faster).
__global__ void __maxnreg__(40) k_ssh_node(Dev d, int sub) {
    const double de = 0.614, ga = 0.088, ep = 0.013, fe = 1.0 - de - ga - ep;
    GRID_LOOP(ii, d.N) {
        const int n = (int)ii;
        double acc = 0.0;   // ssh_rhs: FP64 accumulation of the edge fluxes
        const int p0 = d.node_eptr[n], p1 = d.node_eptr[n + 1];
#pragma unroll 4
        for (int p = p0; p < p1; ++p) {
            const int code = d.node_eidx[p];
            const double c1 = (double)d.sshfl[code >> 1];
            if (code & 1) acc = acc - c1;
            else acc = acc + c1;
        }
        if (d.key_rivers) {
            for (int p = d.node_rptr[n]; p < d.node_rptr[n + 1]; ++p) acc = acc + d.runoff[d.node_ridx[p]];
        }
        const int q = d.obn_of_node[n];
        if (d.TF_presence && q >= 0) acc = d.ob_val[(size_t)sub * d.nobn + q];
        const double en = d.eta_n[n];
        double enew = acc;
        if (d.index_nod2D[n] < 2) enew = en + d.dt_2D_d * acc / (double)d.area[n];
        d.eta_new[n] = enew;
        const double eab = de * enew + fe * en + ga * d.eta_n_1[n] + ep * d.eta_n_2[n];
        d.etaAB[n] = eab;
        if (d.wet_dry_on) d.mask_wd_node[n] = ((double)d.depth[n] + eab > d.Dmin_d) ? real(1.0) : real(0.0);
    }
}

// ---------------------------------------------------------------------------
// sub-step 1 (fv_main.F90:1451-1520): dmean_n, compute_puls_vel
// (fv_3D_vel.F90:257-307), one thread per (element, level).
// ---------------------------------------------------------------------------
__global__ void k_puls_elem(Dev d) {
    const long long total = (long long)d.E * d.L;
    GRID_LOOP(ii, total) {
        const int e = (int)(ii / d.L);
        const int4 en = d.elem_nodes[e];
        const real4 w = d.w_cv[e];
        const real dmn = dmax(d.Dmin, wexp(w, d.eta_n[en.x] + d.depth[en.x], d.eta_n[en.y] + d.depth[en.y],
                                              d.eta_n[en.z] + d.depth[en.z], d.eta_n[en.w] + d.depth[en.w]));
        const real a = dmn / dmax(d.Dmin, wsum(w, d.eta_new[en.x] + d.depth[en.x], d.eta_new[en.y] + d.depth[en.y],
                                                 d.eta_new[en.z] + d.depth[en.z], d.eta_new[en.w] + d.depth[en.w]));
        const real2 u2 = d.U_n_2D[e];
        d.U_puls[ii] = d.U_n[ii] - a * u2.x;
        d.V_puls[ii] = d.V_n[ii] - a * u2.y;
        if (ii % d.L == 0) d.dmean_n[e] = dmn;
    }
}

// compute_el2nodes_3D (fv_utilit.F90:644-700), one thread per (node, level)
__global__ void k_el2nodes(Dev d, const real *Ue, const real *Ve, real *Un, real *Vn) {
    const long long total = (long long)d.N * d.L;
    GRID_LOOP(ii, total) {
        const int n = (int)(ii / d.L);
        const int z = (int)(ii % d.L);
        const real tvol_inv = real(1.0) / d.node_tvol[n];
        real su = real(0.0), sv = real(0.0);
        for (int p = d.node_nptr[n]; p < d.node_nptr[n + 1]; ++p) {
            const int el = d.node_nidx[p];
            const real ar = d.elem_area[el];
            su = su + Ue[(size_t)el * d.L + z] * ar;
            sv = sv + Ve[(size_t)el * d.L + z] * ar;
        }
        Un[ii] = su * tvol_inv;
        Vn[ii] = sv * tvol_inv;
    }
}

// momentum_adv_P1_3D_to_2D (fv_advection.F90:676-793): the edge part
// uu*un, vv*un of every (internal edge, level), thread per (edge, level).
// Stored in the adv3 buffer, which velrhs has finished with.
__global__ void k_p1_edge(Dev d) {
    const long long total = (long long)d.Ed_in * d.L;
    const int L = d.L;
    GRID_LOOP(ii, total) {
        const int ed = (int)(ii / L);
        const int z = (int)(ii % L);
        const int2 nn = d.edge_nodes[ed];
        const int2 et = d.edge_tri[ed];
        const real2 dxy = d.edge_dxdy[ed];
        const real xe = dxy.x * kREarth * real(0.5) * (d.elem_cos[et.x] + d.elem_cos[et.y]);
        const real ye = dxy.y * kREarth;
        const real a1 = jac_a(d, d.eta_jac, nn.x), a2 = jac_a(d, d.eta_jac, nn.y);
        const real uu = real(0.5) * (d.Unode_p[(size_t)nn.x * L + z] + d.Unode_p[(size_t)nn.y * L + z]);
        const real vv = real(0.5) * (d.Vnode_p[(size_t)nn.x * L + z] + d.Vnode_p[(size_t)nn.y * L + z]);
        const real jd = real(0.5) * (jc_of(d, a1, z) + jc_of(d, a2, z));
        const real un = (uu * ye - vv * xe) * jd;
        d.adv3[ii] = make_real2(uu * un, vv * un);
    }
}

// Element part of momentum_adv_P1_3D_to_2D, optional
// viscosity_filt_3D_to_2D (fv_viscosity.F90:870-939) and
// biharmonic_viscosity_3D_to_2D, divided by dmean_n (fv_main.F90:1504-1513).
// A block takes B consecutive elements with one thread per (element, level)
// (coalesced column loads); every thread writes its level's terms of the
// element's edge slots and of the filter / biharmonic slots into shared
// memory, and the first threads of each element also stage its edge codes,
// the nodal factors acc of its edges and dmean_n.  Then, in the reference's
// order of operations: one thread per (element, edge slot, component) sums
// the slot over the levels in level order; one thread per (element,
// component) adds the slot sums in slot order and the filter and
// biharmonic terms level by level.
constexpr int kP1Slots = 5;  // 4 internal-edge slots + the filter
__global__ void k_p1_elem(Dev d) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const int L = d.L;
    const int B = (int)blockDim.x / L;
    const int nsl = kP1Slots + (d.bih_3D ? 1 : 0);  // + biharmonic_viscosity_3D_to_2D
    const int S = 2 * nsl * L + 1;  // per-element stride, odd: conflict-free
    real *sm = reinterpret_cast<real *>(sm_raw);
    real *sums = sm + (size_t)B * S;     // [B][8]: level sums of (slot, component)
    real *accs = sums + (size_t)B * 8;   // [B][4]: acc of the edge slots
    real *dms = accs + (size_t)B * 4;    // [B]: dmean_n
    int *cds = reinterpret_cast<int *>(dms + B);  // [B][4]: edge codes
    const int jl = (int)threadIdx.x / L, z = (int)threadIdx.x % L;
    const int nt = (int)blockDim.x;
    for (long long eb = (long long)blockIdx.x * B; eb < d.E; eb += (long long)gridDim.x * B) {
        const long long e_ = eb + jl;
        if (jl < B && e_ < d.E) {
            const int e = (int)e_;
            real *T = sm + (size_t)jl * S;  // T[(slot*2 + uv)*L + z]
            const real je = d.Je[(size_t)e * L + z];
            const int4 il = d.elem_iedges[e];
            const int codes[4] = {il.x, il.y, il.z, il.w};
            for (int c = z; c < 4; c += L) {
                const int code = c == 0 ? il.x : c == 1 ? il.y : c == 2 ? il.z : il.w;
                cds[jl * 4 + c] = code;
                if (code >= 0) {
                    const int2 nn = d.edge_nodes[code >> 1];
                    accs[jl * 4 + c] = (d.ac[nn.x] + d.ac[nn.y]) * real(.5);
                }
            }
            if (z == 0) dms[jl] = d.dmean_n[e];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if (codes[c] >= 0) {
                    const real2 pq = d.adv3[(size_t)(codes[c] >> 1) * L + z];
                    T[(c * 2 + 0) * L + z] = pq.x * je;
                    T[(c * 2 + 1) * L + z] = pq.y * je;
                }
            }
            if (d.filt_3D) {
                const int4 en = d.elem_nodes[e];
                const int4 nb4 = d.elem_nb[e];
                const int nbs[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
                const int jend = (en.x == en.w) ? 3 : 4;
                const real tau = d.tau_inv_filt, ar = d.elem_area[e];
                const real up = d.U_puls[(size_t)e * L + z], vp = d.V_puls[(size_t)e * L + z];
                real u1 = real(0.0), v1 = real(0.0);
                for (int k = 0; k < jend; ++k) {
                    const int ne = nbs[k];
                    if (ne < 0) continue;
                    const size_t i = (size_t)ne * L + z;
                    const real jn = d.Je[i];
                    u1 = u1 + d.U_puls[i] * jn - up * je;
                    v1 = v1 + d.V_puls[i] * jn - vp * je;
                }
                const real fu = tau * u1 * ar, fv = tau * v1 * ar;
                T[(4 * 2 + 0) * L + z] = fu * je;
                T[(4 * 2 + 1) * L + z] = fv * je;
            }
            if (d.bih_3D) {
                const real2 b = bih_gather(d, e, z);
                T[(5 * 2 + 0) * L + z] = b.x * je;
                T[(5 * 2 + 1) * L + z] = b.y * je;
            }
        }
        __syncthreads();
        // level sums of the edge slots, one thread per (element, slot, component)
        for (int t = (int)threadIdx.x; t < B * 8; t += nt) {
            const int j = t >> 3, ch = t & 7;
            if (eb + j < d.E && cds[j * 4 + (ch >> 1)] >= 0) {
                const real *T = sm + (size_t)j * S + (size_t)ch * L;
                real sl = real(0.0);
                for (int k = 0; k < L; ++k) sl = sl + T[k];
                sums[j * 8 + ch] = sl;
            }
        }
        __syncthreads();
        // one thread per (element, component)
        for (int t = (int)threadIdx.x; t < B * 2; t += nt) {
            const int j = t >> 1, uv = t & 1;
            const long long es = eb + j;
            if (es < d.E) {
                real r = real(0.0);
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int code = cds[j * 4 + c];
                    if (code < 0) break;
                    const real a = accs[j * 4 + c], sc = sums[j * 8 + c * 2 + uv];
                    if (code & 1) r = r + a * sc;
                    else r = r - a * sc;
                }
                const real *T = sm + (size_t)j * S;
                if (d.filt_3D)
                    for (int k = 0; k < L; ++k) r = r + T[(4 * 2 + uv) * L + k];
                if (d.bih_3D)
                    for (int k = 0; k < L; ++k) r = r + T[(5 * 2 + uv) * L + k];
                reinterpret_cast<real *>(d.U_rhs_2D_3D)[2 * es + uv] = r / dms[j];
            }
        }
        __syncthreads();
    }
}

// One upwind edge flux of momentum_adv_upwind_2D (fv_advection.F90:589-643)
__device__ __forceinline__ void adv2d_edge(const Dev &d, int ed, real &uu, real &vv) {
    const int2 nn = d.edge_nodes[ed];
    const int2 et = d.edge_tri[ed];
    const real dmean = (real)dmax(d.Dmin_d, 0.5 * ((d.etaAB[nn.x] + (double)d.depth[nn.x]) +
                                                    (d.etaAB[nn.y] + (double)d.depth[nn.y])));
    const real acc = (d.ac[nn.x] + d.ac[nn.y]) * real(0.5);
    const real4 X = d.edge_cross[ed];
    const real2 U1 = d.UAB[et.x], U2 = d.UAB[et.y];
    const real4 g1 = d.vel_grad[et.x], g2 = d.vel_grad[et.y];
    const real u1 = U1.x - g1.x * X.x - g1.y * X.y;
    const real v1 = U1.y - g1.z * X.x - g1.w * X.y;
    const real u2 = U2.x - g2.x * X.z - g2.y * X.w;
    const real v2 = U2.y - g2.z * X.z - g2.w * X.w;
    const real2 dxy = d.edge_dxdy[ed];
    const real un = real(0.5) * kREarth * dmean *
                      ((u1 + u2) * dxy.y - (v1 * d.elem_cos[et.x] + v2 * d.elem_cos[et.y]) * dxy.x);
    if (un >= real(0.0)) { uu = un * U1.x * acc; vv = un * U1.y * acc; }
    else { uu = un * U2.x * acc; vv = un * U2.y * acc; }
}

// momentum_adv_upwind_2D edge fluxes of the sub-step, once per internal edge
__global__ void k_adv2d_edge(Dev d) {
    GRID_LOOP(ed, d.Ed_in) {
        real uu, vv;
        adv2d_edge(d, (int)ed, uu, vv);
        d.adv2d[ed] = make_real2(uu, vv);
    }
}

// biharmonic_2D (fv_viscosity.F90:338-568, free slip): two Laplacians of the
// 2D velocity.  bih2d_edge: the flux of every edge from U and the gradients
// in vel_grad (boundary edges with the free-slip projection, whose v uses
// the projected u, as the reference); bih2d_ul: Ul = Ah acc sum of the
// fluxes; bih2d_grad: vel_gradients_2D(Ul) into vel_grad (adv2d_edge has
// used the gradients of UAB by then).  u2d_elem gathers the second pass.
__global__ void k_bih2d_edge(Dev d, const real2 *U) {
    GRID_LOOP(ii, d.Ed) {
        const int ed = (int)ii;
        const int2 et = d.edge_tri[ed];
        const real2 dxy = d.edge_dxdy[ed];
        real u1, v1;
        if (ed < d.Ed_in) {
            const real4 X = d.edge_cross[ed];
            const real xe = dxy.x * kREarth * real(0.5) * (d.elem_cos[et.x] + d.elem_cos[et.y]);
            const real ye = dxy.y * kREarth;
            real tx = -X.x + X.z;
            real ty = -X.y + X.w;
            const real tl = sqrt(tx * tx + ty * ty);
            tx = tx / tl;
            ty = ty / tl;
            const real4 a = d.vel_grad[et.x], b = d.vel_grad[et.y];
            const real2 U1 = U[et.x], U2 = U[et.y];
            real g1 = real(0.5) * (a.x + b.x);
            real g2 = real(0.5) * (a.y + b.y);
            real tt = g1 * tx + g2 * ty - (U2.x - U1.x) / tl;
            g1 = g1 - tx * tt;
            g2 = g2 - ty * tt;
            u1 = (g1 * ye - g2 * xe);
            g1 = real(0.5) * (a.z + b.z);
            g2 = real(0.5) * (a.w + b.w);
            tt = g1 * tx + g2 * ty - (U2.y - U1.y) / tl;
            g1 = g1 - tx * tt;
            g2 = g2 - ty * tt;
            v1 = (g1 * ye - g2 * xe);
        } else {
            const real xe = dxy.x * kREarth;
            const real xed = xe * d.elem_cos[et.x];
            const real ye = dxy.y * kREarth;
            const real4 a = d.vel_grad[et.x];
            u1 = (a.x) * ye - (a.y) * xed;
            v1 = (a.z) * ye - (a.w) * xed;
            u1 = ye * (u1 * ye - v1 * xe) / (xe * xe + ye * ye);
            v1 = -xe * (u1 * ye - v1 * xe) / (xe * xe + ye * ye);
        }
        d.b2fl[ed] = make_real2(u1, v1);
    }
}

__global__ void k_bih2d_ul(Dev d) {
    GRID_LOOP(ii, d.E) {
        const int e = (int)ii;
        const int4 se = d.elem_sedges[e];
        const int codes[4] = {se.x, se.y, se.z, se.w};
        real ux = real(0.0), uy = real(0.0);
        for (int c = 0; c < 4; ++c) {
            const int code = codes[c];
            if (code < 0) break;
            const real2 f = d.b2fl[code >> 1];
            if (code & 1) { ux = ux - f.x; uy = uy - f.y; }
            else { ux = ux + f.x; uy = uy + f.y; }
        }
        const real sa = scale_area_of(d, e);
        const real Ah = -d.Abh0 * sqrt(d.elem_area[e] / sa) / sa;
        const real acc = d.elem_acc[e];
        d.b2ul[e] = make_real2(ux * (Ah) * acc, uy * (Ah) * acc);
    }
}

// vel_gradients_2D (fv_gradients.F90:97-176, free slip) of U into vel_grad:
// of UAB after ab3_elem in every sub-step, of Ul in biharmonic_2D
__global__ void k_velgrad2d(Dev d, const real2 *U) {
    GRID_LOOP(ii, d.E) {
        const int e = (int)ii;
        const int4 en = d.elem_nodes[e];
        const int4 nb = d.elem_nb[e];
        const int4 ee = d.elem_edges[e];
        const int nbs[4] = {nb.x, nb.y, nb.z, nb.w};
        const int eds[4] = {ee.x, ee.y, ee.z, ee.w};
        const real4 gx = d.gv_x[e], gy = d.gv_y[e];
        const real gxa[4] = {gx.x, gx.y, gx.z, gx.w};
        const real gya[4] = {gy.x, gy.y, gy.z, gy.w};
        const int jend = (en.x == en.w) ? 3 : 4;
        const real2 u0 = U[e];
        real g1 = real(0.0), g2 = real(0.0), g3 = real(0.0), g4 = real(0.0);
        for (int j = 0; j < jend; ++j) {
            const int e2 = nbs[j];
            if (e2 >= 0) {
                const real2 u2 = U[e2];
                g1 = g1 + gxa[j] * (u2.x - u0.x);
                g2 = g2 + gya[j] * (u2.x - u0.x);
                g3 = g3 + gxa[j] * (u2.y - u0.y);
                g4 = g4 + gya[j] * (u2.y - u0.y);
            } else {
                const real2 dxy = d.edge_dxdy[eds[j]];
                const real zc1 = dxy.x * d.elem_cos[e];
                const real zc2 = dxy.y;
                const real un = -real(2.0) * (u0.x * zc2 - u0.y * zc1) / (zc1 * zc1 + zc2 * zc2);
                g1 = g1 + gxa[j] * un * zc2;
                g2 = g2 + gya[j] * un * zc2;
                g3 = g3 - gxa[j] * un * zc1;
                g4 = g4 - gya[j] * un * zc1;
            }
        }
        d.vel_grad[e] = make_real4(g1, g2, g3, g4);
    }
}

// viscosity_filt2x_2D (fv_viscosity.F90:672-767), first half: U_c of every
// element from the differences of U_n_2D with its neighbours, times K_bi;
// u2d_elem forms UV2_rhs from the neighbours' U_c.  Runs before u2d_elem,
// which rotates U_n_2D.
__global__ void k_filt2x_2d(Dev d) {
    const real tau_inv = d.dt_2D * d.tau_c / real(3600.0) / real(24.0);
    GRID_LOOP(ii, d.E) {
        const int e = (int)ii;
        const int4 nb = d.elem_nb[e];
        const int nbs[4] = {nb.x, nb.y, nb.z, nb.w};
        const real K_bi = tau_inv * sqrt(scale_area_of(d, e) / d.elem_area[e]);
        const real2 u0 = d.U_n_2D[e];
        real uc = real(0.0), vc = real(0.0);
        for (int j = 0; j < 4; ++j) {
            const int ne = nbs[j];
            if (!(ne >= 0 && (j < 3 || ne != nbs[0]))) continue;
            const real2 u2 = d.U_n_2D[ne];
            if (j == 0) { uc = u0.x - u2.x; vc = u0.y - u2.y; }
            else { uc = uc + u0.x - u2.x; vc = vc + u0.y - u2.y; }
        }
        d.f2uv2d[e] = make_real2(uc * K_bi, vc * K_bi);
    }
}

// ---------------------------------------------------------------------------
// u2d_elem: update_2D_vel (fv_average_dynamic.F90:228-443, type_task 3,
// key_atm off) + rotation of U time levels + U_filt accumulation
// (fv_main.F90:1568-1606).
// ---------------------------------------------------------------------------
// FP32: 8 resident blocks (at most 64 registers); FP64: 6.
__global__ void __launch_bounds__(128, FESOMC_FP32 ? 8 : 6) k_u2d_elem(Dev d) {
    const real d0inv = real(1.0) / d.density_0;
    GRID_LOOP(ii, d.E) {
        const int e = (int)ii;
        const int4 en = d.elem_nodes[e];
        const int nd[4] = {en.x, en.y, en.z, en.w};
        // elevations and total depths in FP64 (the elevation gradient and
        // the wet/dry test with them); the momentum terms in 'real'
        double eab[4], dep[4], etag[4];
        for (int k = 0; k < 4; ++k) {
            eab[k] = d.etaAB[nd[k]];
            dep[k] = d.depth[nd[k]];
            if (d.key_atm) {
                // with atmospheric forcing: E - P and the sea-level pressure
                // anomaly (fv_average_dynamic.F90:278-286)
                const double d0i = 1.0 / d.density_0_d;
                etag[k] = kG64 * ((double)d.atp1[nd[k]] * eab[k] - d.emp[nd[k]] * d0i -
                                  (double)d.atp2[nd[k]] * d.ssh_gp[nd[k]]) + (kPref - d.mslp[nd[k]]) * d0i;
            } else {
                etag[k] = kG64 * ((double)d.atp1[nd[k]] * eab[k] - (double)d.atp2[nd[k]] * d.ssh_gp[nd[k]]);
            }
        }
        real mwd = d.mask_wd[e];
        if (d.wet_dry_on) {
            const double dmin4 = dmin(dmin(dep[0], dep[1]), dmin(dep[2], dep[3]));
            const double emax4 = dmax(dmax(eab[0], eab[1]), dmax(eab[2], eab[3]));
            mwd = (dmin4 + emax4 > d.Dmin_d) ? real(1.0) : real(0.0);
            d.mask_wd[e] = mwd;
        }
        const real4 w = d.w_cv[e];
        const real ar = d.elem_area[e];
        const real dmean = (real)dmax(d.Dmin_d, wexp_d(w, eab[0] + dep[0], eab[1] + dep[1], eab[2] + dep[2], eab[3] + dep[3]));
        const real4 gx = d.gs_x[e], gy = d.gs_y[e];
        const real gex = (real)((double)gx.x * etag[0] + (double)gx.y * etag[1] + (double)gx.z * etag[2] + (double)gx.w * etag[3]);
        const real gey = (real)((double)gy.x * etag[0] + (double)gy.y * etag[1] + (double)gy.z * etag[2] + (double)gy.w * etag[3]);
        const real2 uab = d.UAB[e];
        const real cor = d.coriolis[e];
        real rx = ar * (-dmean * gex + uab.y * dmean * cor + d.taux[e] * d0inv);
        real ry = ar * (-dmean * gey - uab.x * dmean * cor + d.tauy[e] * d0inv);
        if (d.mom_adv_2D == 2) {
            const int4 il = d.elem_iedges[e];
            const int codes[4] = {il.x, il.y, il.z, il.w};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int code = codes[c];
                if (code < 0) break;
                const real2 f = d.adv2d[code >> 1];
                if (code & 1) { rx = rx + f.x; ry = ry + f.y; }
                else { rx = rx - f.x; ry = ry - f.y; }
            }
        }
        if (d.filt_2D) {
            const int4 nb = d.elem_nb[e];
            const int nbs[4] = {nb.x, nb.y, nb.z, nb.w};
            const int jend = (en.x == en.w) ? 3 : 4;
            real u1 = real(0.0), u2 = real(0.0);
            for (int j = 0; j < jend; ++j)
                if (nbs[j] >= 0) {
                    const real2 un = d.UAB[nbs[j]];
                    u1 = u1 + un.x - uab.x;
                    u2 = u2 + un.y - uab.y;
                }
            const real sd = (real)wsum_d(w, dep[0], dep[1], dep[2], dep[3]);
            rx = rx + d.tau_inv_filt * u1 * ar * sd;
            ry = ry + d.tau_inv_filt * u2 * ar * sd;
        }
        // biharmonic_2D: the second-pass edge fluxes in edge order
        if (d.bih_2D) {
            const int4 se = d.elem_sedges[e];
            const int codes[4] = {se.x, se.y, se.z, se.w};
            for (int c = 0; c < 4; ++c) {
                const int code = codes[c];
                if (code < 0) break;
                const real2 f = d.b2fl[code >> 1];
                if (code & 1) { rx = rx - f.x; ry = ry - f.y; }
                else { rx = rx + f.x; ry = ry + f.y; }
            }
        }
        const real2 r3 = d.U_rhs_2D_3D[e];
        rx = rx + r3.x;
        ry = ry + r3.y;
        // final update with implicit bottom drag
        double eo[4], enw[4];
        for (int k = 0; k < 4; ++k) { eo[k] = d.eta_n[nd[k]]; enw[k] = d.eta_new[nd[k]]; }
        const real dmo = (real)dmax(d.Dmin_d, wsum_d(w, eo[0] + dep[0], eo[1] + dep[1], eo[2] + dep[2], eo[3] + dep[3]));
        const real4 bf = d.bfric[e];
        const real ub = bf.x, vb = bf.y, friction = bf.z;
        const real ff = real(1.0) / ((real)dmax(d.Dmin_d, wsum_d(w, enw[0] + dep[0], enw[1] + dep[1], enw[2] + dep[2], enw[3] + dep[3]))
                                 + friction * d.dt_2D);
        const real dt2 = d.dt_2D;
        const real2 u0 = d.U_n_2D[e];
        const real2 bp = d.Bar_pr_2D[e];
        // UV2_rhs of viscosity_filt2x_2D (zero when it is off)
        real uvx = real(0.0), uvy = real(0.0);
        if (d.filt_bi_2D) {
            const int4 nb = d.elem_nb[e];
            const int nbs[4] = {nb.x, nb.y, nb.z, nb.w};
            const real2 c0 = d.f2uv2d[e];
            for (int j = 0; j < 4; ++j) {
                const int ne = nbs[j];
                if (!(ne >= 0 && (j < 3 || ne != nbs[0]))) continue;
                const real2 c2 = d.f2uv2d[ne];
                if (j == 0) { uvx = -c0.x + c2.x; uvy = -c0.y + c2.y; }
                else { uvx = uvx - c0.x + c2.x; uvy = uvy - c0.y + c2.y; }
            }
        }
        const real nx = mwd * ((dmo * u0.x - dt2 * friction * (ub - u0.x) + dt2 * bp.x + dt2 * rx / ar) * ff + uvx);
        const real ny = mwd * ((dmo * u0.y - dt2 * friction * (vb - u0.y) + dt2 * bp.y + dt2 * ry / ar) * ff + uvy);
        // rotate U_n_2 <- U_n_1 <- U_n_2D <- new (fv_main.F90:1569-1578)
        d.U_n_2[e] = d.U_n_1[e];
        d.U_n_1[e] = u0;
        d.U_n_2D[e] = make_real2(nx, ny);
        // U_filt accumulation with the new elevation (fv_main.F90:1596-1605)
        const real dmn = (real)dmax(d.Dmin_d, wexp_d(w, enw[0] + dep[0], enw[1] + dep[1], enw[2] + dep[2], enw[3] + dep[3]));
        d.U_filt_2D[e] = d.U_filt_2D[e] + nx * dmn;
        d.V_filt_2D[e] = d.V_filt_2D[e] + ny * dmn;
    }
}

// eta time-level rotation (fv_main.F90:1547-1551)
__global__ void k_rot_nodes(Dev d) {
    GRID_LOOP(ii, d.N) {
        const int n = (int)ii;
        const double e0 = d.eta_n[n], e1 = d.eta_n_1[n];
        d.eta_n_2[n] = e1;
        d.eta_n_1[n] = e0;
        d.eta_n[n] = d.eta_new[n];
    }
}

// U_filt_2D = V_filt_2D = 0 at the start of the sub-cycle, and the bottom
// velocity and quadratic drag a_Cd*|U_b| that update_2D_vel uses in every
// sub-step (fv_average_dynamic.F90:262, 400-420; U_n is fixed during the
// sub-cycle)
__global__ void k_zero_filt(Dev d) {
    GRID_LOOP(ii, d.E) {
        d.U_filt_2D[ii] = real(0.0);
        d.V_filt_2D[ii] = real(0.0);
        const real a_Cd = d.C_d * ((real(1.0) - d.elem_acc[ii]) * d.Cd_bz + real(1.0));
        const real ub = d.U_n[(size_t)ii * d.L + d.L - 1], vb = d.V_n[(size_t)ii * d.L + d.L - 1];
        d.bfric[ii] = make_real4(ub, vb, a_Cd * sqrt(ub * ub + vb * vb), real(0.0));
    }
}

// ---- launch wrappers --------------------------------------------------------
void launch_ab3_elem(const Dev &d, cudaStream_t s) {
    const int b1 = tuned(d, TK_AB3, 256), b2 = tuned(d, TK_VELGRAD2D, 256);
    k_ab3_elem<<<grid_for(d.E, b1), b1, 0, s>>>(d);
    k_velgrad2d<<<grid_for(d.E, b2), b2, 0, s>>>(d, d.UAB);
}
void launch_ssh_node(const Dev &d, int sub, cudaStream_t s) {
    const int b1 = tuned(d, TK_SSHEDGE, 256), b2 = tuned(d, TK_SSHNODE, 256);
    k_ssh_edge<<<grid_for(d.Ed, b1), b1, 0, s>>>(d);
    k_ssh_node<<<grid_for(d.N, b2), b2, 0, s>>>(d, sub);
}
void launch_puls_elem(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_PULS, 256);
    k_puls_elem<<<grid_for((long long)d.E * d.L, b), b, 0, s>>>(d);
}
void launch_el2nodes(const Dev &d, const real *Ue, const real *Ve, real *Un, real *Vn, cudaStream_t s) {
    const int b = tuned(d, TK_EL2NODES, 256);
    k_el2nodes<<<grid_for((long long)d.N * d.L, b), b, 0, s>>>(d, Ue, Ve, Un, Vn);
}
// B elements per block: B*L threads, at most 1024 and at most 32 elements;
// per element its slot tile, 8 slot sums, 4 acc, dmean_n and 4 edge codes
static int p1_elems(const Dev &d) { int b = 1024 / d.L; return b > 32 ? 32 : b; }
static size_t p1_smem(const Dev &d) {
    return (size_t)p1_elems(d) * ((2 * (kP1Slots + (d.bih_3D ? 1 : 0)) * d.L + 1 + 13) * sizeof(real) +
                                  4 * sizeof(int));
}
int config_p1(const Dev &d) {
    return raise_smem_limit(k_p1_elem, p1_smem(d)) == cudaSuccess
               ? 0 : 1;
}
void launch_p1_edge(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_P1EDGE, 256);
    k_p1_edge<<<grid_for((long long)d.Ed_in * d.L, b), b, 0, s>>>(d);
}
void launch_p1_elem(const Dev &d, cudaStream_t s) {
    const int B = p1_elems(d);
    const long long blocks = ((long long)d.E + B - 1) / B;
    k_p1_elem<<<(int)(blocks < 148LL * 16 ? blocks : 148LL * 16), B * d.L, p1_smem(d), s>>>(d);
}
void launch_adv2d_edge(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_ADV2D, 256);
    k_adv2d_edge<<<grid_for(d.Ed_in, b), b, 0, s>>>(d);
}
void launch_filt2x_2d(const Dev &d, cudaStream_t s) { k_filt2x_2d<<<grid_for(d.E, 256), 256, 0, s>>>(d); }
void launch_bih_2d(const Dev &d, cudaStream_t s) {
    k_bih2d_edge<<<grid_for(d.Ed, 256), 256, 0, s>>>(d, d.UAB);
    k_bih2d_ul<<<grid_for(d.E, 256), 256, 0, s>>>(d);
    k_velgrad2d<<<grid_for(d.E, 256), 256, 0, s>>>(d, d.b2ul);
    k_bih2d_edge<<<grid_for(d.Ed, 256), 256, 0, s>>>(d, d.b2ul);
}
void launch_u2d_elem(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_U2D, 128);
    k_u2d_elem<<<grid_for(d.E, b), b, 0, s>>>(d);
}
void launch_rot_nodes(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_ROT, 256);
    k_rot_nodes<<<grid_for(d.N, b), b, 0, s>>>(d);
}
void launch_zero_filt(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_ZEROFILT, 256);
    k_zero_filt<<<grid_for(d.E, b), b, 0, s>>>(d);
}


// Largest block (threads) each tunable kernel of this file can launch with
// (its registers and launch bounds): lim[knob] lowered to that.
static void tune_lower(int *lim, int knob, const void *k) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, k) == cudaSuccess && a.maxThreadsPerBlock < lim[knob]) lim[knob] = a.maxThreadsPerBlock;
}
void tune_limits_barotropic(int *lim) {
    tune_lower(lim, TK_AB3, (const void *)k_ab3_elem);
    tune_lower(lim, TK_VELGRAD2D, (const void *)k_velgrad2d);
    tune_lower(lim, TK_SSHEDGE, (const void *)k_ssh_edge);
    tune_lower(lim, TK_SSHNODE, (const void *)k_ssh_node);
    tune_lower(lim, TK_PULS, (const void *)k_puls_elem);
    tune_lower(lim, TK_EL2NODES, (const void *)k_el2nodes);
    tune_lower(lim, TK_P1EDGE, (const void *)k_p1_edge);
    tune_lower(lim, TK_ADV2D, (const void *)k_adv2d_edge);
    tune_lower(lim, TK_U2D, (const void *)k_u2d_elem);
    tune_lower(lim, TK_ROT, (const void *)k_rot_nodes);
    tune_lower(lim, TK_ZEROFILT, (const void *)k_zero_filt);
}

FESOMC_PREC_END
