// Internal-mode (baroclinic) kernels of oce_timestep case(3)
// (src/fv_main.F90:1983-2070):
//   pressure_col : densityJM + hydrostatic prefix sum per node column
//   bpg_elem     : baroclinic_pressure_gradient_3D per element column
//   velgrad3d    : vel_gradients (least squares, free slip) per (elem, level)
//   adv3_edge    : upwind horizontal momentum flux per (internal edge, level)
//   velrhs       : compute_vel_rhs up to the AB combine, per (elem, level):
//                  pressure force, Coriolis/AB2 history, the edge momentum
//                  fluxes gathered in edge order, filter viscosity, QUICK
//                  vertical advection
//   implvisc     : implicit vertical viscosity per element column
//                  (momentum_vert_impl_visc_tmp / momentum_vert_impl_visc)
//   update3d     : update_3D_vel per element column; stores the new Je, Ze, ZBe
//   wvel         : vert_vel_sigma per node column (edge gather + reverse scan)
//   jac_swap     : jacobian bookkeeping (eta at the previous / last call)
//   je_elem      : Je, Ze, ZBe at init
#include "device_common.cuh"

FESOMC_PREC_BEGIN

// Column blocks: B consecutive entities per block, one thread per (entity,
// level), levels on consecutive threads (coalesced column access).  Level
// sums / scans that the reference does sequentially go through shared memory
// (one row of L per entity, odd row stride) and are done by one thread per
// entity, in level order.
struct ColBlock {
    int L, B, jl, z;
    __device__ ColBlock(int L_) : L(L_), B((int)blockDim.x / L_), jl((int)threadIdx.x / L_), z((int)threadIdx.x % L_) {}
};

// ---------------------------------------------------------------------------
// pressure (fv_pressure_new.F90:91-107): density per (node, level), the
// hydrostatic sum per node in level order
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_pressure_col(Dev d) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    real *sm = reinterpret_cast<real *>(sm_raw);
    const real gd0 = kG / d.density_0;
    const int L = d.L, NS = d.NS;
    const ColBlock cb(L);
    const int S = L | 1;
    for (long long nb = (long long)blockIdx.x * cb.B; nb < d.N; nb += (long long)gridDim.x * cb.B) {
        const long long n_ = nb + cb.jl;
        const bool act = cb.jl < cb.B && n_ < d.N;
        if (act) {
            const int n = (int)n_;
            const real a = jac_a(d, d.eta_jac, n);
            const size_t i = (size_t)n * L + cb.z;
            const real rho = density_jm(d.TF[i], d.SF[i], -z_of(d, a, cb.z), d.density_0);
            d.rho_c[i] = rho;
            sm[cb.jl * S + cb.z] = rho * jc_of(d, a, cb.z) * gd0;
        }
        __syncthreads();
        if ((int)threadIdx.x < cb.B && nb + threadIdx.x < d.N) {
            real *row = sm + threadIdx.x * S;
            real hp = real(0.0);
            for (int k = 0; k < L; ++k) {
                hp = hp + row[k];
                row[k] = hp;
            }
        }
        __syncthreads();
        if (act) {
            const size_t bs = (size_t)n_ * NS;
            d.hpressure[bs + cb.z + 1] = sm[cb.jl * S + cb.z];
            if (cb.z == 0) d.hpressure[bs] = real(0.0);
        }
        __syncthreads();
    }
}

// baroclinic_pressure_gradient_3D (fv_pressure_new.F90:146-221) per
// (element, level); Bar_pr_2D as a level-ordered sum per element.  Also the
// element's surface pressure force of compute_vel_rhs (fv_3D_vel.F90:60-75),
// the same for every level.  Column blocks reach 1024 threads (B * L), so
// the kernel is bounded to 64 registers (unbounded it takes 96, which a
// block of more than 682 threads, i.e. L >= 43, could not launch with).
__global__ void __launch_bounds__(1024) k_bpg_elem(Dev d) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    real *sm = reinterpret_cast<real *>(sm_raw);
    const int L = d.L, NS = d.NS;
    const ColBlock cb(L);
    const int S = 2 * L + 1;
    for (long long eb = (long long)blockIdx.x * cb.B; eb < d.E; eb += (long long)gridDim.x * cb.B) {
        const long long e_ = eb + cb.jl;
        if (cb.jl < cb.B && e_ < d.E) {
            const int e = (int)e_, z = cb.z;
            const int4 en = d.elem_nodes[e];
            const int nd[4] = {en.x, en.y, en.z, en.w};
            const real4 gx = d.gs_x[e], gy = d.gs_y[e], w = d.w_cv[e];
            real dh[4], de[4];
            for (int k = 0; k < 4; ++k) { dh[k] = d.depth[nd[k]] + d.eta_n[nd[k]]; de[k] = d.depth[nd[k]]; }
            const real Ax = wsum(gx, dh[0], dh[1], dh[2], dh[3]);
            const real Ay = wsum(gy, dh[0], dh[1], dh[2], dh[3]);
            const real Bx = wsum(gx, de[0], de[1], de[2], de[3]);
            const real By = wsum(gy, de[0], de[1], de[2], de[3]);
            const real fac = d.elem_bpfac[e];
            const real4 ae = elem_jac_a(d, d.eta_jac, en);
            const real an[4] = {ae.x, ae.y, ae.z, ae.w};
            const real je = d.Je[(size_t)e * L + z];
            const real accJe_inv = -fac / je;
            real hu[4], hl[4], pre[4];
            for (int k = 0; k < 4; ++k) {
                hu[k] = d.hpressure[(size_t)nd[k] * NS + z];
                hl[k] = d.hpressure[(size_t)nd[k] * NS + z + 1];
                pre[k] = real(0.5) * (hu[k] + hl[k]) * jc_of(d, an[k], z);
            }
            const real qd_up = wsum(w, hu[0], hu[1], hu[2], hu[3]);
            const real qd_low = wsum(w, hl[0], hl[1], hl[2], hl[3]);
            const real sx = wsum(gx, pre[0], pre[1], pre[2], pre[3]);
            const real sy = wsum(gy, pre[0], pre[1], pre[2], pre[3]);
            const real s0 = __ldg(d.sig + z), s1 = __ldg(d.sig + z + 1);
            const real bu = accJe_inv * (sx + qd_low * (s1 * Ax - Bx) - qd_up * (s0 * Ax - Bx));
            const real bv = accJe_inv * (sy + qd_low * (s1 * Ay - By) - qd_up * (s0 * Ay - By));
            d.Bar_pru[(size_t)e * L + z] = bu;
            d.Bar_prv[(size_t)e * L + z] = bv;
            sm[cb.jl * S + z] = bu * je;
            sm[cb.jl * S + L + z] = bv * je;
            // surface pressure force of the element (independent of the
            // level sums): in this phase, off the serial path
            if (z == 0) {
                real pr[4];
                for (int k = 0; k < 4; ++k)
                    pr[k] = -kG * (d.atp1[nd[k]] * d.eta_n[nd[k]] - d.atp2[nd[k]] * d.ssh_gp[nd[k]]);
                if (d.key_atm) {
                    // sea-level pressure and E - P of the element (fv_3D_vel.F90:40-53)
                    const real d0i = real(1.0) / d.density_0;
                    const real atm_mean = wsum(w, (real)d.mslp[nd[0]], (real)d.mslp[nd[1]], (real)d.mslp[nd[2]],
                                               (real)d.mslp[nd[3]]);
                    const real emp_mean = wsum(w, (real)d.emp[nd[0]], (real)d.emp[nd[1]], (real)d.emp[nd[2]],
                                               (real)d.emp[nd[3]]);
                    for (int k = 0; k < 4; ++k)
                        pr[k] = pr[k] - (real(kPref) - atm_mean) * d0i + kG * emp_mean * d0i;
                }
                const real ar = d.elem_area[e];
                d.Fp[e] = make_real2(wsum(gx, pr[0], pr[1], pr[2], pr[3]) * ar, wsum(gy, pr[0], pr[1], pr[2], pr[3]) * ar);
            }
        }
        __syncthreads();
        const long long es = eb + threadIdx.x;
        if ((int)threadIdx.x < cb.B && es < d.E) {
            const int e = (int)es;
            const real *row = sm + threadIdx.x * S;
            real b1 = real(0.0), b2 = real(0.0);
            for (int k = 0; k < L; ++k) {
                b1 = b1 + row[k];
                b2 = b2 + row[L + k];
            }
            d.Bar_pr_2D[e] = make_real2(b1, b2);
        }
        __syncthreads();
    }
}

// vel_gradients (fv_gradients.F90:2-93), one thread per (element, level).
// 64 registers: 32 resident warps per SM instead of 24 (11 % faster).
__global__ void __maxnreg__(64) k_velgrad3d(Dev d) {
    const long long total = (long long)d.E * d.L;
    GRID_LOOP(ii, total) {
        const int e = (int)(ii / d.L);
        const int z = (int)(ii % d.L);
        const int L = d.L;
        const int4 en = d.elem_nodes[e];
        const int4 nb = d.elem_nb[e];
        const int4 ee = d.elem_edges[e];
        const int nbs[4] = {nb.x, nb.y, nb.z, nb.w};
        const int eds[4] = {ee.x, ee.y, ee.z, ee.w};
        const real4 gx = d.gv_x[e], gy = d.gv_y[e];
        const real gxa[4] = {gx.x, gx.y, gx.z, gx.w};
        const real gya[4] = {gy.x, gy.y, gy.z, gy.w};
        const int jend = (en.x == en.w) ? 3 : 4;
        const real u0 = d.U_n[ii], v0 = d.V_n[ii];
        real a1 = real(0.0), a2 = real(0.0), a3 = real(0.0), a4 = real(0.0);
        for (int j = 0; j < jend; ++j) {
            const int e2 = nbs[j];
            if (e2 >= 0) {
                const real u2 = d.U_n[(size_t)e2 * L + z], v2 = d.V_n[(size_t)e2 * L + z];
                a1 = a1 + gxa[j] * (u2 - u0);
                a2 = a2 + gya[j] * (u2 - u0);
                a3 = a3 + gxa[j] * (v2 - v0);
                a4 = a4 + gya[j] * (v2 - v0);
            } else {
                const real2 dxy = d.edge_dxdy[eds[j]];
                const real zc1 = dxy.x * d.elem_cos[e], zc2 = dxy.y;
                const real un = -real(2.0) * (u0 * zc2 - v0 * zc1) / (zc1 * zc1 + zc2 * zc2);
                a1 = a1 + gxa[j] * un * zc2;
                a2 = a2 + gya[j] * un * zc2;
                a3 = a3 - gxa[j] * un * zc1;
                a4 = a4 - gya[j] * un * zc1;
            }
        }
        d.vgux[ii] = a1;
        d.vguy[ii] = a2;
        d.vgvx[ii] = a3;
        d.vgvy[ii] = a4;
    }
}

// w-weighted element mean of a node column value: SUM(w_cv*X(k,nodes))
__device__ __forceinline__ real wsum_col(const real4 &w, const real *X, int stride, const int4 &en, int k) {
    return wsum(w, X[(size_t)en.x * stride + k], X[(size_t)en.y * stride + k], X[(size_t)en.z * stride + k],
                X[(size_t)en.w * stride + k]);
}
__device__ __forceinline__ real wsum_zbar(const Dev &d, const real4 &w, const real4 &a, int k) {
    return wsum(w, zbar_of(d, a.x, k), zbar_of(d, a.y, k), zbar_of(d, a.z, k), zbar_of(d, a.w, k));
}
__device__ __forceinline__ real wsum_z(const Dev &d, const real4 &w, const real4 &a, int k) {
    return wsum(w, z_of(d, a.x, k), z_of(d, a.y, k), z_of(d, a.z, k), z_of(d, a.w, k));
}

// Vertical momentum flux uvertAB(:,k) of momentum_vert_adv_upwind at interface
// k (0-based, 0..NS-1) of element e (fv_advection.F90:389-443); the element
// means of Z and zbar come from the stored Ze / ZBe.
__device__ __forceinline__ void uvert_at(const Dev &d, int e, int k, const real4 &w, const int4 &en, real ar,
                                         real &fu, real &fv) {
    const int L = d.L, NS = d.NS;
    const real *U = d.U_n + (size_t)e * L;
    const real *V = d.V_n + (size_t)e * L;
    if (k == NS - 1) { fu = real(0.0); fv = real(0.0); return; }
    const real wv = wsum_col(w, d.Wvel, NS, en, k) * ar;
    if (k == 0) { fu = -wv * U[0]; fv = -wv * V[0]; return; }
    const int nz = k + 1;  // 1-based interface index, 2..NS-1
    const real *ZE = d.Ze + (size_t)e * L;   // ZE[m-1] = SUM(w*Z(m))
    const real *ZB = d.ZBe + (size_t)e * L;  // ZB[m-1] = SUM(w*zbar(m))
    real umean = real(0.0), vmean = real(0.0);
    // U_n(m) 1-based  ->  U[m-1]
    if (wv >= real(0.0)) {
        if (nz == NS - 1) {
            umean = real(0.5) * (U[nz - 2] + U[nz - 1]);
            vmean = real(0.5) * (V[nz - 2] + V[nz - 1]);
        } else {
            const real Z1 = ZB[nz - 1];
            const real aa = Z1 - ZE[nz - 2];
            const real bb = ZE[nz - 1] - Z1;
            const real cc = ZE[nz] - Z1;
            const real dd = (cc + aa) * (bb * bb - aa * aa) - (cc * cc - aa * aa) * (bb + aa);
            const real dg = aa * bb * (aa + bb) / dd;
            const real db = -aa * cc * (aa + cc) / dd;
            const real da = real(1.0) - dg - db;
            umean = U[nz - 2] * da + U[nz - 1] * db + U[nz] * dg;
            vmean = V[nz - 2] * da + V[nz - 1] * db + V[nz] * dg;
        }
    }
    if (wv < real(0.0)) {
        if (nz == 2) {
            umean = real(0.5) * (U[nz - 2] + U[nz - 1]);
            vmean = real(0.5) * (V[nz - 2] + V[nz - 1]);
        } else {
            const real Z1 = ZB[nz - 1];
            const real aa = ZE[nz - 1] - Z1;
            const real bb = Z1 - ZE[nz - 2];
            const real cc = Z1 - ZE[nz - 3];
            const real dd = (cc + aa) * (bb * bb - aa * aa) - (cc * cc - aa * aa) * (bb + aa);
            const real dg = aa * bb * (aa + bb) / dd;
            const real db = -aa * cc * (aa + cc) / dd;
            const real da = real(1.0) - dg - db;
            umean = U[nz - 1] * da + U[nz - 2] * db + U[nz - 3] * dg;
            vmean = V[nz - 1] * da + V[nz - 2] * db + V[nz - 3] * dg;
        }
    }
    fu = -umean * wv;
    fv = -vmean * wv;
}

// Upwind horizontal momentum flux of one (internal edge, level)
// (momentum_adv_upwind, fv_advection.F90:114-188), computed once and gathered
// by the edge's two elements in velrhs.  Thread per (edge, level), levels on
// consecutive threads.
__global__ void k_adv3_edge(Dev d) {
    const long long total = (long long)d.Ed_in * d.L;
    const int L = d.L;
    GRID_LOOP(ii, total) {
        const int ed = (int)(ii / L);
        const int z = (int)(ii % L);
        const int2 nn = d.edge_nodes[ed];
        const int2 et = d.edge_tri[ed];
        const real acc = real(0.5) * (d.ac[nn.x] + d.ac[nn.y]);
        const real4 X = d.edge_cross[ed];
        const size_t i1 = (size_t)et.x * L + z, i2 = (size_t)et.y * L + z;
        const real u1 = d.U_n[i1] - d.vgux[i1] * X.x - d.vguy[i1] * X.y;
        const real v1 = d.V_n[i1] - d.vgvx[i1] * X.x - d.vgvy[i1] * X.y;
        const real u2 = d.U_n[i2] - d.vgux[i2] * X.z - d.vguy[i2] * X.w;
        const real v2 = d.V_n[i2] - d.vgvx[i2] * X.z - d.vgvy[i2] * X.w;
        const real jd = real(0.5) * (jc_of(d, jac_a(d, d.eta_jac, nn.x), z) + jc_of(d, jac_a(d, d.eta_jac, nn.y), z));
        const real2 dxy = d.edge_dxdy[ed];
        const real un = real(0.5) * kREarth * jd *
                          ((u1 + u2) * dxy.y - (v1 * d.elem_cos[et.x] + v2 * d.elem_cos[et.y]) * dxy.x);
        real uu, vv;
        if (un >= real(0.0)) { uu = u1 * un * acc; vv = v1 * un * acc; }
        else { uu = u2 * un * acc; vv = v2 * un * acc; }
        d.adv3[ii] = make_real2(uu, vv);
    }
}

// ---------------------------------------------------------------------------
// biharmonic_viscosity (fv_viscosity.F90:104-334) and its sub-step-1 twin
// biharmonic_viscosity_3D_to_2D (:964-1219): two Laplacians of a velocity,
// each an edge flux of the normal velocity gradient (the mean of the two
// elements' gradients with its tangential part replaced by the difference
// quotient), gathered per element in edge order (internal edges, then
// boundary edges).
// bih_edge: the flux of every (edge, level); mode 0 times Jd, mode 1 times
// Jd and the edge's sponge factor, mode 2 plain.
// bih_uc: U_c = Ah * sum of the mode-0 fluxes; Ah = -Abh0 sqrt(area/s)/s
// (mode 0), -acc Abh0 sqrt(area/s)/s (mode 1, the 3D-to-2D form; its Visc
// term is zero on this path, h_viscosity only runs with the sediment model).
// bih_grad: vel_lapl_gradients (fv_gradients.F90:327-402) of U_c into the
// velocity-gradient arrays.  velgrad_puls: vel_gradients_puls
// (fv_gradients.F90:404-496, free slip) of U_puls.
// velrhs gathers the mode-1 fluxes into U_rhs after the filter viscosity;
// p1_elem gathers the mode-2 fluxes, times Je, into U_rhs_2D_3D.
// ---------------------------------------------------------------------------
__global__ void k_bih_edge(Dev d, const real *U, const real *V, int mode) {
    const long long total = (long long)d.Ed * d.L;
    const int L = d.L;
    GRID_LOOP(ii, total) {
        const int ed = (int)(ii / L);
        const int z = (int)(ii % L);
        const int2 nn = d.edge_nodes[ed];
        const int2 et = d.edge_tri[ed];
        const real2 dxy = d.edge_dxdy[ed];
        const size_t i1 = (size_t)et.x * L + z;
        real u1, v1;
        if (ed < d.Ed_in) {
            const size_t i2 = (size_t)et.y * L + z;
            const real4 X = d.edge_cross[ed];
            const real xe = dxy.x * kREarth * real(0.5) * (d.elem_cos[et.x] + d.elem_cos[et.y]);
            const real ye = dxy.y * kREarth;
            real tx = -X.x + X.z;
            real ty = -X.y + X.w;
            const real tl = sqrt(tx * tx + ty * ty);
            tx = tx / tl;
            ty = ty / tl;
            real g1 = real(0.5) * (d.vgux[i1] + d.vgux[i2]);
            real g2 = real(0.5) * (d.vguy[i1] + d.vguy[i2]);
            real tt = g1 * tx + g2 * ty - (U[i2] - U[i1]) / tl;
            g1 = g1 - tx * tt;
            g2 = g2 - ty * tt;
            u1 = (g1 * ye - g2 * xe);
            g1 = real(0.5) * (d.vgvx[i1] + d.vgvx[i2]);
            g2 = real(0.5) * (d.vgvy[i1] + d.vgvy[i2]);
            tt = g1 * tx + g2 * ty - (V[i2] - V[i1]) / tl;
            g1 = g1 - tx * tt;
            g2 = g2 - ty * tt;
            v1 = (g1 * ye - g2 * xe);
        } else {
            const real xe = dxy.x * kREarth * d.elem_cos[et.x];
            const real ye = dxy.y * kREarth;
            u1 = (d.vgux[i1]) * ye - (d.vguy[i1]) * xe;
            v1 = (d.vgvx[i1]) * ye - (d.vgvy[i1]) * xe;
        }
        real fu = u1, fv = v1;
        if (mode != 2) {
            const real jd = real(0.5) * (jc_of(d, jac_a(d, d.eta_jac, nn.x), z) + jc_of(d, jac_a(d, d.eta_jac, nn.y), z));
            fu = u1 * jd;
            fv = v1 * jd;
            if (mode == 1) {
                const real acc = (d.ac[nn.x] + d.ac[nn.y]) / real(2.0);
                fu = fu * acc;
                fv = fv * acc;
            }
        }
        d.bihfl[ii] = make_real2(fu, fv);
    }
}

__global__ void k_bih_uc(Dev d, int mode) {
    const long long total = (long long)d.E * d.L;
    const int L = d.L;
    GRID_LOOP(ii, total) {
        const int e = (int)(ii / L);
        const int z = (int)(ii % L);
        const real2 c = bih_gather(d, e, z);
        const real sa = scale_area_of(d, e);
        const real Ah = (mode == 0) ? -d.Abh0 * sqrt(d.elem_area[e] / sa) / sa
                                    : -d.elem_acc[e] * d.Abh0 * sqrt(d.elem_area[e] / sa) / sa;
        d.bihU[ii] = c.x * (Ah);
        d.bihV[ii] = c.y * (Ah);
    }
}

// least-squares gradients of (U, V) per (element, level); the boundary
// neighbour is -2 U (vel_lapl_gradients) or the free-slip mirror
// (vel_gradients_puls)
template <bool FREE_SLIP>
__global__ void k_bih_grad(Dev d, const real *U, const real *V) {
    const long long total = (long long)d.E * d.L;
    const int L = d.L;
    GRID_LOOP(ii, total) {
        const int e = (int)(ii / L);
        const int z = (int)(ii % L);
        const int4 en = d.elem_nodes[e];
        const int4 nb = d.elem_nb[e];
        const int4 ee = d.elem_edges[e];
        const int nbs[4] = {nb.x, nb.y, nb.z, nb.w};
        const int eds[4] = {ee.x, ee.y, ee.z, ee.w};
        const real4 gx = d.gv_x[e], gy = d.gv_y[e];
        const real gxa[4] = {gx.x, gx.y, gx.z, gx.w};
        const real gya[4] = {gy.x, gy.y, gy.z, gy.w};
        const int jend = (en.x == en.w) ? 3 : 4;
        const real u0 = U[ii], v0 = V[ii];
        real a1 = real(0.0), a2 = real(0.0), a3 = real(0.0), a4 = real(0.0);
        for (int j = 0; j < jend; ++j) {
            const int e2 = nbs[j];
            real u, v;
            if (e2 >= 0) {
                u = U[(size_t)e2 * L + z] - u0;
                v = V[(size_t)e2 * L + z] - v0;
            } else if (FREE_SLIP) {
                const real2 dxy = d.edge_dxdy[eds[j]];
                const real zc1 = dxy.x * d.elem_cos[e], zc2 = dxy.y;
                const real un = -real(2.0) * (u0 * zc2 - v0 * zc1) / (zc1 * zc1 + zc2 * zc2);
                const real ua = u0 + un * zc2;
                const real va = v0 - un * zc1;
                u = ua - u0;
                v = va - v0;
            } else {
                u = -real(2.0) * u0;
                v = -real(2.0) * v0;
            }
            a1 = a1 + gxa[j] * u;
            a2 = a2 + gya[j] * u;
            a3 = a3 + gxa[j] * v;
            a4 = a4 + gya[j] * v;
        }
        d.vgux[ii] = a1;
        d.vguy[ii] = a2;
        d.vgvx[ii] = a3;
        d.vgvy[ii] = a4;
    }
}

// viscosity_filt2x_3D (fv_viscosity.F90:570-670), first half: U_c of every
// (element, level) from the differences of U*Je with its neighbours
// (neighbour 4 only when it differs from neighbour 1), times K_bi.  velrhs
// forms UV_rhs from the neighbours' U_c.
__global__ void k_filt2x_uc(Dev d) {
    const long long total = (long long)d.E * d.L;
    const int L = d.L;
    const real tau_inv = d.dt * d.tau_c / real(3600.0) / real(24.0);
    GRID_LOOP(ii, total) {
        const int e = (int)(ii / L);
        const int z = (int)(ii % L);
        const int4 nb = d.elem_nb[e];
        const int nbs[4] = {nb.x, nb.y, nb.z, nb.w};
        const real K_bi = tau_inv * sqrt(scale_area_of(d, e) / d.elem_area[e]);
        const real uj = d.U_n[ii] * d.Je[ii], vj = d.V_n[ii] * d.Je[ii];
        real uc = real(0.0), vc = real(0.0);
        for (int j = 0; j < 4; ++j) {
            const int ne = nbs[j];
            if (!(ne >= 0 && (j < 3 || ne != nbs[0]))) continue;
            const size_t i2 = (size_t)ne * L + z;
            if (j == 0) {
                uc = uj - d.U_n[i2] * d.Je[i2];
                vc = vj - d.V_n[i2] * d.Je[i2];
            } else {
                uc = uc + uj - d.U_n[i2] * d.Je[i2];
                vc = vc + vj - d.V_n[i2] * d.Je[i2];
            }
        }
        d.f2U[ii] = uc * K_bi;
        d.f2V[ii] = vc * K_bi;
    }
}

// ---------------------------------------------------------------------------
// velrhs: compute_vel_rhs (fv_3D_vel.F90:1-180), one thread per (element,
// level) with levels on consecutive lanes.  Each warp takes 31 outputs and
// its lane 31 forms the vertical flux at its own index, the interface below
// lane 30's layer, so the flux at interface z+1 comes from the next lane
// for every output and no lane forms a second flux.
// ff = 1 on the very first call (lfirst), 1.5+epsilon afterwards.
// (Sharing the fluxes across the block through shared memory was measured
// 16 % slower than recomputing them: the block-wide barrier costs more.)
// ---------------------------------------------------------------------------
// 4 resident blocks (at most 64 registers) in both forms: in FP64 the few
// spilled registers cost less than the lost warps (11 % faster than 3
// blocks at 80 registers).
__global__ void __launch_bounds__(256, 4) k_velrhs(Dev d, real ff) {
    const long long total = (long long)d.E * d.L;
    const int lane = threadIdx.x & 31;
    const long long nwarp = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c * 31 < total; c += nwarp) {
        const long long iw = c * 31 + lane;
        const bool valid = lane < 31 && iw < total;
        const long long ii = iw < total ? iw : total - 1;
        const int e = (int)(ii / d.L);
        const int z = (int)(ii % d.L);
        const int L = d.L;
        const int4 en = d.elem_nodes[e];
        const real4 w = d.w_cv[e];
        const real ar = d.elem_area[e];
        const real je = d.Je[ii];
        // pressure force from eta_n (per element, from bpg_elem)
        const real2 F = d.Fp[e];
        const real Fx = F.x, Fy = F.y;
        const real un0 = d.U_n[ii], vn0 = d.V_n[ii];
        real ur = -(real(0.5) + d.epsilon) * d.U_rhsAB[ii] + Fx * je;
        real vr = -(real(0.5) + d.epsilon) * d.V_rhsAB[ii] + Fy * je;
        const real cor = d.coriolis[e];
        real uab = vn0 * cor * ar * je;
        real vab = -un0 * cor * ar * je;
        // horizontal upwind momentum advection (fv_advection.F90:114-188):
        // edge fluxes in edge order
        if (d.mom_adv_3D == 1) {
            const int4 il = d.elem_iedges[e];
            const int codes[4] = {il.x, il.y, il.z, il.w};
            for (int c = 0; c < 4; ++c) {
                const int code = codes[c];
                if (code < 0) break;
                const real2 f = d.adv3[(size_t)(code >> 1) * L + z];
                if (code & 1) { uab = uab + f.x; vab = vab + f.y; }
                else { uab = uab - f.x; vab = vab - f.y; }
            }
        }
        // filter viscosity (fv_viscosity.F90:842-860)
        if (d.filt_3D) {
            const int4 nb = d.elem_nb[e];
            const int nbs[4] = {nb.x, nb.y, nb.z, nb.w};
            const int jend = (en.x == en.w) ? 3 : 4;
            real u1 = real(0.0), v1 = real(0.0);
            for (int j = 0; j < jend; ++j)
                if (nbs[j] >= 0) {
                    u1 = u1 + d.U_n[(size_t)nbs[j] * L + z] - un0;
                    v1 = v1 + d.V_n[(size_t)nbs[j] * L + z] - vn0;
                }
            ur = ur + d.tau_inv_filt * u1 * ar * je;
            vr = vr + d.tau_inv_filt * v1 * ar * je;
        }
        // biharmonic viscosity (fv_viscosity.F90:248-330): the pass-2 edge
        // fluxes in edge order, internal edges then boundary edges
        if (d.bih_3D) {
            const int4 se = d.elem_sedges[e];
            const int codes[4] = {se.x, se.y, se.z, se.w};
            for (int c = 0; c < 4; ++c) {
                const int code = codes[c];
                if (code < 0) break;
                const real2 f = d.bihfl[(size_t)(code >> 1) * L + z];
                if (code & 1) { ur = ur - f.x; vr = vr - f.y; }
                else { ur = ur + f.x; vr = vr + f.y; }
            }
        }
        // vertical advection (fv_advection.F90:354-469): flux at interface z
        // here, at z+1 from the next lane (same element) or computed
        const real mwd = d.mask_wd[e];
        if (d.vert_adv == 1) {
            real fu0, fv0;
            uvert_at(d, e, z, w, en, ar, fu0, fv0);
            real fu1 = __shfl_down_sync(kFull, fu0, 1), fv1 = __shfl_down_sync(kFull, fv0, 1);
            if (z == L - 1) { fu1 = real(0.0); fv1 = real(0.0); }   // the bottom interface carries no flux
            if (mwd != real(0.0)) {
                const real acc = d.elem_acc[e];
                uab = uab + (fu0 - fu1) * acc;
                vab = vab + (fv0 - fv1) * acc;
            } else {
                uab = real(0.0);
                vab = real(0.0);
            }
        }
        if (valid) {
            d.U_rhsAB[ii] = uab;
            d.V_rhsAB[ii] = vab;
            const real area_inv = real(1.0) / ar;
            const real dt = d.dt;
            // UV_rhs of viscosity_filt2x_3D (zero when it is off)
            real uvx = real(0.0), uvy = real(0.0);
            if (d.filt_bi_3D) {
                const int4 nb = d.elem_nb[e];
                const int nbs[4] = {nb.x, nb.y, nb.z, nb.w};
                const real uc = d.f2U[ii], vc = d.f2V[ii];
                for (int j = 0; j < 4; ++j) {
                    const int ne = nbs[j];
                    if (!(ne >= 0 && (j < 3 || ne != nbs[0]))) continue;
                    const size_t i2 = (size_t)ne * L + z;
                    if (j == 0) { uvx = -uc + d.f2U[i2]; uvy = -vc + d.f2V[i2]; }
                    else { uvx = uvx - uc + d.f2U[i2]; uvy = uvy - vc + d.f2V[i2]; }
                }
            }
            d.U_rhs[ii] = mwd * (un0 + d.Bar_pru[ii] * dt + (dt * (ur + uab * ff) * area_inv + uvx) / je);
            d.V_rhs[ii] = mwd * (vn0 + d.Bar_prv[ii] * dt + (dt * (vr + vab * ff) * area_inv + uvy) / je);
        }
    }
}

// ---------------------------------------------------------------------------
// implvisc: momentum_vert_impl_visc_tmp (fv_viscosity.F90:1374-1486, no ice)
// or momentum_vert_impl_visc (fv_viscosity.F90:1266-1371); thread per column.
// ---------------------------------------------------------------------------
template <int MAXL>
__global__ void k_implvisc(Dev d) {
    GRID_LOOP(ii, d.E) {
        const int e = (int)ii;
        const int L = d.L, NS = d.NS;
        real *ur = d.U_rhs + (size_t)e * L;
        real *vr = d.V_rhs + (size_t)e * L;
        const real *Av = d.Av + (size_t)e * NS;
        const real mwd = d.mask_wd[e];
        const real dt = d.dt;
        const real ub = d.U_n[(size_t)e * L + L - 1], vb = d.V_n[(size_t)e * L + L - 1];
        const real a_Cd = d.C_d * ((real(1.0) - d.elem_acc[e]) * d.Cd_bz + real(1.0));
        const real *je = d.Je + (size_t)e * L;
        if (d.im_vert_visc) {
            real a[MAXL], b[MAXL], c[MAXL], cp[MAXL], up[MAXL], vp[MAXL], uu[MAXL], vv[MAXL];
            const real *zc = d.Ze + (size_t)e * L;
            for (int z = 1; z <= L - 2; ++z) {
                const real zinv = dt / je[z];
                a[z] = -Av[z] / (zc[z] - zc[z - 1]) * zinv;
                c[z] = -Av[z + 1] / (zc[z + 1] - zc[z]) * zinv;
                b[z] = -a[z] - c[z] + real(1.0);
            }
            real zinv = dt / je[L - 1];
            a[L - 1] = -Av[L - 1] / (zc[L - 1] - zc[L - 2]) * zinv;
            b[L - 1] = -a[L - 1] + real(1.0);
            c[L - 1] = real(0.0);
            zinv = dt / je[0];
            c[0] = -Av[1] / (zc[1] - zc[0]) * zinv;
            a[0] = real(0.0);
            b[0] = -c[0] + real(1.0);
            for (int z = 0; z < L; ++z) { uu[z] = ur[z]; vv[z] = vr[z]; }
            uu[0] = uu[0] + zinv * d.taux[e] / d.density_0;
            vv[0] = vv[0] + zinv * d.tauy[e] / d.density_0;
            zinv = dt / je[L - 1];
            const real friction = -a_Cd * sqrt(ub * ub + vb * vb);
            uu[L - 1] = uu[L - 1] + zinv * friction * ub;
            vv[L - 1] = vv[L - 1] + zinv * friction * vb;
            // the recurrences carry their last value in registers
            real cpv = c[0] / b[0], upv = uu[0] / b[0], vpv = vv[0] / b[0];
            cp[0] = cpv;
            up[0] = upv;
            vp[0] = vpv;
            for (int z = 1; z < L; ++z) {
                const real az = a[z];
                const real m = b[z] - cpv * az;
                cpv = c[z] / m;
                upv = (uu[z] - upv * az) / m;
                vpv = (vv[z] - vpv * az) / m;
                cp[z] = cpv;
                up[z] = upv;
                vp[z] = vpv;
            }
            real un = upv, vn = vpv;
            uu[L - 1] = un;
            vv[L - 1] = vn;
            for (int z = L - 2; z >= 0; --z) {
                un = up[z] - cp[z] * un;
                vn = vp[z] - cp[z] * vn;
                uu[z] = un;
                vv[z] = vn;
            }
            for (int z = 0; z < L; ++z) { ur[z] = uu[z] * mwd; vr[z] = vv[z] * mwd; }
        }
        if (d.im_vert_visc_fic) {
            if (mwd != real(0.0)) {
                real xx1[MAXL + 2], yu[MAXL + 2], yv[MAXL + 2];
                xx1[0] = real(1.0);
                real de = je[0] / (Av[0] + Av[1]);
                const real rw = de / d.density_0;
                yu[0] = d.taux[e] * rw;
                yv[0] = d.tauy[e] * rw;
                // the recurrences carry their last value in registers; the
                // column values of the next level are loaded one level ahead
                real xv = xx1[0], yuv = yu[0], yvv = yv[0];
                real je_m = real(0.0), je_0 = je[0], je_p = L > 1 ? je[1] : real(0.0);
                real av_0 = Av[0], av_p = Av[1];
                real fx_n = ur[0], fy_n = vr[0];
                for (int z = 0; z < L; ++z) {
                    const real Fx = fx_n, Fy = fy_n;
                    const real jz = je_0, jm = je_m, jp = je_p, a0 = av_0, a1 = av_p;
                    if (z + 1 < L) {
                        fx_n = ur[z + 1];
                        fy_n = vr[z + 1];
                        je_m = je_0;
                        je_0 = je_p;
                        if (z + 2 < L) je_p = je[z + 2];
                        av_0 = av_p;
                        av_p = Av[z + 2];
                    }
                    const real d1 = (z == 0) ? real(0.5) * jz : real(0.5) * (jz + jm);
                    const real d2 = (z == L - 1) ? real(0.5) * jz : real(0.5) * (jz + jp);
                    const real zt = dt / jz;
                    const real a = zt * a0 / d1;
                    const real c = zt * a1 / d2;
                    const real b = a + c + real(1.0);
                    const real dd = b - a * xv;
                    xv = c / dd;
                    yuv = (a * yuv + Fx) / dd;
                    yvv = (a * yvv + Fy) / dd;
                    xx1[z + 1] = xv;
                    yu[z + 1] = yuv;
                    yv[z + 1] = yvv;
                }
                de = je[L - 1] / (Av[NS - 1] + Av[L - 1]);
                const real friction = de * a_Cd * sqrt(ub * ub + vb * vb);
                real Ut, Vt;
                if (d.fic_point == 0) { Ut = real(0.0); Vt = real(0.0); }
                else if (d.fic_point == 1) {
                    const real a = friction + real(1.0) - xx1[L];
                    Ut = yu[L] / a; Vt = yv[L] / a;
                } else {
                    const real a = real(1.0) / (real(1.0) - friction) - xx1[L];
                    Ut = yu[L] / a; Vt = yv[L] / a;
                }
                for (int z = L - 1; z >= 0; --z) {
                    Ut = Ut * xx1[z + 1] + yu[z + 1];
                    Vt = Vt * xx1[z + 1] + yv[z + 1];
                    ur[z] = Ut * mwd;
                    vr[z] = Vt * mwd;
                }
            } else {
                for (int z = 0; z < L; ++z) { ur[z] = real(0.0); vr[z] = real(0.0); }
            }
        }
    }
}

// jacobian bookkeeping after the sub-cycle (fv_main.F90:2050): Jc_old <- Jc
__global__ void k_jac_swap(Dev d) {
    GRID_LOOP(ii, d.N) {
        d.eta_jac_old[ii] = d.eta_jac[ii];
        d.eta_jac[ii] = d.eta_n[ii];
    }
}

// Je, Ze, ZBe of every (element, level) from eta_jac (jacobian,
// fv_main.F90:1208-1267); at init, afterwards refreshed by update3d
__global__ void k_je_elem(Dev d) {
    const long long total = (long long)d.E * d.L;
    GRID_LOOP(ii, total) {
        const int e = (int)(ii / d.L);
        const int z = (int)(ii % d.L);
        const real4 w = d.w_cv[e];
        const real4 a = elem_jac_a(d, d.eta_jac, d.elem_nodes[e]);
        d.Je[ii] = je_of(d, w, a, z);
        d.Ze[ii] = wsum_z(d, w, a, z);
        d.ZBe[ii] = wsum_zbar(d, w, a, z);
    }
}

// update_3D_vel (fv_3D_vel.F90:201-255) with the U_filt averaging of
// oce_barotropic_timestep (fv_main.F90:1670-1677) folded in; column block
// per element.  Runs right after the jacobian call: the stored Je still holds
// the previous jacobian (Jc_old), and is replaced here by the new Je / Ze /
// ZBe.
constexpr int kU3Sc = 14;  // per element: U2p, V2p, uf, vf, w_cv(4), a(4), U_n_2D(2)
// 48 registers: 4 resident column blocks per SM instead of 3 (15 % faster).
__global__ void __maxnreg__(48) k_update3d(Dev d, real Mt_inv) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    real *sm = reinterpret_cast<real *>(sm_raw);
    const int L = d.L;
    const ColBlock cb(L);
    const int S = 2 * L + 1;
    real *sc = sm + (size_t)cb.B * S;  // kU3Sc scalars per element
    for (long long eb = (long long)blockIdx.x * cb.B; eb < d.E; eb += (long long)gridDim.x * cb.B) {
        const long long e_ = eb + cb.jl;
        const bool act = cb.jl < cb.B && e_ < d.E;
        const size_t i = (size_t)e_ * L + cb.z;
        real a_old = real(0.0), ur = real(0.0), vr = real(0.0);
        if (act) {
            a_old = d.Je[i];
            ur = d.U_rhs[i];
            vr = d.V_rhs[i];
            sm[cb.jl * S + cb.z] = ur * a_old;
            sm[cb.jl * S + L + cb.z] = vr * a_old;
            // the element's scalars, here rather than in the serial sum or
            // the level loop, so that both read shared memory only
            if (cb.z == 0) {
                const int e = (int)e_;
                const int4 en = d.elem_nodes[e];
                const real4 w = d.w_cv[e];
                const real dmean_inv = real(1.0) / dmax(d.Dmin, wsum(w, d.depth[en.x] + d.eta_n[en.x], d.depth[en.y] + d.eta_n[en.y],
                                                                d.depth[en.z] + d.eta_n[en.z], d.depth[en.w] + d.eta_n[en.w]));
                const real uf = (d.U_filt_2D[e] * Mt_inv) * dmean_inv;
                const real vf = (d.V_filt_2D[e] * Mt_inv) * dmean_inv;
                d.U_filt_2D[e] = uf;
                d.V_filt_2D[e] = vf;
                const real4 an = elem_jac_a(d, d.eta_jac, en);
                const real2 u2d = d.U_n_2D[e];
                real *o = sc + kU3Sc * cb.jl;
                o[0] = dmean_inv;
                o[2] = uf; o[3] = vf;
                o[4] = w.x; o[5] = w.y; o[6] = w.z; o[7] = w.w;
                o[8] = an.x; o[9] = an.y; o[10] = an.z; o[11] = an.w;
                o[12] = u2d.x; o[13] = u2d.y;
            }
        }
        __syncthreads();
        const long long es = eb + threadIdx.x;
        if ((int)threadIdx.x < cb.B && es < d.E) {
            const real *row = sm + threadIdx.x * S;
            real su = real(0.0), sv = real(0.0);
            for (int k = 0; k < L; ++k) {
                su = su + row[k];
                sv = sv + row[L + k];
            }
            real *o = sc + kU3Sc * threadIdx.x;
            const real dmean_inv = o[0];
            o[0] = su * dmean_inv;
            o[1] = sv * dmean_inv;
        }
        __syncthreads();
        if (act) {
            const int z = cb.z;
            const real *o = sc + kU3Sc * cb.jl;
            const real U2p = o[0], V2p = o[1], uf = o[2], vf = o[3];
            const real4 w = make_real4(o[4], o[5], o[6], o[7]);
            const real4 an = make_real4(o[8], o[9], o[10], o[11]);
            const real jn = je_of(d, w, an, z);
            const real az = a_old / jn;
            d.U_n_filt[i] = az * ur + uf - U2p;
            d.V_n_filt[i] = az * vr + vf - V2p;
            d.U_n[i] = az * ur + o[12] - U2p;
            d.V_n[i] = az * vr + o[13] - V2p;
            d.Je[i] = jn;
            d.Ze[i] = wsum_z(d, w, an, z);
            d.ZBe[i] = wsum_zbar(d, w, an, z);
        }
        __syncthreads();
    }
}

// vert_vel_sigma (fv_3D_vel.F90:309-456): column block per node; the layer
// transport divergence of (node, level) gathered over the node's edges in
// edge order, then summed upward from the bottom per node.
__global__ void k_wvel(Dev d) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    real *sm = reinterpret_cast<real *>(sm_raw);
    const int L = d.L, NS = d.NS;
    const ColBlock cb(L);
    const int S = L | 1;
    real *sc = sm + (size_t)cb.B * S;  // per node: bottom Wvel, 1/area
    for (long long nb = (long long)blockIdx.x * cb.B; nb < d.N; nb += (long long)gridDim.x * cb.B) {
        const long long n_ = nb + cb.jl;
        const bool act = cb.jl < cb.B && n_ < d.N;
        if (act) {
            const int n = (int)n_, z = cb.z;
            if (z == 0) {
                sc[2 * cb.jl] = d.Wvel[(size_t)n * NS + NS - 1];
                sc[2 * cb.jl + 1] = real(1.0) / d.area[n];
            }
            const int p0 = d.node_eptr[n], p1 = d.node_eptr[n + 1];
            real W = real(0.0);
#pragma unroll 4
            for (int p = p0; p < p1; ++p) {
                const int code = d.node_eidx[p];
                const int ed = code >> 1;
                const int2 et = d.edge_tri[ed];
                const real4 X = d.edge_cross[ed];
                const real uf1 = d.U_filt_2D[et.x], vf1 = d.V_filt_2D[et.x];
                const size_t i1 = (size_t)et.x * L + z;
                real c1 = d.Je[i1] * ((d.V_n_filt[i1] - vf1) * X.x - (d.U_n_filt[i1] - uf1) * X.y);
                if (ed < d.Ed_in) {
                    const real uf2 = d.U_filt_2D[et.y], vf2 = d.V_filt_2D[et.y];
                    const size_t i2 = (size_t)et.y * L + z;
                    c1 = c1 + d.Je[i2] * (-(d.V_n_filt[i2] - vf2) * X.z + (d.U_n_filt[i2] - uf2) * X.w);
                }
                if (code & 1) W = W - c1;
                else W = W + c1;
            }
            sm[cb.jl * S + z] = W;
        }
        __syncthreads();
        const long long ns = nb + threadIdx.x;
        if ((int)threadIdx.x < cb.B && ns < d.N) {
            real *row = sm + threadIdx.x * S;
            real below = sc[2 * threadIdx.x];
            for (int k = L - 1; k >= 0; --k) {
                below = row[k] + below;
                row[k] = below;
            }
        }
        __syncthreads();
        if (act) d.Wvel[(size_t)n_ * NS + cb.z] = sm[cb.jl * S + cb.z] * sc[2 * cb.jl + 1];
        __syncthreads();
    }
}

// ---- momentum_vert_impl_visc_tmp on tiles of element columns --------------
// (launch-shape knob "implvisc_form" 2, the default for 10 and 20 layers):
// a block takes kIvCols consecutive elements, whose columns are one
// contiguous range of U_rhs, V_rhs, Je and Av, stages them in shared memory
// with coalesced loads (kIvBatch per thread in flight), solves each column
// with one thread from shared memory (odd row strides: no bank conflicts),
// the recurrences in registers (LC layers fixed at compile time), writes the
// result over the staged U_rhs / V_rhs and stores it coalesced.  The
// arithmetic and its order are k_implvisc's im_vert_visc_fic branch.
constexpr int kIvCols = 64;
constexpr int kIvBatch = 4;
__host__ __device__ __forceinline__ int iv_odd(int x) { return x | 1; }

template <int LC>
__global__ void __launch_bounds__(kIvCols) k_implvisc_fic_tile(Dev d) {
    extern __shared__ __align__(16) unsigned char iv_smem[];
    constexpr int L = LC, LP = LC | 1;
    const int NS = d.NS, KP = iv_odd(d.NS), E = d.E;
    real *sU = reinterpret_cast<real *>(iv_smem);   // row j: element e0 + j
    real *sV = sU + kIvCols * LP;
    real *sJ = sV + kIvCols * LP;
    real *sA = sJ + kIvCols * LP;                   // Av, stride KP
    const real dt = d.dt;
    for (long long e0 = (long long)blockIdx.x * kIvCols; e0 < E; e0 += (long long)gridDim.x * kIvCols) {
        const int nt = (int)(E - e0 < kIvCols ? E - e0 : kIvCols);
        for (int i0 = threadIdx.x; i0 < nt * NS; i0 += kIvBatch * kIvCols) {
            real av[kIvBatch];
#pragma unroll
            for (int u = 0; u < kIvBatch; ++u) {
                const int i = i0 + u * kIvCols;
                av[u] = i < nt * NS ? d.Av[(size_t)e0 * NS + i] : real(0.0);
            }
#pragma unroll
            for (int u = 0; u < kIvBatch; ++u) {
                const int i = i0 + u * kIvCols, j = i / NS;
                if (i < nt * NS) sA[j * KP + (i - j * NS)] = av[u];
            }
        }
        for (int i0 = threadIdx.x; i0 < nt * L; i0 += kIvBatch * kIvCols) {
            real ur[kIvBatch], vr[kIvBatch], jv[kIvBatch];
#pragma unroll
            for (int u = 0; u < kIvBatch; ++u) {
                const int i = i0 + u * kIvCols;
                const size_t g = (size_t)e0 * L + (i < nt * L ? i : 0);
                ur[u] = d.U_rhs[g];
                vr[u] = d.V_rhs[g];
                jv[u] = d.Je[g];
            }
#pragma unroll
            for (int u = 0; u < kIvBatch; ++u) {
                const int i = i0 + u * kIvCols;
                if (i >= nt * L) continue;
                const int j = i / L, z = i - j * L;
                sU[j * LP + z] = ur[u];
                sV[j * LP + z] = vr[u];
                sJ[j * LP + z] = jv[u];
            }
        }
        __syncthreads();
        if ((int)threadIdx.x < nt) {
            const int j = threadIdx.x, e = (int)e0 + j;
            real *U = sU + j * LP, *V = sV + j * LP;
            const real *J = sJ + j * LP, *A = sA + j * KP;
            const real mwd = d.mask_wd[e];
            if (mwd != real(0.0)) {
                const real ub = d.U_n[(size_t)e * L + L - 1], vb = d.V_n[(size_t)e * L + L - 1];
                const real a_Cd = d.C_d * ((real(1.0) - d.elem_acc[e]) * d.Cd_bz + real(1.0));
                real xx1[LC + 1], yu[LC + 1], yv[LC + 1];
                real de = J[0] / (A[0] + A[1]);
                const real rw = de / d.density_0;
                real xv = real(1.0), yuv = d.taux[e] * rw, yvv = d.tauy[e] * rw;
                xx1[0] = xv;
                yu[0] = yuv;
                yv[0] = yvv;
#pragma unroll
                for (int z = 0; z < L; ++z) {
                    const real jz = J[z];
                    const real d1 = (z == 0) ? real(0.5) * jz : real(0.5) * (jz + J[z > 0 ? z - 1 : 0]);
                    const real d2 = (z == L - 1) ? real(0.5) * jz : real(0.5) * (jz + J[z + 1 < L ? z + 1 : z]);
                    const real zt = dt / jz;
                    const real a = zt * A[z] / d1;
                    const real c = zt * A[z + 1] / d2;
                    const real b = a + c + real(1.0);
                    const real dd = b - a * xv;
                    xv = c / dd;
                    yuv = (a * yuv + U[z]) / dd;
                    yvv = (a * yvv + V[z]) / dd;
                    xx1[z + 1] = xv;
                    yu[z + 1] = yuv;
                    yv[z + 1] = yvv;
                }
                de = J[L - 1] / (A[NS - 1] + A[L - 1]);
                const real friction = de * a_Cd * sqrt(ub * ub + vb * vb);
                real Ut, Vt;
                if (d.fic_point == 0) { Ut = real(0.0); Vt = real(0.0); }
                else if (d.fic_point == 1) {
                    const real a = friction + real(1.0) - xx1[L];
                    Ut = yu[L] / a; Vt = yv[L] / a;
                } else {
                    const real a = real(1.0) / (real(1.0) - friction) - xx1[L];
                    Ut = yu[L] / a; Vt = yv[L] / a;
                }
#pragma unroll
                for (int z = L - 1; z >= 0; --z) {
                    Ut = Ut * xx1[z + 1] + yu[z + 1];
                    Vt = Vt * xx1[z + 1] + yv[z + 1];
                    U[z] = Ut * mwd;
                    V[z] = Vt * mwd;
                }
            } else {
#pragma unroll
                for (int z = 0; z < L; ++z) { U[z] = real(0.0); V[z] = real(0.0); }
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nt * L; i += kIvCols) {
            const int j = i / L, z = i - j * L;
            const size_t g = (size_t)e0 * L + i;
            d.U_rhs[g] = sU[j * LP + z];
            d.V_rhs[g] = sV[j * LP + z];
        }
        __syncthreads();
    }
}
static size_t implvisc_tile_smem(const Dev &d) {
    return (size_t)kIvCols * (3 * iv_odd(d.L) + iv_odd(d.NS)) * sizeof(real);
}
// the tiled form: the fic variant alone, 10 or 20 layers
static bool implvisc_tiled(const Dev &d) {
    return d.tune[TK_IMPLVISC] != 1 && !d.im_vert_visc && d.im_vert_visc_fic && (d.L == 10 || d.L == 20);
}

// ---- launch wrappers --------------------------------------------------------
// column blocks: B = min(16, 1024 / L) entities, B * L threads
static int col_b(const Dev &d) {
    if (d.tune[TK_COLUMNS] > 0) return d.tune[TK_COLUMNS];
    int b = 1024 / d.L;
    return b > 16 ? 16 : b;
}
static int col_grid(const Dev &d, long long count) {
    const long long blocks = (count + col_b(d) - 1) / col_b(d);
    return (int)(blocks < 148LL * 8 ? blocks : 148LL * 8);
}
static size_t col_smem(const Dev &d, int rows, int scalars) {
    const int S = rows == 1 ? (d.L | 1) : rows * d.L + 1;
    return ((size_t)col_b(d) * S + (size_t)col_b(d) * scalars) * sizeof(real);
}
int config_columns(const Dev &d) {
    const size_t big = col_smem(d, 2, kU3Sc);
    cudaError_t e = cudaSuccess;
    if (d.L == 10) e = raise_smem_limit(k_implvisc_fic_tile<10>, implvisc_tile_smem(d));
    if (d.L == 20) e = raise_smem_limit(k_implvisc_fic_tile<20>, implvisc_tile_smem(d));
    if (e == cudaSuccess) e = raise_smem_limit(k_bpg_elem, big);
    if (e == cudaSuccess) e = raise_smem_limit(k_update3d, big);
    if (e == cudaSuccess) e = raise_smem_limit(k_pressure_col, big);
    if (e == cudaSuccess) e = raise_smem_limit(k_wvel, big);
    return e == cudaSuccess ? 0 : 1;
}
void launch_pressure_col(const Dev &d, cudaStream_t s) {
    k_pressure_col<<<col_grid(d, d.N), col_b(d) * d.L, col_smem(d, 1, 0), s>>>(d);
}
void launch_bpg_elem(const Dev &d, cudaStream_t s) {
    k_bpg_elem<<<col_grid(d, d.E), col_b(d) * d.L, col_smem(d, 2, 0), s>>>(d);
}
void launch_velgrad3d(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_VELGRAD3D, 256);
    k_velgrad3d<<<grid_for((long long)d.E * d.L, b), b, 0, s>>>(d);
}
void launch_adv3_edge(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_ADV3, 256);
    k_adv3_edge<<<grid_for((long long)d.Ed_in * d.L, b), b, 0, s>>>(d);
}
void launch_filt2x(const Dev &d, cudaStream_t s) {
    k_filt2x_uc<<<grid_for((long long)d.E * d.L, 256), 256, 0, s>>>(d);
}
void launch_bih(const Dev &d, cudaStream_t s) {
    const int ge = grid_for((long long)d.Ed * d.L, 256), gl = grid_for((long long)d.E * d.L, 256);
    k_bih_edge<<<ge, 256, 0, s>>>(d, d.U_n, d.V_n, 0);
    k_bih_uc<<<gl, 256, 0, s>>>(d, 0);
    k_bih_grad<false><<<gl, 256, 0, s>>>(d, d.bihU, d.bihV);
    k_bih_edge<<<ge, 256, 0, s>>>(d, d.bihU, d.bihV, 1);
}
void launch_bih_puls(const Dev &d, cudaStream_t s) {
    const int ge = grid_for((long long)d.Ed * d.L, 256), gl = grid_for((long long)d.E * d.L, 256);
    k_bih_grad<true><<<gl, 256, 0, s>>>(d, d.U_puls, d.V_puls);
    k_bih_edge<<<ge, 256, 0, s>>>(d, d.U_puls, d.V_puls, 0);
    k_bih_uc<<<gl, 256, 0, s>>>(d, 1);
    k_bih_grad<false><<<gl, 256, 0, s>>>(d, d.bihU, d.bihV);
    k_bih_edge<<<ge, 256, 0, s>>>(d, d.bihU, d.bihV, 2);
}
void launch_velrhs(const Dev &d, real ff, cudaStream_t s) {
    const int b = tuned(d, TK_VELRHS, 256);
    k_velrhs<<<grid_for((long long)d.E * d.L, b), b, 0, s>>>(d, ff);
}
#define MAXL_DISPATCH(KERNEL, GRID, BLOCK, STREAM, ...)                                   \
    do {                                                                                   \
        if (d.L <= 24) KERNEL<24><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__);                \
        else if (d.L <= 48) KERNEL<48><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__);           \
        else KERNEL<128><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__);                         \
    } while (0)
void launch_implvisc(const Dev &d, cudaStream_t s) {
    if (implvisc_tiled(d)) {
        const long long tiles = ((long long)d.E + kIvCols - 1) / kIvCols;
        const int g = (int)(tiles < (1LL << 30) ? tiles : (1LL << 30));
        if (d.L == 10) k_implvisc_fic_tile<10><<<g, kIvCols, implvisc_tile_smem(d), s>>>(d);
        else k_implvisc_fic_tile<20><<<g, kIvCols, implvisc_tile_smem(d), s>>>(d);
        return;
    }
    MAXL_DISPATCH(k_implvisc, grid_for(d.E, 128), 128, s, d);
}
void launch_jac_swap(const Dev &d, cudaStream_t s) { k_jac_swap<<<grid_for(d.N, 256), 256, 0, s>>>(d); }
void launch_je(const Dev &d, cudaStream_t s) { k_je_elem<<<grid_for((long long)d.E * d.L, 256), 256, 0, s>>>(d); }
void launch_update3d(const Dev &d, real Mt_inv, cudaStream_t s) {
    k_update3d<<<col_grid(d, d.E), col_b(d) * d.L, col_smem(d, 2, kU3Sc), s>>>(d, Mt_inv);
}
void launch_wvel(const Dev &d, cudaStream_t s) { k_wvel<<<col_grid(d, d.N), col_b(d) * d.L, col_smem(d, 1, 2), s>>>(d); }


// Largest block (threads) each tunable kernel of this file can launch with
// (its registers and launch bounds): lim[knob] lowered to that.
static void tune_lower(int *lim, int knob, const void *k) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, k) == cudaSuccess && a.maxThreadsPerBlock < lim[knob]) lim[knob] = a.maxThreadsPerBlock;
}
void tune_limits_baroclinic(int *lim) {
    tune_lower(lim, TK_VELRHS, (const void *)k_velrhs);
    tune_lower(lim, TK_VELGRAD3D, (const void *)k_velgrad3d);
    tune_lower(lim, TK_ADV3, (const void *)k_adv3_edge);
}

FESOMC_PREC_END
