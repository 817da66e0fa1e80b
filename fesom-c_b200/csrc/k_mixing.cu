// Vertical turbulence closure d3_end (src/fv_mixing.F90:73-347): one thread
// per node column.  Each column iterates its implicit turbulence-energy
// sweep up to 200 times (relative tolerance 1e-6); columns that reach the cap
// are counted in the device status (the reference silently continues).
// Compute / latency bound (FP64 divisions, log, sqrt).
#include "device_common.cuh"

FESOMC_PREC_BEGIN

// Convergence test of d3_end's sweep (fv_mixing.F90:250-259) for one level:
// the reference forms c = |a/b| and stops when the largest c is below 1e-6
// (a NaN c never raises the maximum).  Returns true when this level forbids
// convergence, i.e. when RN(|a|/|b|) >= 1e-6.  The quotient is only formed
// when |a| lies within a relative 2^-30 of 1e-6*|b|; outside that band the
// comparison of |a| with the product decides it with certainty (the band is
// far wider than the rounding of the product and of the quotient).
__device__ __forceinline__ bool d3_above_tol(real a, real b) {
    const real aa = fabs(a), bb = fabs(b);
    if (bb > real(1.0e-290) && bb < real(1.0e290) && aa < real(1.0e300)) {
        const real t = real(1.0e-6) * bb;
        if (aa <= t * (real(1.0) - 0x1p-30)) return false;
        if (aa >= t * (real(1.0) + 0x1p-30)) return true;
    }
    return fabs(a / b) >= real(1.0e-6);
}

// d3_end per node column (local-memory arrays indexed 1..NS like the Fortran
// ones, ARR >= NS + 1 entries each).  The kernel is bound by the traffic of
// those arrays: the working set of the resident columns does not fit in L2,
// so each iteration streams them through DRAM.  It therefore keeps the
// array count and the accesses per level low:
//   * -b1-b2, t_inv*bo and c2 are formed once per level; am and cm are
//     recomputed in each iteration from snu(k-1..k+1) held in registers (the
//     reference recomputes them the same way);
//   * xx1(k), yy1(k) feed the next level from registers, the arrays only
//     carry them to the back substitution;
//   * btr and btr1 alternate between two arrays instead of being copied;
//   * tke_dissip, which the reference overwrites in every iteration, is
//     written once from the btr of the last iteration;
//   * the convergence test forms the quotient only near the threshold;
//   * both sweeps load the next level's array values one level ahead, so
//     that their latency overlaps the current level's division chain (3 %
//     faster; unrolling by 4 instead was 9 % slower).
// (The same arrays in shared memory, [array][level][thread], take the DRAM
// traffic down to the algorithmic bytes but leave room for 6 warps per SM
// only, and the kernel then waits on its FP64 chains: 3.85 against 2.54 ms
// on cfg1.)
//
// kList: the columns are list[0 .. *count) instead of every node (the
// columns the learned closure hands back to the plain one).
template <int ARR, bool kList>
__global__ void k_d3end(Dev d, const int *list, const unsigned long long *count) {
    const real t_inv = real(1.0) / d.dt;
    const real cka = d.cka;
    const real B1cka2 = real(16.6) * (cka * cka);
    const long long ncol = kList ? (long long)*count : (long long)d.N;
    GRID_LOOP(ii, ncol) {
        const int node = kList ? list[ii] : (int)ii;
        const int NS = d.NS, L = d.L;
        const real *bt = d.bt + (size_t)node * NS;
        const real *snu = d.snu + (size_t)node * NS;
        const real *Kv = d.Kv + (size_t)node * NS;
        const real *Un = d.Unode + (size_t)node * L;
        const real *Vn = d.Vnode + (size_t)node * L;
        const real *T = d.TF + (size_t)node * L;
        const real *S = d.SF + (size_t)node * L;
        real *Ri = d.Ri + (size_t)node * NS;
        real *tke = d.tke_dissip + (size_t)node * NS;
        real xx1[ARR], yy1[ARR], bA[ARR], bB[ARR], pb[ARR], qb[ARR], c2[ARR], sn[ARR];
        const real dmean = dmax<real>(d.Dmin, d.depth[node] + d.eta_n[node]);
        const real dmean2 = dmean * dmean;
        const real ajac = jac_a(d, d.eta_jac, node);
        for (int nz = 1; nz <= NS; ++nz) {
            bA[nz] = bt[nz - 1];
            sn[nz] = snu[nz - 1];
        }
        Ri[0] = real(0.0);
        Ri[NS - 1] = real(0.0);
        for (int nz = 2; nz <= NS - 1; ++nz) {
            const real s_m = __ldg(d.sig + nz - 2), s_0 = __ldg(d.sig + nz - 1), s_p = __ldg(d.sig + nz);
            const real d1 = s_m - s_0;
            const real d2 = s_0 - s_p;
            const real dd = real(0.5) * (d1 + d2);
            real ap1 = Un[nz - 2] - Un[nz - 1];
            const real ap2 = Vn[nz - 2] - Vn[nz - 1];
            real b1 = sn[nz] * (ap1 * ap1 + ap2 * ap2) / (dd * dd);
            b1 = b1 / dmean2;
            const real zb = zbar_of(d, ajac, nz - 1);
            const real rho_up = density_jm(T[nz - 2], S[nz - 2], -zb, d.density_0);
            const real rho_dn = density_jm(T[nz - 1], S[nz - 1], -zb, d.density_0);
            ap1 = (rho_up - rho_dn) / dd;
            const real b2 = -real(0.5) * kG * Kv[nz - 1] * ap1 / (d.density_0 * dmean);
            const real snu_p = real(0.5) * (sn[nz - 1] + sn[nz]);
            const real snu_m = real(0.5) * (sn[nz] + sn[nz + 1]);
            const real cc = real(0.5) * real(0.73) * (snu_p * (bt[nz - 2] - bt[nz - 1]) / d1 - snu_m * (bt[nz - 1] - bt[nz]) / d2) / dd;
            c2[nz] = cc / dmean2;
            if (b1 > real(0.0)) Ri[nz - 1] = -kG * ap1 / (d.density_0 * dmean) / b1 * sn[nz];
            else Ri[nz - 1] = real(10000.0);
            pb[nz] = -b1 - b2;
            qb[nz] = t_inv * bt[nz - 1];
        }
        real y2;
        {
            const real d1 = real(0.5) * (__ldg(d.sig + NS - 2) - __ldg(d.sig + NS - 1));
            const real wx = d.windx[node], wy = d.windy[node];
            const real u_din_sur = real(0.05) * (wx * wx + wy * wy);
            const real snu_m = real(0.5) * (sn[NS] + sn[NS - 1]);
            y2 = (real(0.4e-3) * (u_din_sur * u_din_sur * u_din_sur) * dmean * d1) / (snu_m * real(0.76));
        }
        xx1[2] = real(1.0);
        yy1[2] = y2;
        // bottom boundary value (independent of the iteration)
        const real delta_b = jc_of(d, ajac, NS - 2) + d.z0b_min;
        const real lg = fesomc_log(delta_b / d.z0b_min);
        const real bott_R = B1cka2 / (lg * lg);
        const real ubt = Un[L - 1], vbt = Vn[L - 1];
        const real bot = bott_R * (ubt * ubt + vbt * vbt);
        real *btr = bA, *btr1 = bB;
        bool converged = false;
        int iters = 200;
        for (int it = 1; it <= 200; ++it) {
            real x = real(1.0), y = y2;
            real s_lo = sn[1], s_mid = sn[2];
            real b_n = btr[2], pb_n = pb[2], qb_n = qb[2], c2_n = c2[2], sh_n = sn[3];
            for (int nz = 2; nz <= NS - 1; ++nz) {
                const real s_hi = sh_n;
                const real b = b_n, pbv = pb_n, qbv = qb_n, c2v = c2_n;
                if (nz + 1 <= NS - 1) {
                    b_n = btr[nz + 1]; pb_n = pb[nz + 1]; qb_n = qb[nz + 1]; c2_n = c2[nz + 1]; sh_n = sn[nz + 2];
                }
                const real s_m = __ldg(d.sig + nz - 2), s_0 = __ldg(d.sig + nz - 1), s_p = __ldg(d.sig + nz);
                const real dd1 = s_m - s_0;
                const real dd2 = s_0 - s_p;
                const real dd = real(0.5) * (dd1 + dd2);
                const real c1 = real(0.046) * (b * b) / s_mid;
                if (it == 200) tke[nz - 1] = c1;
                const real fr = pbv - c1 - qbv - c2v;
                const real snu_p = real(0.5) * (s_lo + s_mid);
                const real snu_mm = real(0.5) * (s_mid + s_hi);
                const real am = real(0.5) * (snu_p * real(0.73)) / (dmean2 * dd1 * dd);
                const real cm = real(0.5) * (snu_mm * real(0.73)) / (dmean2 * dd2 * dd);
                const real bm = am + cm + (real(2.0) * real(0.046) * b) / s_mid + t_inv;
                const real a = bm - am * x;
                const real xn = cm / a;
                const real yn = (am * y - fr) / a;
                xx1[nz + 1] = xn;
                yy1[nz + 1] = yn;
                x = xn;
                y = yn;
                s_lo = s_mid;
                s_mid = s_hi;
            }
            real b1v = bot;  // btr1(NS)
            btr1[NS] = b1v;
            bool above = d3_above_tol(btr[NS] - b1v, dmax(b1v, btr[NS]) + real(1.0e-8));
            real x_n = xx1[NS], y_n = yy1[NS], o_n = btr[NS - 1];
            for (int nz = NS; nz >= 2; --nz) {
                const real xv = x_n, yv = y_n, ov = o_n;
                if (nz - 1 >= 2) { x_n = xx1[nz - 1]; y_n = yy1[nz - 1]; o_n = btr[nz - 2]; }
                b1v = b1v * xv + yv;  // btr1(nz-1)
                btr1[nz - 1] = b1v;
                above |= d3_above_tol(ov - b1v, dmax(b1v, ov) + real(1.0e-8));
            }
            if (!above) { converged = true; iters = it; break; }
            real *t = btr;
            btr = btr1;
            btr1 = t;
        }
        if (d.d3_iters) d.d3_iters[node] = iters;   // measurement only (fesomc_gpu_d3end_iterations)
        if (converged) {
            for (int nz = 2; nz <= NS - 1; ++nz) tke[nz - 1] = real(0.046) * (btr[nz] * btr[nz]) / sn[nz];
        } else {
            atomicAdd(d.notconv, 1);
        }
        real *btw = d.bt + (size_t)node * NS;
        real *snw = d.snu + (size_t)node * NS;
        real *Kvw = d.Kv + (size_t)node * NS;
        for (int nz = 1; nz <= NS; ++nz) {
            const real btn = dmax(btr[nz], real(1.0e-8));
            btw[nz - 1] = btn;
            const real zt = __ldg(d.sig + nz - 1) * dmean;
            const real Zh = zt + d.z0b_min;
            const real Zd = fabs(dmean - zt) + d.z0s_min;
            const real Z0 = real(1.0) - d.beta_scale * Zh * Zd / (dmean * dmean);
            const real scale_t = cka * Zh * Zd * Z0 / dmean;
            real s = scale_t * sqrt(btn) + d.snul;
            if (s >= real(0.2)) s = real(0.2);
            snw[nz - 1] = s;
            Kvw[nz - 1] = d.Pr_num * s;
        }
    }
}

// The same closure with the column arrays in shared memory, laid out
// [array][level][thread] so that a warp's access to one level is 32
// consecutive words (launch-shape knob "d3end_arrays" = 2):
//   sn        snu(nz), nz = 1..NS                 (constant over the iteration)
//   bA, bB    btr / btr1 / xx1, nz = 1..NS        (alternating; the back
//             substitution writes btr1(k) into the xx1(k) slot it has just
//             read, xx1(2) = 1 and yy1(2) = y2 being constants)
//   yy1       yy1(nz), nz = 3..NS
//   pb, qb, c2  -b1-b2, t_inv*bt and c2, nz = 2..NS-1 (constant)
// i.e. 7*NS - 8 values per column: its DRAM traffic is the algorithmic
// bytes, but only 6 warps of 32 columns fit an SM, so the set-up and final
// level loops are unrolled for independent work per thread.  The same
// arithmetic as k_d3end, in the same order.
constexpr int kD3Block = 32;

__host__ __device__ inline int d3end_values(int NS) { return 7 * NS - 8; }

template <bool kList>
__global__ void __launch_bounds__(kD3Block, 6) k_d3end_sm(Dev d, const int *list, const unsigned long long *count) {
    extern __shared__ unsigned char d3_smem[];
    constexpr int B = kD3Block;
    const int NS = d.NS, L = d.L;
    real *const base = reinterpret_cast<real *>(d3_smem) + threadIdx.x;
    // per-array views: element nz of an array at [(nz - first) * B]
    real *const s_sn = base - 1 * B;                     // nz = 1..NS
    real *const s_bA = base + (NS - 1) * B;              // nz = 1..NS
    real *const s_bB = base + (2 * NS - 1) * B;          // nz = 1..NS
    real *const s_yy = base + (3 * NS - 3) * B;          // nz = 3..NS
    real *const s_pb = base + (4 * NS - 4) * B;          // nz = 2..NS-1
    real *const s_qb = base + (5 * NS - 6) * B;          // nz = 2..NS-1
    real *const s_c2 = base + (6 * NS - 8) * B;          // nz = 2..NS-1
#define D3(a, nz) a[(size_t)(nz) * B]
    const real t_inv = real(1.0) / d.dt;
    const real cka = d.cka;
    const real B1cka2 = real(16.6) * (cka * cka);
    const long long ncol = kList ? (long long)*count : (long long)d.N;
    GRID_LOOP(ii, ncol) {
        const int node = kList ? list[ii] : (int)ii;
        const real *bt = d.bt + (size_t)node * NS;
        const real *snu = d.snu + (size_t)node * NS;
        const real *Kv = d.Kv + (size_t)node * NS;
        const real *Un = d.Unode + (size_t)node * L;
        const real *Vn = d.Vnode + (size_t)node * L;
        const real *T = d.TF + (size_t)node * L;
        const real *S = d.SF + (size_t)node * L;
        real *Ri = d.Ri + (size_t)node * NS;
        real *tke = d.tke_dissip + (size_t)node * NS;
        const real dmean = dmax<real>(d.Dmin, d.depth[node] + d.eta_n[node]);
        const real dmean2 = dmean * dmean;
        const real ajac = jac_a(d, d.eta_jac, node);
        for (int nz = 1; nz <= NS; ++nz) {
            D3(s_bA, nz) = bt[nz - 1];
            D3(s_sn, nz) = snu[nz - 1];
        }
        Ri[0] = real(0.0);
        Ri[NS - 1] = real(0.0);
#pragma unroll 4
        for (int nz = 2; nz <= NS - 1; ++nz) {
            const real s_m = __ldg(d.sig + nz - 2), s_0 = __ldg(d.sig + nz - 1), s_p = __ldg(d.sig + nz);
            const real d1 = s_m - s_0;
            const real d2 = s_0 - s_p;
            const real dd = real(0.5) * (d1 + d2);
            real ap1 = Un[nz - 2] - Un[nz - 1];
            const real ap2 = Vn[nz - 2] - Vn[nz - 1];
            const real sn_m = snu[nz - 2], sn_0 = snu[nz - 1], sn_p = snu[nz];
            real b1 = sn_0 * (ap1 * ap1 + ap2 * ap2) / (dd * dd);
            b1 = b1 / dmean2;
            const real zb = zbar_of(d, ajac, nz - 1);
            const real rho_up = density_jm(T[nz - 2], S[nz - 2], -zb, d.density_0);
            const real rho_dn = density_jm(T[nz - 1], S[nz - 1], -zb, d.density_0);
            ap1 = (rho_up - rho_dn) / dd;
            const real b2 = -real(0.5) * kG * Kv[nz - 1] * ap1 / (d.density_0 * dmean);
            const real snu_p = real(0.5) * (sn_m + sn_0);
            const real snu_m = real(0.5) * (sn_0 + sn_p);
            const real cc = real(0.5) * real(0.73) * (snu_p * (bt[nz - 2] - bt[nz - 1]) / d1 - snu_m * (bt[nz - 1] - bt[nz]) / d2) / dd;
            D3(s_c2, nz) = cc / dmean2;
            if (b1 > real(0.0)) Ri[nz - 1] = -kG * ap1 / (d.density_0 * dmean) / b1 * sn_0;
            else Ri[nz - 1] = real(10000.0);
            D3(s_pb, nz) = -b1 - b2;
            D3(s_qb, nz) = t_inv * bt[nz - 1];
        }
        real y2;
        {
            const real d1 = real(0.5) * (__ldg(d.sig + NS - 2) - __ldg(d.sig + NS - 1));
            const real wx = d.windx[node], wy = d.windy[node];
            const real u_din_sur = real(0.05) * (wx * wx + wy * wy);
            const real snu_m = real(0.5) * (snu[NS - 1] + snu[NS - 2]);
            y2 = (real(0.4e-3) * (u_din_sur * u_din_sur * u_din_sur) * dmean * d1) / (snu_m * real(0.76));
        }
        // bottom boundary value (independent of the iteration)
        const real delta_b = jc_of(d, ajac, NS - 2) + d.z0b_min;
        const real lg = fesomc_log(delta_b / d.z0b_min);
        const real bott_R = B1cka2 / (lg * lg);
        const real ubt = Un[L - 1], vbt = Vn[L - 1];
        const real bot = bott_R * (ubt * ubt + vbt * vbt);
        real *btr = s_bA, *xq = s_bB;   // xq: this iteration's xx1, then its btr1
        bool converged = false;
        int iters = 200;
        for (int it = 1; it <= 200; ++it) {
            real x = real(1.0), y = y2;
            real s_lo = D3(s_sn, 1), s_mid = D3(s_sn, 2);
            real b_n = D3(btr, 2), pb_n = D3(s_pb, 2), qb_n = D3(s_qb, 2), c2_n = D3(s_c2, 2), sh_n = D3(s_sn, 3);
            for (int nz = 2; nz <= NS - 1; ++nz) {
                const real s_hi = sh_n;
                const real b = b_n, pbv = pb_n, qbv = qb_n, c2v = c2_n;
                if (nz + 1 <= NS - 1) {
                    b_n = D3(btr, nz + 1); pb_n = D3(s_pb, nz + 1); qb_n = D3(s_qb, nz + 1);
                    c2_n = D3(s_c2, nz + 1); sh_n = D3(s_sn, nz + 2);
                }
                const real s_m = __ldg(d.sig + nz - 2), s_0 = __ldg(d.sig + nz - 1), s_p = __ldg(d.sig + nz);
                const real dd1 = s_m - s_0;
                const real dd2 = s_0 - s_p;
                const real dd = real(0.5) * (dd1 + dd2);
                const real c1 = real(0.046) * (b * b) / s_mid;
                if (it == 200) tke[nz - 1] = c1;
                const real fr = pbv - c1 - qbv - c2v;
                const real snu_p = real(0.5) * (s_lo + s_mid);
                const real snu_mm = real(0.5) * (s_mid + s_hi);
                const real am = real(0.5) * (snu_p * real(0.73)) / (dmean2 * dd1 * dd);
                const real cm = real(0.5) * (snu_mm * real(0.73)) / (dmean2 * dd2 * dd);
                const real bm = am + cm + (real(2.0) * real(0.046) * b) / s_mid + t_inv;
                const real a = bm - am * x;
                const real xn = cm / a;
                const real yn = (am * y - fr) / a;
                D3(xq, nz + 1) = xn;
                D3(s_yy, nz + 1) = yn;
                x = xn;
                y = yn;
                s_lo = s_mid;
                s_mid = s_hi;
            }
            real b1v = bot;  // btr1(NS)
            real x_n = D3(xq, NS), y_n = D3(s_yy, NS), o_n = D3(btr, NS - 1);
            const real top = D3(btr, NS);
            D3(xq, NS) = b1v;
            bool above = d3_above_tol(top - b1v, dmax(b1v, top) + real(1.0e-8));
            for (int nz = NS; nz >= 2; --nz) {
                const real xv = x_n, yv = y_n, ov = o_n;
                if (nz - 1 >= 3) { x_n = D3(xq, nz - 1); y_n = D3(s_yy, nz - 1); o_n = D3(btr, nz - 2); }
                else if (nz - 1 == 2) { x_n = real(1.0); y_n = y2; o_n = D3(btr, nz - 2); }
                b1v = b1v * xv + yv;  // btr1(nz-1), into the xx1(nz-1) slot already read
                D3(xq, nz - 1) = b1v;
                above |= d3_above_tol(ov - b1v, dmax(b1v, ov) + real(1.0e-8));
            }
            if (!above) { converged = true; iters = it; break; }
            real *t = btr;
            btr = xq;
            xq = t;
        }
        if (d.d3_iters) d.d3_iters[node] = iters;   // measurement only (fesomc_gpu_d3end_iterations)
        if (converged) {
            for (int nz = 2; nz <= NS - 1; ++nz) {
                const real b = D3(btr, nz);
                tke[nz - 1] = real(0.046) * (b * b) / D3(s_sn, nz);
            }
        } else {
            atomicAdd(d.notconv, 1);
        }
        real *btw = d.bt + (size_t)node * NS;
        real *snw = d.snu + (size_t)node * NS;
        real *Kvw = d.Kv + (size_t)node * NS;
#pragma unroll 4
        for (int nz = 1; nz <= NS; ++nz) {
            const real btn = dmax(D3(btr, nz), real(1.0e-8));
            btw[nz - 1] = btn;
            const real zt = __ldg(d.sig + nz - 1) * dmean;
            const real Zh = zt + d.z0b_min;
            const real Zd = fabs(dmean - zt) + d.z0s_min;
            const real Z0 = real(1.0) - d.beta_scale * Zh * Zd / (dmean * dmean);
            const real scale_t = cka * Zh * Zd * Z0 / dmean;
            real s = scale_t * sqrt(btn) + d.snul;
            if (s >= real(0.2)) s = real(0.2);
            snw[nz - 1] = s;
            Kvw[nz - 1] = d.Pr_num * s;
        }
    }
#undef D3
}

// ---- d3_end in two kernels (launch-shape knob "d3end_arrays" = 3) ----------
// The set-up of a column (its per-interface constants, which take most of the
// FP64 work: two densityJM per interface and the divisions of b1, b2, c2,
// Ri) does not depend on the sweep, and its interfaces are independent.  The
// set-up kernel takes blocks of kD3Tile consecutive nodes, stages their
// columns in shared memory with coalesced loads, forms the constants with
// one thread per (node, interface) exactly as k_d3end's first loop does, and
// writes -b1-b2, t_inv*bt, c2 and snu level-major ([interface][node]: a warp
// of 32 consecutive nodes reads 256 contiguous bytes of one interface) and
// Ri in the column layout.  The sweep kernel then keeps only xx1, yy1 and
// the btr pair in local memory (4 arrays instead of 8: the working set of
// the resident columns fits in L2) and reads the constants level-major.
constexpr int kD3Tile = 32;
constexpr int kD3SetupThreads = 256;

__global__ void __launch_bounds__(kD3SetupThreads) k_d3end_setup(Dev d) {
    extern __shared__ unsigned char d3s_smem[];
    const int NS = d.NS, L = d.L, N = d.N;
    real *sm = reinterpret_cast<real *>(d3s_smem);
    // per node j of the tile, stride NS: U, V, T, S (L levels), bt, snu, Kv, Ri (NS)
    real *sU = sm, *sV = sm + 1 * kD3Tile * NS, *sT = sm + 2 * kD3Tile * NS, *sS = sm + 3 * kD3Tile * NS;
    real *sB = sm + 4 * kD3Tile * NS, *sN = sm + 5 * kD3Tile * NS, *sK = sm + 6 * kD3Tile * NS;
    real *sR = sm + 7 * kD3Tile * NS;
    real *sDm = sm + 8 * kD3Tile * NS, *sAj = sDm + kD3Tile;
    const real t_inv = real(1.0) / d.dt;
    for (long long n0 = (long long)blockIdx.x * kD3Tile; n0 < N; n0 += (long long)gridDim.x * kD3Tile) {
        const int nt = (int)(N - n0 < kD3Tile ? N - n0 : kD3Tile);
        for (int i = threadIdx.x; i < nt * L; i += blockDim.x) {
            const int j = i / L, k = i - j * L;
            const size_t g = (size_t)n0 * L + i;
            sU[j * NS + k] = d.Unode[g];
            sV[j * NS + k] = d.Vnode[g];
            sT[j * NS + k] = d.TF[g];
            sS[j * NS + k] = d.SF[g];
        }
        for (int i = threadIdx.x; i < nt * NS; i += blockDim.x) {
            const size_t g = (size_t)n0 * NS + i;
            sB[i] = d.bt[g];
            sN[i] = d.snu[g];
            sK[i] = d.Kv[g];
        }
        if ((int)threadIdx.x < nt) {
            const int node = (int)n0 + threadIdx.x;
            sDm[threadIdx.x] = dmax<real>(d.Dmin, d.depth[node] + d.eta_n[node]);
            sAj[threadIdx.x] = jac_a(d, d.eta_jac, node);
        }
        __syncthreads();
        // snu level-major, and Ri(1) = Ri(NS) = 0
        for (int i = threadIdx.x; i < kD3Tile * NS; i += blockDim.x) {
            const int j = i % kD3Tile, k = i / kD3Tile;   // node fastest
            if (j < nt) d.d3_sn[(size_t)k * N + n0 + j] = sN[j * NS + k];
        }
        for (int j = threadIdx.x; j < nt; j += blockDim.x) {
            sR[j * NS] = real(0.0);
            sR[j * NS + NS - 1] = real(0.0);
        }
        // the interfaces nz = 2..NS-1, node fastest (k_d3end's first loop)
        for (int i = threadIdx.x; i < kD3Tile * (NS - 2); i += blockDim.x) {
            const int j = i % kD3Tile, nz = 2 + i / kD3Tile;
            if (j >= nt) continue;
            const real *Un = sU + j * NS, *Vn = sV + j * NS, *T = sT + j * NS, *S = sS + j * NS;
            const real *bt = sB + j * NS, *Kv = sK + j * NS, *snc = sN + j * NS;
            const real dmean = sDm[j], dmean2 = dmean * dmean, ajac = sAj[j];
            const real s_m = __ldg(d.sig + nz - 2), s_0 = __ldg(d.sig + nz - 1), s_p = __ldg(d.sig + nz);
            const real d1 = s_m - s_0;
            const real d2 = s_0 - s_p;
            const real dd = real(0.5) * (d1 + d2);
            real ap1 = Un[nz - 2] - Un[nz - 1];
            const real ap2 = Vn[nz - 2] - Vn[nz - 1];
            const real sn_m = snc[nz - 2], sn_0 = snc[nz - 1], sn_p = snc[nz];
            real b1 = sn_0 * (ap1 * ap1 + ap2 * ap2) / (dd * dd);
            b1 = b1 / dmean2;
            const real zb = zbar_of(d, ajac, nz - 1);
            const real rho_up = density_jm(T[nz - 2], S[nz - 2], -zb, d.density_0);
            const real rho_dn = density_jm(T[nz - 1], S[nz - 1], -zb, d.density_0);
            ap1 = (rho_up - rho_dn) / dd;
            const real b2 = -real(0.5) * kG * Kv[nz - 1] * ap1 / (d.density_0 * dmean);
            const real snu_p = real(0.5) * (sn_m + sn_0);
            const real snu_m = real(0.5) * (sn_0 + sn_p);
            const real cc = real(0.5) * real(0.73) * (snu_p * (bt[nz - 2] - bt[nz - 1]) / d1 - snu_m * (bt[nz - 1] - bt[nz]) / d2) / dd;
            const size_t o = (size_t)(nz - 2) * N + n0 + j;
            d.d3_c2[o] = cc / dmean2;
            if (b1 > real(0.0)) sR[j * NS + nz - 1] = -kG * ap1 / (d.density_0 * dmean) / b1 * sn_0;
            else sR[j * NS + nz - 1] = real(10000.0);
            d.d3_pb[o] = -b1 - b2;
            d.d3_qb[o] = t_inv * bt[nz - 1];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nt * NS; i += blockDim.x) d.Ri[(size_t)n0 * NS + i] = sR[i];
        __syncthreads();
    }
}

// The sweeps of d3_end per node column, from the set-up's level-major
// constants; the same arithmetic as k_d3end, in the same order.
template <int ARR, bool kList>
__global__ void k_d3end_sweep(Dev d, const int *list, const unsigned long long *count) {
    const real t_inv = real(1.0) / d.dt;
    const real cka = d.cka;
    const real B1cka2 = real(16.6) * (cka * cka);
    const long long ncol = kList ? (long long)*count : (long long)d.N;
    const size_t N = d.N;
    GRID_LOOP(ii, ncol) {
        const int node = kList ? list[ii] : (int)ii;
        const int NS = d.NS, L = d.L;
        const real *bt = d.bt + (size_t)node * NS;
        const real *Un = d.Unode + (size_t)node * L;
        const real *Vn = d.Vnode + (size_t)node * L;
        real *tke = d.tke_dissip + (size_t)node * NS;
        // constants of interface nz (2..NS-1) and snu(nz) (1..NS), level-major
        auto PB = [&](int nz) { return d.d3_pb[(size_t)(nz - 2) * N + node]; };
        auto QB = [&](int nz) { return d.d3_qb[(size_t)(nz - 2) * N + node]; };
        auto C2 = [&](int nz) { return d.d3_c2[(size_t)(nz - 2) * N + node]; };
        auto SN = [&](int nz) { return d.d3_sn[(size_t)(nz - 1) * N + node]; };
        real xx1[ARR], yy1[ARR], bA[ARR], bB[ARR];
        const real dmean = dmax<real>(d.Dmin, d.depth[node] + d.eta_n[node]);
        const real dmean2 = dmean * dmean;
        const real ajac = jac_a(d, d.eta_jac, node);
        for (int nz = 1; nz <= NS; ++nz) bA[nz] = bt[nz - 1];
        real y2;
        {
            const real d1 = real(0.5) * (__ldg(d.sig + NS - 2) - __ldg(d.sig + NS - 1));
            const real wx = d.windx[node], wy = d.windy[node];
            const real u_din_sur = real(0.05) * (wx * wx + wy * wy);
            const real snu_m = real(0.5) * (SN(NS) + SN(NS - 1));
            y2 = (real(0.4e-3) * (u_din_sur * u_din_sur * u_din_sur) * dmean * d1) / (snu_m * real(0.76));
        }
        xx1[2] = real(1.0);
        yy1[2] = y2;
        const real delta_b = jc_of(d, ajac, NS - 2) + d.z0b_min;
        const real lg = fesomc_log(delta_b / d.z0b_min);
        const real bott_R = B1cka2 / (lg * lg);
        const real ubt = Un[L - 1], vbt = Vn[L - 1];
        const real bot = bott_R * (ubt * ubt + vbt * vbt);
        real *btr = bA, *btr1 = bB;
        bool converged = false;
        int iters = 200;
        for (int it = 1; it <= 200; ++it) {
            real x = real(1.0), y = y2;
            real s_lo = SN(1), s_mid = SN(2);
            real b_n = btr[2], pb_n = PB(2), qb_n = QB(2), c2_n = C2(2), sh_n = SN(3);
            for (int nz = 2; nz <= NS - 1; ++nz) {
                const real s_hi = sh_n;
                const real b = b_n, pbv = pb_n, qbv = qb_n, c2v = c2_n;
                if (nz + 1 <= NS - 1) {
                    b_n = btr[nz + 1]; pb_n = PB(nz + 1); qb_n = QB(nz + 1); c2_n = C2(nz + 1); sh_n = SN(nz + 2);
                }
                const real s_m = __ldg(d.sig + nz - 2), s_0 = __ldg(d.sig + nz - 1), s_p = __ldg(d.sig + nz);
                const real dd1 = s_m - s_0;
                const real dd2 = s_0 - s_p;
                const real dd = real(0.5) * (dd1 + dd2);
                const real c1 = real(0.046) * (b * b) / s_mid;
                if (it == 200) tke[nz - 1] = c1;
                const real fr = pbv - c1 - qbv - c2v;
                const real snu_p = real(0.5) * (s_lo + s_mid);
                const real snu_mm = real(0.5) * (s_mid + s_hi);
                const real am = real(0.5) * (snu_p * real(0.73)) / (dmean2 * dd1 * dd);
                const real cm = real(0.5) * (snu_mm * real(0.73)) / (dmean2 * dd2 * dd);
                const real bm = am + cm + (real(2.0) * real(0.046) * b) / s_mid + t_inv;
                const real a = bm - am * x;
                const real xn = cm / a;
                const real yn = (am * y - fr) / a;
                xx1[nz + 1] = xn;
                yy1[nz + 1] = yn;
                x = xn;
                y = yn;
                s_lo = s_mid;
                s_mid = s_hi;
            }
            real b1v = bot;  // btr1(NS)
            btr1[NS] = b1v;
            bool above = d3_above_tol(btr[NS] - b1v, dmax(b1v, btr[NS]) + real(1.0e-8));
            real x_n = xx1[NS], y_n = yy1[NS], o_n = btr[NS - 1];
            for (int nz = NS; nz >= 2; --nz) {
                const real xv = x_n, yv = y_n, ov = o_n;
                if (nz - 1 >= 2) { x_n = xx1[nz - 1]; y_n = yy1[nz - 1]; o_n = btr[nz - 2]; }
                b1v = b1v * xv + yv;  // btr1(nz-1)
                btr1[nz - 1] = b1v;
                above |= d3_above_tol(ov - b1v, dmax(b1v, ov) + real(1.0e-8));
            }
            if (!above) { converged = true; iters = it; break; }
            real *t = btr;
            btr = btr1;
            btr1 = t;
        }
        if (d.d3_iters) d.d3_iters[node] = iters;   // measurement only (fesomc_gpu_d3end_iterations)
        if (converged) {
            for (int nz = 2; nz <= NS - 1; ++nz) tke[nz - 1] = real(0.046) * (btr[nz] * btr[nz]) / SN(nz);
        } else {
            atomicAdd(d.notconv, 1);
        }
        real *btw = d.bt + (size_t)node * NS;
        real *snw = d.snu + (size_t)node * NS;
        real *Kvw = d.Kv + (size_t)node * NS;
        for (int nz = 1; nz <= NS; ++nz) {
            const real btn = dmax(btr[nz], real(1.0e-8));
            btw[nz - 1] = btn;
            const real zt = __ldg(d.sig + nz - 1) * dmean;
            const real Zh = zt + d.z0b_min;
            const real Zd = fabs(dmean - zt) + d.z0s_min;
            const real Z0 = real(1.0) - d.beta_scale * Zh * Zd / (dmean * dmean);
            const real scale_t = cka * Zh * Zd * Z0 / dmean;
            real s = scale_t * sqrt(btn) + d.snul;
            if (s >= real(0.2)) s = real(0.2);
            snw[nz - 1] = s;
            Kvw[nz - 1] = d.Pr_num * s;
        }
    }
}

// The sweeps with xx1, yy1 and the btr pair in shared memory, [array][level]
// [thread] (launch-shape knob "d3end_arrays" = 4): no local memory at all,
// 4*NS - 2 values per column, blocks of kD3Block columns.
__global__ void __launch_bounds__(kD3Block) k_d3end_sweep_sm(Dev d) {
    extern __shared__ unsigned char d3w_smem[];
    constexpr int B = kD3Block;
    const real t_inv = real(1.0) / d.dt;
    const real cka = d.cka;
    const real B1cka2 = real(16.6) * (cka * cka);
    const size_t N = d.N;
    const int NS = d.NS, L = d.L;
    real *const base = reinterpret_cast<real *>(d3w_smem) + threadIdx.x;
    // element nz of an array at [(nz - first) * B]
    real *const s_x = base - 2 * B;                      // xx1, nz = 2..NS
    real *const s_y = base + (NS - 1 - 2) * B;           // yy1, nz = 2..NS
    real *const s_bA = base + (2 * NS - 2 - 1) * B;      // nz = 1..NS
    real *const s_bB = base + (3 * NS - 2 - 1) * B;      // nz = 1..NS
#define W3(a, nz) a[(size_t)(nz) * B]
    GRID_LOOP(ii, (long long)d.N) {
        const int node = (int)ii;
        const real *bt = d.bt + (size_t)node * NS;
        const real *Un = d.Unode + (size_t)node * L;
        const real *Vn = d.Vnode + (size_t)node * L;
        real *tke = d.tke_dissip + (size_t)node * NS;
        // constants of interface nz (2..NS-1) and snu(nz) (1..NS), level-major
        auto PB = [&](int nz) { return d.d3_pb[(size_t)(nz - 2) * N + node]; };
        auto QB = [&](int nz) { return d.d3_qb[(size_t)(nz - 2) * N + node]; };
        auto C2 = [&](int nz) { return d.d3_c2[(size_t)(nz - 2) * N + node]; };
        auto SN = [&](int nz) { return d.d3_sn[(size_t)(nz - 1) * N + node]; };
        const real dmean = dmax<real>(d.Dmin, d.depth[node] + d.eta_n[node]);
        const real dmean2 = dmean * dmean;
        const real ajac = jac_a(d, d.eta_jac, node);
        for (int nz = 1; nz <= NS; ++nz) W3(s_bA, nz) = bt[nz - 1];
        real y2;
        {
            const real d1 = real(0.5) * (__ldg(d.sig + NS - 2) - __ldg(d.sig + NS - 1));
            const real wx = d.windx[node], wy = d.windy[node];
            const real u_din_sur = real(0.05) * (wx * wx + wy * wy);
            const real snu_m = real(0.5) * (SN(NS) + SN(NS - 1));
            y2 = (real(0.4e-3) * (u_din_sur * u_din_sur * u_din_sur) * dmean * d1) / (snu_m * real(0.76));
        }
        W3(s_x, 2) = real(1.0);
        W3(s_y, 2) = y2;
        const real delta_b = jc_of(d, ajac, NS - 2) + d.z0b_min;
        const real lg = fesomc_log(delta_b / d.z0b_min);
        const real bott_R = B1cka2 / (lg * lg);
        const real ubt = Un[L - 1], vbt = Vn[L - 1];
        const real bot = bott_R * (ubt * ubt + vbt * vbt);
        real *btr = s_bA, *btr1 = s_bB;
        bool converged = false;
        int iters = 200;
        for (int it = 1; it <= 200; ++it) {
            real x = real(1.0), y = y2;
            real s_lo = SN(1), s_mid = SN(2);
            real b_n = W3(btr, 2), pb_n = PB(2), qb_n = QB(2), c2_n = C2(2), sh_n = SN(3);
            for (int nz = 2; nz <= NS - 1; ++nz) {
                const real s_hi = sh_n;
                const real b = b_n, pbv = pb_n, qbv = qb_n, c2v = c2_n;
                if (nz + 1 <= NS - 1) {
                    b_n = W3(btr, nz + 1); pb_n = PB(nz + 1); qb_n = QB(nz + 1); c2_n = C2(nz + 1); sh_n = SN(nz + 2);
                }
                const real s_m = __ldg(d.sig + nz - 2), s_0 = __ldg(d.sig + nz - 1), s_p = __ldg(d.sig + nz);
                const real dd1 = s_m - s_0;
                const real dd2 = s_0 - s_p;
                const real dd = real(0.5) * (dd1 + dd2);
                const real c1 = real(0.046) * (b * b) / s_mid;
                if (it == 200) tke[nz - 1] = c1;
                const real fr = pbv - c1 - qbv - c2v;
                const real snu_p = real(0.5) * (s_lo + s_mid);
                const real snu_mm = real(0.5) * (s_mid + s_hi);
                const real am = real(0.5) * (snu_p * real(0.73)) / (dmean2 * dd1 * dd);
                const real cm = real(0.5) * (snu_mm * real(0.73)) / (dmean2 * dd2 * dd);
                const real bm = am + cm + (real(2.0) * real(0.046) * b) / s_mid + t_inv;
                const real a = bm - am * x;
                const real xn = cm / a;
                const real yn = (am * y - fr) / a;
                W3(s_x, nz + 1) = xn;
                W3(s_y, nz + 1) = yn;
                x = xn;
                y = yn;
                s_lo = s_mid;
                s_mid = s_hi;
            }
            real b1v = bot;  // btr1(NS)
            const real top = W3(btr, NS);
            W3(btr1, NS) = b1v;
            bool above = d3_above_tol(top - b1v, dmax(b1v, top) + real(1.0e-8));
            real x_n = W3(s_x, NS), y_n = W3(s_y, NS), o_n = W3(btr, NS - 1);
            for (int nz = NS; nz >= 2; --nz) {
                const real xv = x_n, yv = y_n, ov = o_n;
                if (nz - 1 >= 2) { x_n = W3(s_x, nz - 1); y_n = W3(s_y, nz - 1); o_n = W3(btr, nz - 2); }
                b1v = b1v * xv + yv;  // btr1(nz-1)
                W3(btr1, nz - 1) = b1v;
                above |= d3_above_tol(ov - b1v, dmax(b1v, ov) + real(1.0e-8));
            }
            if (!above) { converged = true; iters = it; break; }
            real *t = btr;
            btr = btr1;
            btr1 = t;
        }
        if (d.d3_iters) d.d3_iters[node] = iters;   // measurement only (fesomc_gpu_d3end_iterations)
        if (converged) {
            for (int nz = 2; nz <= NS - 1; ++nz) {
                const real b = W3(btr, nz);
                tke[nz - 1] = real(0.046) * (b * b) / SN(nz);
            }
        } else {
            atomicAdd(d.notconv, 1);
        }
        real *btw = d.bt + (size_t)node * NS;
        real *snw = d.snu + (size_t)node * NS;
        real *Kvw = d.Kv + (size_t)node * NS;
        for (int nz = 1; nz <= NS; ++nz) {
            const real btn = dmax(W3(btr, nz), real(1.0e-8));
            btw[nz - 1] = btn;
            const real zt = __ldg(d.sig + nz - 1) * dmean;
            const real Zh = zt + d.z0b_min;
            const real Zd = fabs(dmean - zt) + d.z0s_min;
            const real Z0 = real(1.0) - d.beta_scale * Zh * Zd / (dmean * dmean);
            const real scale_t = cka * Zh * Zd * Z0 / dmean;
            real s = scale_t * sqrt(btn) + d.snul;
            if (s >= real(0.2)) s = real(0.2);
            snw[nz - 1] = s;
            Kvw[nz - 1] = d.Pr_num * s;
        }
    }
#undef W3
}


// ---- the sweeps in registers (launch-shape knob "d3end_arrays" = 5, 6) -----
// For a level count fixed at compile time (NSC) every loop over the levels
// unrolls, so the column arrays live in registers and the sweep touches no
// local memory.  Three arrays instead of four: the back substitution writes
// btr1(m) into the slot of xx1(m + 1) it has just read (xx1(2) = 1 is a
// constant), so with btr(m) = P[m] the sweep leaves btr1(m) in Q[m + 1],
// copied back into P when the column has not converged.  yy1 keeps its own
// array (yy1(2) = y2 a constant).  The arithmetic is k_d3end_sweep's, in
// the same order; the constants are read level-major through the
// read-only path.
template <int NSC>
__device__ __forceinline__ bool d3_sweep_reg(const Dev &d, size_t N, int node, const real (&P)[NSC + 2],
                                             real (&Q)[NSC + 2], real (&Y)[NSC + 2], real y2, real bot, real dmean2,
                                             real t_inv, bool last, real *tke) {
    constexpr int PO = 0, QO = 0;
    const real *pb = d.d3_pb + node, *qb = d.d3_qb + node, *c2 = d.d3_c2 + node, *sn = d.d3_sn + node;
    real x = real(1.0), y = y2;
    real s_lo = __ldg(sn), s_mid = __ldg(sn + N);
#pragma unroll
    for (int nz = 2; nz <= NSC - 1; ++nz) {
        const real s_hi = __ldg(sn + (size_t)nz * N);
        const real b = P[nz + PO];
        const real pbv = __ldg(pb + (size_t)(nz - 2) * N), qbv = __ldg(qb + (size_t)(nz - 2) * N);
        const real c2v = __ldg(c2 + (size_t)(nz - 2) * N);
        const real s_m = __ldg(d.sig + nz - 2), s_0 = __ldg(d.sig + nz - 1), s_p = __ldg(d.sig + nz);
        const real dd1 = s_m - s_0;
        const real dd2 = s_0 - s_p;
        const real dd = real(0.5) * (dd1 + dd2);
        const real c1 = real(0.046) * (b * b) / s_mid;
        if (last) tke[nz - 1] = c1;
        const real fr = pbv - c1 - qbv - c2v;
        const real snu_p = real(0.5) * (s_lo + s_mid);
        const real snu_mm = real(0.5) * (s_mid + s_hi);
        const real am = real(0.5) * (snu_p * real(0.73)) / (dmean2 * dd1 * dd);
        const real cm = real(0.5) * (snu_mm * real(0.73)) / (dmean2 * dd2 * dd);
        const real bm = am + cm + (real(2.0) * real(0.046) * b) / s_mid + t_inv;
        const real a = bm - am * x;
        const real xn = cm / a;
        const real yn = (am * y - fr) / a;
        Q[nz + 1 + QO] = xn;
        Y[nz + 1] = yn;
        x = xn;
        y = yn;
        s_lo = s_mid;
        s_mid = s_hi;
    }
    real b1v = bot;  // btr1(NS)
    bool above = d3_above_tol(P[NSC + PO] - b1v, dmax(b1v, P[NSC + PO]) + real(1.0e-8));
    Q[NSC + 1 + QO] = b1v;
#pragma unroll
    for (int nz = NSC; nz >= 2; --nz) {
        const real xv = nz == 2 ? real(1.0) : Q[nz + QO];
        const real yv = nz == 2 ? y2 : Y[nz];
        const real ov = P[nz - 1 + PO];
        b1v = b1v * xv + yv;  // btr1(nz-1)
        Q[nz + QO] = b1v;
        above |= d3_above_tol(ov - b1v, dmax(b1v, ov) + real(1.0e-8));
    }
    return above;
}

// MINB resident blocks of 64 columns per SM: 6 (at most 168 registers) or
// 8 (128 registers, a few spilled)
template <int NSC, int MINB>
__global__ void __launch_bounds__(64, MINB) k_d3end_sweep_reg(Dev d) {
    const real t_inv = real(1.0) / d.dt;
    const real cka = d.cka;
    const real B1cka2 = real(16.6) * (cka * cka);
    const size_t N = d.N;
    constexpr int NS = NSC;
    const int L = d.L;
    GRID_LOOP(ii, (long long)d.N) {
        const int node = (int)ii;
        const real *bt = d.bt + (size_t)node * NS;
        const real *Un = d.Unode + (size_t)node * L;
        const real *Vn = d.Vnode + (size_t)node * L;
        real *tke = d.tke_dissip + (size_t)node * NS;
        auto SN = [&](int nz) { return __ldg(d.d3_sn + (size_t)(nz - 1) * N + node); };
        real A[NSC + 2], B[NSC + 2], Y[NSC + 2];
        const real dmean = dmax<real>(d.Dmin, d.depth[node] + d.eta_n[node]);
        const real dmean2 = dmean * dmean;
        const real ajac = jac_a(d, d.eta_jac, node);
#pragma unroll
        for (int nz = 1; nz <= NS; ++nz) A[nz] = bt[nz - 1];
        real y2;
        {
            const real d1 = real(0.5) * (__ldg(d.sig + NS - 2) - __ldg(d.sig + NS - 1));
            const real wx = d.windx[node], wy = d.windy[node];
            const real u_din_sur = real(0.05) * (wx * wx + wy * wy);
            const real snu_m = real(0.5) * (SN(NS) + SN(NS - 1));
            y2 = (real(0.4e-3) * (u_din_sur * u_din_sur * u_din_sur) * dmean * d1) / (snu_m * real(0.76));
        }
        const real delta_b = jc_of(d, ajac, NS - 2) + d.z0b_min;
        const real lg = fesomc_log(delta_b / d.z0b_min);
        const real bott_R = B1cka2 / (lg * lg);
        const real ubt = Un[L - 1], vbt = Vn[L - 1];
        const real bot = bott_R * (ubt * ubt + vbt * vbt);
        // A ends as the final btr: the previous iterate when a sweep
        // converges, the last sweep's result after 200 without convergence
        bool converged = false;
        int iters = 200;
        for (int it = 1; it <= 200; ++it) {
            if (!d3_sweep_reg<NSC>(d, N, node, A, B, Y, y2, bot, dmean2, t_inv, it == 200, tke)) {
                converged = true;
                iters = it;
                break;
            }
#pragma unroll
            for (int m = 1; m <= NS; ++m) A[m] = B[m + 1];
        }
        if (d.d3_iters) d.d3_iters[node] = iters;   // measurement only (fesomc_gpu_d3end_iterations)
        if (converged) {
#pragma unroll
            for (int nz = 2; nz <= NS - 1; ++nz) tke[nz - 1] = real(0.046) * (A[nz] * A[nz]) / SN(nz);
        } else {
            atomicAdd(d.notconv, 1);
        }
        real *btw = d.bt + (size_t)node * NS;
        real *snw = d.snu + (size_t)node * NS;
        real *Kvw = d.Kv + (size_t)node * NS;
#pragma unroll
        for (int nz = 1; nz <= NS; ++nz) {
            const real btn = dmax(A[nz], real(1.0e-8));
            btw[nz - 1] = btn;
            const real zt = __ldg(d.sig + nz - 1) * dmean;
            const real Zh = zt + d.z0b_min;
            const real Zd = fabs(dmean - zt) + d.z0s_min;
            const real Z0 = real(1.0) - d.beta_scale * Zh * Zd / (dmean * dmean);
            const real scale_t = cka * Zh * Zd * Z0 / dmean;
            real s = scale_t * sqrt(btn) + d.snul;
            if (s >= real(0.2)) s = real(0.2);
            snw[nz - 1] = s;
            Kvw[nz - 1] = d.Pr_num * s;
        }
    }
}

// Av(nz,elem) = sum(w_cv*snu(nz,nodes)) (fv_mixing.F90:308-313)
__global__ void k_av(Dev d) {
    const long long total = (long long)d.E * d.NS;
    GRID_LOOP(ii, total) {
        const int e = (int)(ii / d.NS);
        const int z = (int)(ii % d.NS);
        const int4 en = d.elem_nodes[e];
        const real4 w = d.w_cv[e];
        const int NS = d.NS;
        d.Av[ii] = wsum(w, d.snu[(size_t)en.x * NS + z], d.snu[(size_t)en.y * NS + z], d.snu[(size_t)en.z * NS + z],
                        d.snu[(size_t)en.w * NS + z]);
    }
}

static size_t d3end_smem(const Dev &d) { return (size_t)d3end_values(d.NS) * kD3Block * sizeof(real); }
static size_t d3end_setup_smem(const Dev &d) { return ((size_t)8 * kD3Tile * d.NS + 2 * kD3Tile) * sizeof(real); }
// the two-kernel form: up to 40 levels (its sweep's local arrays are sized
// like k_d3end's)
static bool d3end_split(const Dev &d) { return d.tune[TK_D3END] >= 3 && d.NS <= 40; }
// the register sweep is compiled for these level counts; others take the
// local-memory sweep
static bool d3end_reg(const Dev &d) { return d.tune[TK_D3END] >= 5 && (d.NS == 11 || d.NS == 21); }
static size_t d3end_sweep_smem(const Dev &d) { return (size_t)(4 * d.NS - 2) * kD3Block * sizeof(real); }
int config_d3end(const Dev &d) {
    if (d.NS > 127) return 1;
    if (d.NS <= 40 && (raise_smem_limit(k_d3end_setup, d3end_setup_smem(d)) != cudaSuccess ||
                       raise_smem_limit(k_d3end_sweep_sm, d3end_sweep_smem(d)) != cudaSuccess))
        return 1;
    return (raise_smem_limit(k_d3end_sm<false>, d3end_smem(d)) == cudaSuccess &&
            raise_smem_limit(k_d3end_sm<true>, d3end_smem(d)) == cudaSuccess) ? 0 : 1;
}
static void launch_d3end_split(const Dev &d, cudaStream_t s) {
    const int tiles = (d.N + kD3Tile - 1) / kD3Tile;
    k_d3end_setup<<<tiles < 148 * 16 ? tiles : 148 * 16, kD3SetupThreads, d3end_setup_smem(d), s>>>(d);
    if (d3end_reg(d)) {
        const bool b8 = d.tune[TK_D3END] == 6;
        if (d.NS == 11 && b8) k_d3end_sweep_reg<11, 8><<<grid_for(d.N, 64), 64, 0, s>>>(d);
        else if (d.NS == 11) k_d3end_sweep_reg<11, 6><<<grid_for(d.N, 64), 64, 0, s>>>(d);
        else if (b8) k_d3end_sweep_reg<21, 8><<<grid_for(d.N, 64), 64, 0, s>>>(d);
        else k_d3end_sweep_reg<21, 6><<<grid_for(d.N, 64), 64, 0, s>>>(d);
    }
    else if (d.tune[TK_D3END] == 4) k_d3end_sweep_sm<<<grid_for(d.N, kD3Block), kD3Block, d3end_sweep_smem(d), s>>>(d);
    else if (d.NS <= 11) k_d3end_sweep<12, false><<<grid_for(d.N, 64), 64, 0, s>>>(d, nullptr, nullptr);
    else if (d.NS <= 21) k_d3end_sweep<22, false><<<grid_for(d.N, 64), 64, 0, s>>>(d, nullptr, nullptr);
    else k_d3end_sweep<41, false><<<grid_for(d.N, 64), 64, 0, s>>>(d, nullptr, nullptr);
}
void launch_d3end(const Dev &d, cudaStream_t s) {
    if (d3end_split(d)) launch_d3end_split(d, s);
    else if (d.tune[TK_D3END] == 2) k_d3end_sm<false><<<grid_for(d.N, kD3Block), kD3Block, d3end_smem(d), s>>>(d, nullptr, nullptr);
    else if (d.NS <= 11) k_d3end<12, false><<<grid_for(d.N, 64), 64, 0, s>>>(d, nullptr, nullptr);
    else if (d.NS <= 21) k_d3end<22, false><<<grid_for(d.N, 64), 64, 0, s>>>(d, nullptr, nullptr);
    else if (d.NS <= 40) k_d3end<41, false><<<grid_for(d.N, 64), 64, 0, s>>>(d, nullptr, nullptr);
    else k_d3end<128, false><<<grid_for(d.N, 64), 64, 0, s>>>(d, nullptr, nullptr);
}
// the plain closure on the listed columns (count read on the device, so the
// launch covers every node and the grid-stride loop stops at the count)
// (the two-kernel form sets up every column, so the listed columns take the
// one-kernel forms, which leave the others' Ri alone)
void launch_d3end_list(const Dev &d, const int *list, const unsigned long long *count, cudaStream_t s) {
    if (d.tune[TK_D3END] == 2) k_d3end_sm<true><<<grid_for(d.N, kD3Block), kD3Block, d3end_smem(d), s>>>(d, list, count);
    else if (d.NS <= 11) k_d3end<12, true><<<grid_for(d.N, 64), 64, 0, s>>>(d, list, count);
    else if (d.NS <= 21) k_d3end<22, true><<<grid_for(d.N, 64), 64, 0, s>>>(d, list, count);
    else if (d.NS <= 40) k_d3end<41, true><<<grid_for(d.N, 64), 64, 0, s>>>(d, list, count);
    else k_d3end<128, true><<<grid_for(d.N, 64), 64, 0, s>>>(d, list, count);
}
void launch_av(const Dev &d, cudaStream_t s) {
    const int b = tuned(d, TK_AV, 256);
    k_av<<<grid_for((long long)d.E * d.NS, b), b, 0, s>>>(d);
}


// Largest block (threads) each tunable kernel of this file can launch with
// (its registers and launch bounds): lim[knob] lowered to that.
static void tune_lower(int *lim, int knob, const void *k) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, k) == cudaSuccess && a.maxThreadsPerBlock < lim[knob]) lim[knob] = a.maxThreadsPerBlock;
}
void tune_limits_mixing(int *lim) {
    tune_lower(lim, TK_AV, (const void *)k_av);
}

FESOMC_PREC_END
