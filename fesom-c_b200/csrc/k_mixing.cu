// Vertical turbulence closure d3_end (src/fv_mixing.F90:73-347): one thread
// per node column.  Each column iterates its implicit turbulence-energy
// sweep up to 200 times (relative tolerance 1e-6); columns that reach the cap
// are counted in the device status (the reference silently continues).
// Compute / latency bound (FP64 divisions, log, sqrt).
#include "device_common.cuh"

namespace fesomc {

// Convergence test of d3_end's sweep (fv_mixing.F90:250-259) for one level:
// the reference forms c = |a/b| and stops when the largest c is below 1e-6
// (a NaN c never raises the maximum).  Returns true when this level forbids
// convergence, i.e. when RN(|a|/|b|) >= 1e-6.  The quotient is only formed
// when |a| lies within a relative 2^-30 of 1e-6*|b|; outside that band the
// comparison of |a| with the product decides it with certainty (the band is
// far wider than the rounding of the product and of the quotient).
__device__ __forceinline__ bool d3_above_tol(double a, double b) {
    const double aa = fabs(a), bb = fabs(b);
    if (bb > 1.0e-290 && bb < 1.0e290 && aa < 1.0e300) {
        const double t = 1.0e-6 * bb;
        if (aa <= t * (1.0 - 0x1p-30)) return false;
        if (aa >= t * (1.0 + 0x1p-30)) return true;
    }
    return fabs(a / b) >= 1.0e-6;
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
//   * the convergence test forms the quotient only near the threshold.
template <int ARR>
__global__ void k_d3end(Dev d) {
    const double t_inv = 1.0 / d.dt;
    const double cka = d.cka;
    const double B1cka2 = 16.6 * (cka * cka);
    GRID_LOOP(ii, d.N) {
        const int node = (int)ii;
        const int NS = d.NS, L = d.L;
        const double *bt = d.bt + (size_t)node * NS;
        const double *snu = d.snu + (size_t)node * NS;
        const double *Kv = d.Kv + (size_t)node * NS;
        const double *Un = d.Unode + (size_t)node * L;
        const double *Vn = d.Vnode + (size_t)node * L;
        const double *T = d.TF + (size_t)node * L;
        const double *S = d.SF + (size_t)node * L;
        double *Ri = d.Ri + (size_t)node * NS;
        double *tke = d.tke_dissip + (size_t)node * NS;
        double xx1[ARR], yy1[ARR], bA[ARR], bB[ARR], pb[ARR], qb[ARR], c2[ARR], sn[ARR];
        const double dmean = dmax(d.Dmin, d.depth[node] + d.eta_n[node]);
        const double dmean2 = dmean * dmean;
        const double ajac = jac_a(d, d.eta_jac, node);
        for (int nz = 1; nz <= NS; ++nz) {
            bA[nz] = bt[nz - 1];
            sn[nz] = snu[nz - 1];
        }
        Ri[0] = 0.0;
        Ri[NS - 1] = 0.0;
        for (int nz = 2; nz <= NS - 1; ++nz) {
            const double s_m = __ldg(d.sig + nz - 2), s_0 = __ldg(d.sig + nz - 1), s_p = __ldg(d.sig + nz);
            const double d1 = s_m - s_0;
            const double d2 = s_0 - s_p;
            const double dd = 0.5 * (d1 + d2);
            double ap1 = Un[nz - 2] - Un[nz - 1];
            const double ap2 = Vn[nz - 2] - Vn[nz - 1];
            double b1 = sn[nz] * (ap1 * ap1 + ap2 * ap2) / (dd * dd);
            b1 = b1 / dmean2;
            const double zb = zbar_of(d, ajac, nz - 1);
            const double rho_up = density_jm(T[nz - 2], S[nz - 2], -zb, d.density_0);
            const double rho_dn = density_jm(T[nz - 1], S[nz - 1], -zb, d.density_0);
            ap1 = (rho_up - rho_dn) / dd;
            const double b2 = -0.5 * kG * Kv[nz - 1] * ap1 / (d.density_0 * dmean);
            const double snu_p = 0.5 * (sn[nz - 1] + sn[nz]);
            const double snu_m = 0.5 * (sn[nz] + sn[nz + 1]);
            const double cc = 0.5 * 0.73 * (snu_p * (bt[nz - 2] - bt[nz - 1]) / d1 - snu_m * (bt[nz - 1] - bt[nz]) / d2) / dd;
            c2[nz] = cc / dmean2;
            if (b1 > 0.0) Ri[nz - 1] = -kG * ap1 / (d.density_0 * dmean) / b1 * sn[nz];
            else Ri[nz - 1] = 10000.0;
            pb[nz] = -b1 - b2;
            qb[nz] = t_inv * bt[nz - 1];
        }
        double y2;
        {
            const double d1 = 0.5 * (__ldg(d.sig + NS - 2) - __ldg(d.sig + NS - 1));
            const double wx = d.windx[node], wy = d.windy[node];
            const double u_din_sur = 0.05 * (wx * wx + wy * wy);
            const double snu_m = 0.5 * (sn[NS] + sn[NS - 1]);
            y2 = (0.4e-3 * (u_din_sur * u_din_sur * u_din_sur) * dmean * d1) / (snu_m * 0.76);
        }
        xx1[2] = 1.0;
        yy1[2] = y2;
        // bottom boundary value (independent of the iteration)
        const double delta_b = jc_of(d, ajac, NS - 2) + d.z0b_min;
        const double lg = log(delta_b / d.z0b_min);
        const double bott_R = B1cka2 / (lg * lg);
        const double ubt = Un[L - 1], vbt = Vn[L - 1];
        const double bot = bott_R * (ubt * ubt + vbt * vbt);
        double *btr = bA, *btr1 = bB;
        bool converged = false;
        for (int it = 1; it <= 200; ++it) {
            double x = 1.0, y = y2;
            double s_lo = sn[1], s_mid = sn[2];
            for (int nz = 2; nz <= NS - 1; ++nz) {
                const double s_hi = sn[nz + 1];
                const double s_m = __ldg(d.sig + nz - 2), s_0 = __ldg(d.sig + nz - 1), s_p = __ldg(d.sig + nz);
                const double dd1 = s_m - s_0;
                const double dd2 = s_0 - s_p;
                const double dd = 0.5 * (dd1 + dd2);
                const double b = btr[nz];
                const double c1 = 0.046 * (b * b) / s_mid;
                if (it == 200) tke[nz - 1] = c1;
                const double fr = pb[nz] - c1 - qb[nz] - c2[nz];
                const double snu_p = 0.5 * (s_lo + s_mid);
                const double snu_mm = 0.5 * (s_mid + s_hi);
                const double am = 0.5 * (snu_p * 0.73) / (dmean2 * dd1 * dd);
                const double cm = 0.5 * (snu_mm * 0.73) / (dmean2 * dd2 * dd);
                const double bm = am + cm + (2.0 * 0.046 * b) / s_mid + t_inv;
                const double a = bm - am * x;
                const double xn = cm / a;
                const double yn = (am * y - fr) / a;
                xx1[nz + 1] = xn;
                yy1[nz + 1] = yn;
                x = xn;
                y = yn;
                s_lo = s_mid;
                s_mid = s_hi;
            }
            double b1v = bot;  // btr1(NS)
            btr1[NS] = b1v;
            bool above = d3_above_tol(btr[NS] - b1v, dmax(b1v, btr[NS]) + 1.0e-8);
            for (int nz = NS; nz >= 2; --nz) {
                b1v = b1v * xx1[nz] + yy1[nz];  // btr1(nz-1)
                btr1[nz - 1] = b1v;
                above |= d3_above_tol(btr[nz - 1] - b1v, dmax(b1v, btr[nz - 1]) + 1.0e-8);
            }
            if (!above) { converged = true; break; }
            double *t = btr;
            btr = btr1;
            btr1 = t;
        }
        if (converged) {
            for (int nz = 2; nz <= NS - 1; ++nz) tke[nz - 1] = 0.046 * (btr[nz] * btr[nz]) / sn[nz];
        } else {
            atomicAdd(d.notconv, 1);
        }
        double *btw = d.bt + (size_t)node * NS;
        double *snw = d.snu + (size_t)node * NS;
        double *Kvw = d.Kv + (size_t)node * NS;
        for (int nz = 1; nz <= NS; ++nz) {
            const double btn = dmax(btr[nz], 1.0e-8);
            btw[nz - 1] = btn;
            const double zt = __ldg(d.sig + nz - 1) * dmean;
            const double Zh = zt + d.z0b_min;
            const double Zd = fabs(dmean - zt) + d.z0s_min;
            const double Z0 = 1.0 - d.beta_scale * Zh * Zd / (dmean * dmean);
            const double scale_t = cka * Zh * Zd * Z0 / dmean;
            double s = scale_t * sqrt(btn) + d.snul;
            if (s >= 0.2) s = 0.2;
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
        const double4 w = d.w_cv[e];
        const int NS = d.NS;
        d.Av[ii] = wsum(w, d.snu[(size_t)en.x * NS + z], d.snu[(size_t)en.y * NS + z], d.snu[(size_t)en.z * NS + z],
                        d.snu[(size_t)en.w * NS + z]);
    }
}

int config_d3end(const Dev &d) { return d.NS <= 127 ? 0 : 1; }
void launch_d3end(const Dev &d, cudaStream_t s) {
    if (d.NS <= 11) k_d3end<12><<<grid_for(d.N, 64), 64, 0, s>>>(d);
    else if (d.NS <= 21) k_d3end<22><<<grid_for(d.N, 64), 64, 0, s>>>(d);
    else if (d.NS <= 40) k_d3end<41><<<grid_for(d.N, 64), 64, 0, s>>>(d);
    else k_d3end<128><<<grid_for(d.N, 64), 64, 0, s>>>(d);
}
void launch_av(const Dev &d, cudaStream_t s) { k_av<<<grid_for((long long)d.E * d.NS, 256), 256, 0, s>>>(d); }

}  // namespace fesomc
