// Learned vertical-mixing closure, the model side: per node column the
// network's inputs (from the same state d3_end reads, src/fv_mixing.F90:
// 109-196), the training-envelope test that hands a column to the plain
// closure, the training-set harvest, the application of the network's
// output to snu, Kv and bt, and the judge statistics.  Compiled once per
// arithmetic precision like the other state kernels.  No counterpart in the
// reference.
#include "closure.h"
#include "device_common.cuh"

FESOMC_PREC_BEGIN

// Raw (transformed, not normalised) inputs of node column 'node', written to
// f[0..IN) with stride 1 (layout in closure.h).
__device__ void lc_inputs(const Dev &d, int node, float *f) {
    const int NS = d.NS, L = d.L;
    const real *Un = d.Unode + (size_t)node * L;
    const real *Vn = d.Vnode + (size_t)node * L;
    const real *T = d.TF + (size_t)node * L;
    const real *S = d.SF + (size_t)node * L;
    const real dmean = dmax<real>(d.Dmin, d.depth[node] + d.eta_n[node]);
    const real dmean2 = dmean * dmean;
    const real ajac = jac_a(d, d.eta_jac, node);
    for (int k = 0; k < NS; ++k) {
        real sh = real(0.0), n2 = real(0.0);
        if (k >= 1 && k <= NS - 2) {
            const real d1 = __ldg(d.sig + k - 1) - __ldg(d.sig + k);
            const real d2 = __ldg(d.sig + k) - __ldg(d.sig + k + 1);
            const real dd = real(0.5) * (d1 + d2);
            const real ap1 = Un[k - 1] - Un[k], ap2 = Vn[k - 1] - Vn[k];
            sh = (ap1 * ap1 + ap2 * ap2) / (dd * dd) / dmean2;
            const real zb = zbar_of(d, ajac, k);
            const real rho_up = density_jm(T[k - 1], S[k - 1], -zb, d.density_0);
            const real rho_dn = density_jm(T[k], S[k], -zb, d.density_0);
            n2 = -kG * (rho_up - rho_dn) / dd / (d.density_0 * dmean);
        }
        f[k] = asinhf((float)sh / kLcX0);
        f[NS + k] = asinhf((float)n2 / kLcX0);
        f[2 * NS + k] = (float)zbar_of(d, ajac, k);
    }
    const real wx = d.windx[node], wy = d.windy[node];
    const real u_din_sur = real(0.05) * (wx * wx + wy * wy);
    const real delta_b = jc_of(d, ajac, NS - 2) + d.z0b_min;
    const real lg = log(delta_b / d.z0b_min);
    const real bott_R = real(16.6) * (d.cka * d.cka) / (lg * lg);
    const real bot = bott_R * (Un[L - 1] * Un[L - 1] + Vn[L - 1] * Vn[L - 1]);
    f[3 * NS] = asinhf((float)u_din_sur / kLcX0);
    f[3 * NS + 1] = asinhf((float)bot / kLcX0);
    f[3 * NS + 2] = (float)dmean;
}

// warp-aggregated append of 'take' lanes to a list counter
__device__ __forceinline__ unsigned long long warp_append(bool take, unsigned long long *ctr) {
    const unsigned mask = __activemask();
    const unsigned b = __ballot_sync(mask, take);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if (lane == leader && b) base = atomicAdd(ctr, (unsigned long long)__popc(b));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(b & ((1u << lane) - 1u));
}

// Inputs of every column, normalised into X; the envelope test; the list of
// columns the plain closure takes (dry or outside the envelope); counters.
__global__ void k_lc_features(Dev d, LcView c) {
    GRID_LOOP(ii, d.N) {
        const int node = (int)ii;
        float *x = c.X + (size_t)node * c.IN;
        lc_inputs(d, node, x);
        const bool wet = d.mask_wd_node[node] != real(0.0);
        bool in = true;
        // statically unstable column (a negative N^2 input, sign kept by asinh)
        if (c.rules & kLcRuleUnstable)
            for (int k = 1; k <= c.NS - 2; ++k) in = in && !(x[c.NS + k] < 0.0f);
        // coastline and open-boundary columns
        if ((c.rules & kLcRuleBoundary) && d.index_nod2D[node] != 0) in = false;
        for (int j = 0; j < c.IN; ++j) {
            const float v = (x[j] - c.mu_x[j]) / c.sd_x[j];
            x[j] = v;
            in = in && (v >= c.lo_x[j]) && (v <= c.hi_x[j]);
        }
        const bool net = wet && in;
        c.flag[node] = net ? 1 : 0;
        const unsigned long long slot = warp_append(!net, c.count);
        if (!net) c.list[slot] = node;
        if (wet) atomicAdd(&c.acc[0], 1ULL);
        if (wet && !in) atomicAdd(&c.acc[1], 1ULL);
        if (!wet) atomicAdd(&c.acc[2], 1ULL);
    }
}

// The network's closure state of interface k: bt from its output, held to
// the range of the training targets, and snu, Kv from bt exactly as d3_end
// forms them (fv_mixing.F90:280-300).
__device__ __forceinline__ void lc_state(const Dev &d, const LcView &c, int node, int k, real dmean, real &bt,
                                         real &snu) {
    float lb = c.Y[(size_t)node * c.OUT + k] * c.sd_y[k] + c.mu_y[k];
    if (!(lb >= c.lo_y[k])) lb = c.lo_y[k];   // NaN too
    if (lb > c.hi_y[k]) lb = c.hi_y[k];
    const real btn = dmax((real)expf(lb), real(1.0e-8));
    const real zt = __ldg(d.sig + k) * dmean;
    const real Zh = zt + d.z0b_min;
    const real Zd = fabs(dmean - zt) + d.z0s_min;
    const real Z0 = real(1.0) - d.beta_scale * Zh * Zd / (dmean * dmean);
    const real scale_t = d.cka * Zh * Zd * Z0 / dmean;
    real s = scale_t * sqrt(btn) + d.snul;
    if (s >= real(0.2)) s = real(0.2);
    bt = btn;
    snu = s;
}

// Network columns: bt, snu and Kv of the network's closure state.
__global__ void k_lc_apply(Dev d, LcView c) {
    GRID_LOOP(ii, d.N) {
        const int node = (int)ii;
        if (!c.flag[node]) continue;
        const int NS = d.NS;
        const real dmean = dmax<real>(d.Dmin, d.depth[node] + d.eta_n[node]);
        real *bt = d.bt + (size_t)node * NS;
        real *sn = d.snu + (size_t)node * NS;
        real *kv = d.Kv + (size_t)node * NS;
        for (int k = 0; k < NS; ++k) {
            real b, s;
            lc_state(d, c, node, k, dmean, b, s);
            bt[k] = b;
            sn[k] = s;
            kv[k] = d.Pr_num * s;
        }
    }
}

// Training pairs: raw inputs and log bt of the wet columns, after the plain
// closure has run on the step, appended in node order (the order of the
// training set, hence the minibatches, does not depend on scheduling):
// each block of kLcHarvestBlock consecutive nodes counts its wet columns,
// one block turns the counts into first slots (an ordered scan from the
// current count), and each block writes its columns at its slots.
__global__ void k_lc_wetcount(Dev d, LcView c) {
    const int node = blockIdx.x * kLcHarvestBlock + threadIdx.x;
    const bool wet = node < d.N && d.mask_wd_node[node] != real(0.0);
    const int n = __syncthreads_count(wet);
    if (threadIdx.x == 0) c.blk[blockIdx.x] = n;
}

// blk[b] <- the slot of block b's first wet column (capped at hcap);
// hcount <- hcount + all wet columns.  One block of 1024 threads.
__global__ void k_lc_slots(int nblk, LcView c) {
    __shared__ unsigned long long wsum[32];
    __shared__ unsigned long long base;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) base = *c.hcount;
    __syncthreads();
    for (int c0 = 0; c0 < nblk; c0 += 1024) {
        const int i = c0 + (int)threadIdx.x;
        const unsigned long long v = i < nblk ? (unsigned long long)c.blk[i] : 0ULL;
        unsigned long long incl = v;   // inclusive scan within the warp
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) wsum[w] = incl;
        __syncthreads();
        if (w == 0) {
            unsigned long long t = wsum[lane], ti = t;
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long u = __shfl_up_sync(0xffffffffu, ti, o);
                if (lane >= o) ti += u;
            }
            wsum[lane] = ti - t;   // exclusive over warps
        }
        __syncthreads();
        const unsigned long long slot = base + wsum[w] + incl - v;
        if (i < nblk) c.blk[i] = (int)(slot < (unsigned long long)c.hcap ? slot : (unsigned long long)c.hcap);
        __syncthreads();
        if (threadIdx.x == 1023) base = slot + v;   // the last thread holds the chunk's end
        __syncthreads();
    }
    if (threadIdx.x == 0) *c.hcount = base;
}

__global__ void k_lc_harvest(Dev d, LcView c) {
    __shared__ int wcount[kLcHarvestBlock / 32];
    const int node = blockIdx.x * kLcHarvestBlock + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const bool wet = node < d.N && d.mask_wd_node[node] != real(0.0);
    const unsigned b = __ballot_sync(0xffffffffu, wet);
    if (lane == 0) wcount[w] = __popc(b);
    __syncthreads();
    int before = 0;
    for (int k = 0; k < w; ++k) before += wcount[k];
    const long long slot = (long long)c.blk[blockIdx.x] + before + __popc(b & ((1u << lane) - 1u));
    if (!wet || slot >= c.hcap) return;
    lc_inputs(d, node, c.hx + slot * c.IN);
    const int NS = d.NS;
    float *y = c.hy + slot * c.OUT;
    for (int k = 0; k < NS; ++k) y[k] = logf((float)d.bt[(size_t)node * NS + k]);   // bt >= 1e-8
}

// judge: the plain closure ran on every column; compare the network's
// viscosity on the columns it would have taken (log difference)
__global__ void k_lc_judge(Dev d, LcView c) {
    double s2 = 0.0, n = 0.0, mx = 0.0;
    GRID_LOOP(ii, d.N) {
        const int node = (int)ii;
        if (!c.flag[node]) continue;
        const real dmean = dmax<real>(d.Dmin, d.depth[node] + d.eta_n[node]);
        for (int k = 0; k < d.NS; ++k) {
            real b, s;
            lc_state(d, c, node, k, dmean, b, s);
            const real sp = d.snu[(size_t)node * d.NS + k];
            if (!(s > real(0.0) && sp > real(0.0))) continue;   // log of a non-positive viscosity
            const double e = log((double)s) - log((double)sp);
            s2 += e * e;
            n += 1.0;
            mx = fmax(mx, fabs(e));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
        n += __shfl_down_sync(0xffffffffu, n, o);
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0 && n > 0.0) {
        atomicAdd(&c.judge[0], s2);
        atomicAdd(&c.judge[1], n);
        // max of non-negative doubles through their ordered bit patterns
        atomicMax(reinterpret_cast<unsigned long long *>(&c.judge[2]), (unsigned long long)__double_as_longlong(mx));
    }
}

void launch_lc_features(const Dev &d, const LcView &c, cudaStream_t s) {
    k_lc_features<<<grid_for(d.N, 128), 128, 0, s>>>(d, c);
}
void launch_lc_apply(const Dev &d, const LcView &c, cudaStream_t s) {
    k_lc_apply<<<grid_for(d.N, 128), 128, 0, s>>>(d, c);
}
int lc_harvest_blocks(int N) { return (N + kLcHarvestBlock - 1) / kLcHarvestBlock; }
void launch_lc_harvest(const Dev &d, const LcView &c, cudaStream_t s) {
    const int nblk = lc_harvest_blocks(d.N);
    k_lc_wetcount<<<nblk, kLcHarvestBlock, 0, s>>>(d, c);
    k_lc_slots<<<1, 1024, 0, s>>>(nblk, c);
    k_lc_harvest<<<nblk, kLcHarvestBlock, 0, s>>>(d, c);
}
void launch_lc_judge(const Dev &d, const LcView &c, cudaStream_t s) {
    k_lc_judge<<<grid_for(d.N, 128), 128, 0, s>>>(d, c);
}

FESOMC_PREC_END
