// Learned vertical-mixing closure, the network side: FP32 training on the
// GPU with hand-written kernels (tiled SGEMM with fused bias / SiLU / SiLU'
// epilogues, squared-error loss, bias-gradient column sums, Adam), the FP32
// forward pass, and the training-set statistics (normalisation and the
// envelope the plain closure takes over outside of).  No counterpart in the
// reference; the network stands in for d3_end (src/fv_mixing.F90:73-347).
// The layout conventions are in closure.h.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "closure.h"
#include "mlp.h"

namespace fesomc {
namespace {

__device__ __forceinline__ float silu_f(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu_grad_f(float z) {
    const float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

enum { EPI_STORE = 0, EPI_BIAS = 1, EPI_BIAS_SILU = 2, EPI_SILU_GRAD = 3, EPI_SILU_ONLY = 4 };

// C[M x N] = op(A)[M x K] op(B)[K x N]: A(m,k) = TA ? A[k*lda+m] : A[m*lda+k],
// B(k,n) = TB ? B[n*ldb+k] : B[k*ldb+n].  64 x 64 tiles, 16-deep k slices in
// shared memory, 4 x 4 outputs per thread, FP32 with explicit fused
// multiply-adds.  Epilogues: store; + bias[n]; + bias[n] and SiLU (Z to C,
// SiLU(Z) to C2); times SiLU'(Zin[m,n]).
template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, const float *__restrict__ A, int lda,
                                              const float *__restrict__ B, int ldb, float *__restrict__ C, int ldc,
                                              const float *__restrict__ bias, float *__restrict__ C2,
                                              const float *__restrict__ Zin) {
    __shared__ __align__(16) float As[16][68];
    __shared__ __align__(16) float Bs[16][68];
    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
    for (int k0 = 0; k0 < K; k0 += 16) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int e = tid + r * 256;
            int mm, kk;
            if (TA) { mm = e % 64; kk = e / 64; }
            else { kk = e % 16; mm = e / 16; }
            const int gm = m0 + mm, gk = k0 + kk;
            float v = 0.0f;
            if (gm < M && gk < K) v = TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
            As[kk][mm] = v;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int e = tid + r * 256;
            int nn, kk;
            if (TB) { kk = e % 16; nn = e / 16; }
            else { nn = e % 64; kk = e / 64; }
            const int gn = n0 + nn, gk = k0 + kk;
            float v = 0.0f;
            if (gn < N && gk < K) v = TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
            Bs[kk][nn] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            const float4 a = *reinterpret_cast<const float4 *>(&As[kk][ty * 4]);
            const float4 b = *reinterpret_cast<const float4 *>(&Bs[kk][tx * 4]);
            const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gm = m0 + ty * 4 + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gn = n0 + tx * 4 + j;
            if (gn >= N) continue;
            float v = acc[i][j];
            const size_t o = (size_t)gm * ldc + gn;
            if (EPI == EPI_BIAS || EPI == EPI_BIAS_SILU || EPI == EPI_SILU_ONLY) v = v + bias[gn];
            if (EPI == EPI_SILU_GRAD) v = v * silu_grad_f(Zin[o]);
            if (EPI == EPI_SILU_ONLY) v = silu_f(v);
            C[o] = v;
            if (EPI == EPI_BIAS_SILU) C2[o] = silu_f(v);
        }
    }
}

template <bool TA, bool TB, int EPI>
void sgemm(cudaStream_t s, int M, int N, int K, const float *A, int lda, const float *B, int ldb, float *C, int ldc,
           const float *bias = nullptr, float *C2 = nullptr, const float *Zin = nullptr) {
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    k_sgemm<TA, TB, EPI><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, C2, Zin);
}

// delta = 2 (Y - T) / (B OUT) and the sum of squared residuals
__global__ void k_mse_delta(long long n, const float *Y, const float *T, float *D, float scale, double *loss) {
    double part = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float r = Y[i] - T[i];
        D[i] = 2.0f * r * scale;
        part += (double)r * (double)r;
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    __shared__ double sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        atomicAdd(loss, t);
    }
}

// column sums of D[B x N] in row chunks (deterministic: partials, then an
// ordered sum over the chunks)
constexpr int kColChunk = 512;
__global__ void k_colsum_part(int B, int N, const float *D, float *part) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (n >= N) return;
    const int r0 = c * kColChunk, r1 = min(B, r0 + kColChunk);
    float s = 0.0f;
    for (int r = r0; r < r1; ++r) s += D[(size_t)r * N + n];
    part[(size_t)c * N + n] = s;
}
__global__ void k_colsum_final(int nchunk, int N, const float *part, float *out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.0f;
    for (int c = 0; c < nchunk; ++c) s += part[(size_t)c * N + n];
    out[n] = s;
}

__global__ void k_adam(long long n, float *p, const float *g, float *m, float *v, float lr, float c1, float c2) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = 0.9f * m[i] + 0.1f * gi;
        const float vi = 0.999f * v[i] + 0.001f * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
    }
}

// minibatch: sample i of the batch is harvested column (a*(start+i) + c) mod
// n, an affine permutation of the training set per epoch; normalised on the
// way
__global__ void k_gather(int B, int W, const float *src, unsigned long long n, unsigned long long a,
                         unsigned long long c, unsigned long long start, const float *mu, const float *sd, float *dst) {
    const long long total = (long long)B * W;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e / W), j = (int)(e % W);
        // a, c < n < 2^31 and start + i < 2^31: the product fits in 64 bits
        const unsigned long long row = (a * (start + i) + c) % n;
        dst[e] = (src[row * W + j] - mu[j]) / sd[j];
    }
}

// per column j of data[n x W]: sum, sum of squares, min, max (FP64)
__global__ void k_colstats(unsigned long long n, int W, const float *data, double *out) {
    const int j = blockIdx.x;
    double s = 0.0, q = 0.0, lo = 1e300, hi = -1e300;
    for (unsigned long long r = threadIdx.x; r < n; r += blockDim.x) {
        const double v = data[r * W + j];
        s += v;
        q += v * v;
        lo = fmin(lo, v);
        hi = fmax(hi, v);
    }
    __shared__ double sh[4][256];
    sh[0][threadIdx.x] = s;
    sh[1][threadIdx.x] = q;
    sh[2][threadIdx.x] = lo;
    sh[3][threadIdx.x] = hi;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
            sh[2][threadIdx.x] = fmin(sh[2][threadIdx.x], sh[2][threadIdx.x + o]);
            sh[3][threadIdx.x] = fmax(sh[3][threadIdx.x], sh[3][threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) out[4 * j + k] = sh[k][0];
}

int grid_of(long long n, int block) {
    long long g = (n + block - 1) / block;
    return (int)std::max(1LL, std::min(g, 148LL * 16));
}

#define LCK(x)                                         \
    do {                                               \
        if ((x) != cudaSuccess) return FESOMC_ECUDA_LC; \
    } while (0)

}  // namespace

template <typename T>
static int lc_alloc(LcNet *n, T **p, size_t count) {
    void *q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return FESOMC_ENOMEM_LC;
    // zero fill on the legacy default stream, finished before the closure's
    // non-blocking stream may touch the buffer
    cudaMemset(q, 0, std::max<size_t>(count, 1) * sizeof(T));
    if (cudaDeviceSynchronize() != cudaSuccess) {
        cudaFree(q);
        return FESOMC_ECUDA_LC;
    }
    n->allocs.push_back(q);
    *p = static_cast<T *>(q);
    return 0;
}

LcNet *lc_create(int NS, long long hcap, unsigned long long seed, int Bmax, cudaStream_t s, int *rc) {
    *rc = 0;
    LcNet *n = new (std::nothrow) LcNet();
    if (!n) { *rc = FESOMC_ENOMEM_LC; return nullptr; }
    n->NS = NS;
    n->IN = lc_in(NS);
    n->OUT = lc_out(NS);
    n->dims[0] = n->IN;
    n->dims[1] = n->dims[2] = n->dims[3] = kLcHidden;
    n->dims[4] = n->OUT;
    long long o = 0;
    for (int l = 0; l < 4; ++l) {
        n->off[l] = o;
        o += (long long)n->dims[l + 1] * n->dims[l] + n->dims[l + 1];
    }
    n->np = o;
    n->Bmax = Bmax;
    n->hcap = hcap;
    n->stream = s;
    int r = 0;
    if ((r = lc_alloc(n, &n->params, n->np)) || (r = lc_alloc(n, &n->grads, n->np)) ||
        (r = lc_alloc(n, &n->mom, n->np)) || (r = lc_alloc(n, &n->var, n->np)) ||
        (r = lc_alloc(n, &n->stats, kLcStatRows * (size_t)std::max(n->IN, n->OUT))) || (r = lc_alloc(n, &n->dloss, 2)) ||
        (r = lc_alloc(n, &n->Xb, (size_t)Bmax * n->IN)) || (r = lc_alloc(n, &n->Tb, (size_t)Bmax * n->OUT)) ||
        (r = lc_alloc(n, &n->part, (size_t)((Bmax + kColChunk - 1) / kColChunk) * kLcHidden)) ||
        (r = lc_alloc(n, &n->hcount, 1)) || (hcap > 0 && ((r = lc_alloc(n, &n->hx, (size_t)hcap * n->IN)) ||
                                                          (r = lc_alloc(n, &n->hy, (size_t)hcap * n->OUT))))) {
        *rc = r;
        lc_free(n);
        return nullptr;
    }
    for (int l = 0; l < 4; ++l)
        if ((r = lc_alloc(n, &n->Z[l], (size_t)Bmax * kLcHidden)) || (r = lc_alloc(n, &n->A[l], (size_t)Bmax * kLcHidden)) ||
            (r = lc_alloc(n, &n->Dl[l], (size_t)Bmax * kLcHidden))) {
            *rc = r;
            lc_free(n);
            return nullptr;
        }
    // normalisation starts as the identity (mean 0, sd 1, envelope and
    // target range +-inf)
    std::vector<float> st(kLcStatRows * (size_t)std::max(n->IN, n->OUT));
    const int W = std::max(n->IN, n->OUT);
    for (int j = 0; j < W; ++j) {
        st[0 * W + j] = 0.0f; st[1 * W + j] = 1.0f; st[2 * W + j] = 0.0f; st[3 * W + j] = 1.0f;
        st[4 * W + j] = -INFINITY; st[5 * W + j] = INFINITY;
        st[6 * W + j] = -INFINITY; st[7 * W + j] = INFINITY;
    }
    cudaMemcpy(n->stats, st.data(), st.size() * sizeof(float), cudaMemcpyHostToDevice);
    // He-uniform weights (bound sqrt(6 / fan_in)), zero biases
    std::vector<float> p(n->np, 0.0f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < 4; ++l) {
        const int ni = n->dims[l], no = n->dims[l + 1];
        const float bound = std::sqrt(6.0f / (float)ni) * (l == 3 ? 0.5f : 1.0f);
        std::uniform_real_distribution<float> U(-bound, bound);
        for (long long i = 0; i < (long long)no * ni; ++i) p[n->off[l] + i] = U(rng);
    }
    cudaMemcpy(n->params, p.data(), p.size() * sizeof(float), cudaMemcpyHostToDevice);
    return n;
}

void lc_free(LcNet *n) {
    if (!n) return;
    for (void *p : n->allocs) cudaFree(p);
    delete n;
}

// forward pass of B <= Bmax normalised samples X (B x IN) into the batch
// buffers; the outputs are in A[3]'s slot Y = Z[3]
static void forward_batch(LcNet *n, const float *X, int B, float *Yout) {
    cudaStream_t s = n->stream;
    const float *in = X;
    for (int l = 0; l < 3; ++l) {
        const int ni = n->dims[l], no = n->dims[l + 1];
        sgemm<false, true, EPI_BIAS_SILU>(s, B, no, ni, in, ni, n->params + n->off[l], ni, n->Z[l], no,
                                         n->params + n->off[l] + (long long)no * ni, n->A[l]);
        in = n->A[l];
    }
    const int ni = n->dims[3], no = n->dims[4];
    sgemm<false, true, EPI_BIAS>(s, B, no, ni, in, ni, n->params + n->off[3], ni, Yout, no,
                                 n->params + n->off[3] + (long long)no * ni);
}

// forward pass over B columns at once (the model's step): activations in
// two caller buffers of B x 256, four launches on stream s
int lc_forward_full(const LcNet *n, const float *X, long long B, float *Y, float *bufA, float *bufB, cudaStream_t s) {
    const float *in = X;
    float *bufs[2] = {bufA, bufB};
    for (int l = 0; l < 3; ++l) {
        const int ni = n->dims[l], no = n->dims[l + 1];
        sgemm<false, true, EPI_SILU_ONLY>(s, (int)B, no, ni, in, ni, n->params + n->off[l], ni, bufs[l & 1], no,
                                          n->params + n->off[l] + (long long)no * ni);
        in = bufs[l & 1];
    }
    const int ni = n->dims[3], no = n->dims[4];
    sgemm<false, true, EPI_BIAS>(s, (int)B, no, ni, in, ni, n->params + n->off[3], ni, Y, no,
                                 n->params + n->off[3] + (long long)no * ni);
    return 0;
}

int lc_forward(LcNet *n, const float *X, long long B, float *Y) {
    for (long long b0 = 0; b0 < B; b0 += n->Bmax) {
        const int nb = (int)std::min<long long>(n->Bmax, B - b0);
        forward_batch(n, X + b0 * n->IN, nb, Y + b0 * n->OUT);
    }
    LCK(cudaGetLastError());
    return 0;
}

// loss and gradients of one batch (X, T normalised, B <= Bmax) into grads
static void grad_batch(LcNet *n, const float *X, const float *T, int B) {
    cudaStream_t s = n->stream;
    float *Y = n->Z[3];
    forward_batch(n, X, B, Y);
    const int OUT = n->OUT;
    const long long ny = (long long)B * OUT;
    float *D = n->Dl[3];
    k_mse_delta<<<grid_of(ny, 256), 256, 0, s>>>(ny, Y, T, D, 1.0f / (float)ny, n->dloss);
    const int nchunk = (B + kColChunk - 1) / kColChunk;
    for (int l = 3; l >= 0; --l) {
        const int ni = n->dims[l], no = n->dims[l + 1];
        const float *ain = (l == 0) ? X : n->A[l - 1];
        float *gW = n->grads + n->off[l], *gb = gW + (long long)no * ni;
        // gW = D^T A_in   (no x ni), gb = column sums of D
        sgemm<true, false, EPI_STORE>(s, no, ni, B, D, no, ain, ni, gW, ni);
        dim3 g((no + 255) / 256, nchunk);
        k_colsum_part<<<g, 256, 0, s>>>(B, no, D, n->part);
        k_colsum_final<<<(no + 255) / 256, 256, 0, s>>>(nchunk, no, n->part, gb);
        if (l > 0) {
            // D_prev = (D W) * SiLU'(Z_{l-1})
            float *Dp = n->Dl[l - 1];
            sgemm<false, false, EPI_SILU_GRAD>(s, B, ni, no, D, no, n->params + n->off[l], ni, Dp, ni, nullptr,
                                               nullptr, n->Z[l - 1]);
            D = Dp;
        }
    }
}

int lc_grad(LcNet *n, const float *X, const float *T, int B, double *loss) {
    if (B < 1 || B > n->Bmax) return FESOMC_EINVAL_LC;
    LCK(cudaMemsetAsync(n->dloss, 0, sizeof(double), n->stream));
    grad_batch(n, X, T, B);
    double h = 0.0;
    LCK(cudaMemcpyAsync(&h, n->dloss, sizeof(double), cudaMemcpyDeviceToHost, n->stream));
    LCK(cudaStreamSynchronize(n->stream));
    *loss = h / ((double)B * n->OUT);
    return 0;
}

int lc_fit_stats(LcNet *n) {
    unsigned long long cnt = 0;
    LCK(cudaMemcpy(&cnt, n->hcount, sizeof(cnt), cudaMemcpyDeviceToHost));
    cnt = std::min<unsigned long long>(cnt, (unsigned long long)n->hcap);
    if (cnt < 2) return FESOMC_ESTATE_LC;
    double *d = nullptr;
    const int W = std::max(n->IN, n->OUT);
    LCK(cudaMalloc(&d, sizeof(double) * 4 * (n->IN + n->OUT)));
    k_colstats<<<n->IN, 256, 0, n->stream>>>(cnt, n->IN, n->hx, d);
    k_colstats<<<n->OUT, 256, 0, n->stream>>>(cnt, n->OUT, n->hy, d + 4 * n->IN);
    std::vector<double> h(4 * (n->IN + n->OUT));
    cudaError_t e = cudaMemcpyAsync(h.data(), d, h.size() * sizeof(double), cudaMemcpyDeviceToHost, n->stream);
    cudaStreamSynchronize(n->stream);
    cudaFree(d);
    LCK(e);
    std::vector<float> st(kLcStatRows * (size_t)W, 0.0f);
    for (int j = 0; j < n->IN + n->OUT; ++j) {
        const double *q = &h[4 * j];
        const double mean = q[0] / cnt;
        const double var = std::max(0.0, q[1] / cnt - mean * mean);
        double sd = std::sqrt(var);
        if (!(sd > 1e-6 * (std::fabs(mean) + 1e-30)) || sd < 1e-12) sd = 1.0;   // constant input
        if (j < n->IN) {
            st[0 * W + j] = (float)mean;
            st[1 * W + j] = (float)sd;
            st[4 * W + j] = (float)((q[2] - mean) / sd);
            st[5 * W + j] = (float)((q[3] - mean) / sd);
        } else {
            st[2 * W + (j - n->IN)] = (float)mean;
            st[3 * W + (j - n->IN)] = (float)sd;
            st[6 * W + (j - n->IN)] = (float)q[2];
            st[7 * W + (j - n->IN)] = (float)q[3];
        }
    }
    n->h_stats = st;
    n->n_train = (long long)cnt;
    LCK(cudaMemcpy(n->stats, st.data(), st.size() * sizeof(float), cudaMemcpyHostToDevice));
    return 0;
}

int lc_train(LcNet *n, int epochs, int B, float lr, unsigned long long seed, float *losses) {
    if (B < 1 || B > n->Bmax || epochs < 0) return FESOMC_EINVAL_LC;
    const unsigned long long cnt = (unsigned long long)n->n_train;
    if (cnt < (unsigned long long)B) return FESOMC_ESTATE_LC;
    const int W = std::max(n->IN, n->OUT);
    const float *mu_x = n->stats, *sd_x = n->stats + W, *mu_y = n->stats + 2 * W, *sd_y = n->stats + 3 * W;
    std::mt19937_64 rng(seed);
    const long long nb = (long long)(cnt / B);
    n->tc_ready = false;   // the BF16 copies no longer match
    for (int ep = 0; ep < epochs; ++ep) {
        unsigned long long a;
        do { a = (rng() % cnt) | 1ULL; } while (std::gcd(a, cnt) != 1ULL);
        const unsigned long long c = rng() % cnt;
        LCK(cudaMemsetAsync(n->dloss, 0, sizeof(double), n->stream));
        for (long long b = 0; b < nb; ++b) {
            const unsigned long long start = (unsigned long long)b * B;
            k_gather<<<grid_of((long long)B * n->IN, 256), 256, 0, n->stream>>>(B, n->IN, n->hx, cnt, a, c, start,
                                                                                 mu_x, sd_x, n->Xb);
            k_gather<<<grid_of((long long)B * n->OUT, 256), 256, 0, n->stream>>>(B, n->OUT, n->hy, cnt, a, c, start,
                                                                                  mu_y, sd_y, n->Tb);
            grad_batch(n, n->Xb, n->Tb, B);
            n->adam_t += 1;
            const float c1 = 1.0f - std::pow(0.9f, (float)n->adam_t);
            const float c2 = 1.0f - std::pow(0.999f, (float)n->adam_t);
            k_adam<<<grid_of(n->np, 256), 256, 0, n->stream>>>(n->np, n->params, n->grads, n->mom, n->var, lr, c1, c2);
        }
        double h = 0.0;
        LCK(cudaMemcpyAsync(&h, n->dloss, sizeof(double), cudaMemcpyDeviceToHost, n->stream));
        LCK(cudaStreamSynchronize(n->stream));
        if (losses) losses[ep] = (float)(h / ((double)nb * B * n->OUT));
    }
    LCK(cudaGetLastError());
    return 0;
}

}  // namespace fesomc
